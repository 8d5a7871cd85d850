// Register-FFT kernels for the mixed-radix line lengths 96, 160, 192 and 320 (LineFFT3G, a 12-
// or 20-point register DFT as the first level): the instantiations of kwb_fast_impl.cuh's
// kernels for these lengths, in a translation unit of their own so that they compile alongside
// the power-of-two ones.
#include "kwb_fast_impl.cuh"

namespace kwb {

bool fast_mixed_size(int N) { return N == 96 || N == 160 || N == 192 || N == 320; }

#define KWB_MIXED_SWITCH(N, FN, ARGS)      \
  switch (N) {                             \
    case 96: return fast::FN<96> ARGS;     \
    case 160: return fast::FN<160> ARGS;   \
    case 192: return fast::FN<192> ARGS;   \
    case 320: return fast::FN<320> ARGS;   \
    default: return cudaErrorInvalidValue; \
  }

static cudaError_t prime_eos_mixed(int N) { KWB_MIXED_SWITCH(N, prime_eos_n, ()) }
static cudaError_t prime_line_mixed(int N) { KWB_MIXED_SWITCH(N, prime_line, ()) }
cudaError_t fast_mixed_prime(int N) {
  cudaError_t e = prime_eos_mixed(N);
  return e != cudaSuccess ? e : prime_line_mixed(N);
}
cudaError_t fast_mixed_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                 cudaStream_t st) {
  KWB_MIXED_SWITCH(h.N[axis], launch_line_n, (d_sim, h, axis, mode, s, st))
}
cudaError_t fast_mixed_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  KWB_MIXED_SWITCH(h.N[0], launch_eos_n, (d_sim, h, fwd, s, st))
}
cudaError_t fast_mixed_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                            cudaStream_t st) {
  KWB_MIXED_SWITCH(h.N[axis], launch_spec_n, (d_sim, h, axis, op, s, st))
}
cudaError_t fast_mixed_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st) {
  KWB_MIXED_SWITCH(h.N[axis], launch_el_n, (h, axis, g, s, st))
}

}  // namespace kwb
