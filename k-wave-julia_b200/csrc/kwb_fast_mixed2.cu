// Register-FFT kernels for the mixed-radix line lengths 80 (LineFFT3G, 20*2*2) and 384, 640, 768
// (LineFFT4G, 12*4*4*2, 20*4*4*2, 12*4*4*4): the instantiations of kwb_fast_impl.cuh's kernels for
// these lengths, in a translation unit of their own so that they compile alongside the others.
#include "kwb_fast_impl.cuh"

namespace kwb {

bool fast_mixed2_size(int N) { return N == 80 || N == 384 || N == 640 || N == 768; }

#define KWB_MIXED2_SWITCH(N, FN, ARGS)      \
  switch (N) {                             \
    case 80: return fast::FN<80> ARGS;     \
    case 384: return fast::FN<384> ARGS;   \
    case 640: return fast::FN<640> ARGS;   \
    case 768: return fast::FN<768> ARGS;   \
    default: return cudaErrorInvalidValue; \
  }

static cudaError_t prime_eos_mixed2(int N) { KWB_MIXED2_SWITCH(N, prime_eos_n, ()) }
static cudaError_t prime_line_mixed2(int N) { KWB_MIXED2_SWITCH(N, prime_line, ()) }
cudaError_t fast_mixed2_prime(int N) {
  cudaError_t e = prime_eos_mixed2(N);
  return e != cudaSuccess ? e : prime_line_mixed2(N);
}
cudaError_t fast_mixed2_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                 cudaStream_t st) {
  KWB_MIXED2_SWITCH(h.N[axis], launch_line_n, (d_sim, h, axis, mode, s, st))
}
cudaError_t fast_mixed2_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  KWB_MIXED2_SWITCH(h.N[0], launch_eos_n, (d_sim, h, fwd, s, st))
}
cudaError_t fast_mixed2_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                            cudaStream_t st) {
  KWB_MIXED2_SWITCH(h.N[axis], launch_spec_n, (d_sim, h, axis, op, s, st))
}
cudaError_t fast_mixed2_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st) {
  KWB_MIXED2_SWITCH(h.N[axis], launch_el_n, (h, axis, g, s, st))
}

}  // namespace kwb
