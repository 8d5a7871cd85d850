// Register-FFT kernels for the mixed-radix line lengths 144, 288, 432 (LineFFT3G with threads per line
// not a power of two): the instantiations of kwb_fast_impl.cuh's kernels for these lengths, in a
// translation unit of their own so that they compile alongside the others.
#include "kwb_fast_impl.cuh"

namespace kwb {

bool fast_mixed3_size(int N) { return N == 144 || N == 288 || N == 432; }

#define KWB_MIXED3_SWITCH(N, FN, ARGS)      \
  switch (N) {                             \
    case 144: return fast::FN<144> ARGS; \
    case 288: return fast::FN<288> ARGS; \
    case 432: return fast::FN<432> ARGS; \
    default: return cudaErrorInvalidValue; \
  }

static cudaError_t prime_eos_mixed3(int N) { KWB_MIXED3_SWITCH(N, prime_eos_n, ()) }
static cudaError_t prime_line_mixed3(int N) { KWB_MIXED3_SWITCH(N, prime_line, ()) }
cudaError_t fast_mixed3_prime(int N) {
  cudaError_t e = prime_eos_mixed3(N);
  return e != cudaSuccess ? e : prime_line_mixed3(N);
}
cudaError_t fast_mixed3_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                 cudaStream_t st) {
  KWB_MIXED3_SWITCH(h.N[axis], launch_line_n, (d_sim, h, axis, mode, s, st))
}
cudaError_t fast_mixed3_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  KWB_MIXED3_SWITCH(h.N[0], launch_eos_n, (d_sim, h, fwd, s, st))
}
cudaError_t fast_mixed3_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                            cudaStream_t st) {
  KWB_MIXED3_SWITCH(h.N[axis], launch_spec_n, (d_sim, h, axis, op, s, st))
}
cudaError_t fast_mixed3_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st) {
  KWB_MIXED3_SWITCH(h.N[axis], launch_el_n, (h, axis, g, s, st))
}

}  // namespace kwb
