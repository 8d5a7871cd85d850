// Register-FFT kernels for the mixed-radix line lengths 576, 864, 400 (LineFFT3G with threads per line
// not a power of two): the instantiations of kwb_fast_impl.cuh's kernels for these lengths, in a
// translation unit of their own so that they compile alongside the others.
#include "kwb_fast_impl.cuh"

namespace kwb {

bool fast_mixed4_size(int N) { return N == 576 || N == 864 || N == 400; }

#define KWB_MIXED4_SWITCH(N, FN, ARGS)      \
  switch (N) {                             \
    case 576: return fast::FN<576> ARGS; \
    case 864: return fast::FN<864> ARGS; \
    case 400: return fast::FN<400> ARGS; \
    default: return cudaErrorInvalidValue; \
  }

static cudaError_t prime_eos_mixed4(int N) { KWB_MIXED4_SWITCH(N, prime_eos_n, ()) }
static cudaError_t prime_line_mixed4(int N) { KWB_MIXED4_SWITCH(N, prime_line, ()) }
cudaError_t fast_mixed4_prime(int N) {
  cudaError_t e = prime_eos_mixed4(N);
  return e != cudaSuccess ? e : prime_line_mixed4(N);
}
cudaError_t fast_mixed4_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                 cudaStream_t st) {
  KWB_MIXED4_SWITCH(h.N[axis], launch_line_n, (d_sim, h, axis, mode, s, st))
}
cudaError_t fast_mixed4_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  KWB_MIXED4_SWITCH(h.N[0], launch_eos_n, (d_sim, h, fwd, s, st))
}
cudaError_t fast_mixed4_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                            cudaStream_t st) {
  KWB_MIXED4_SWITCH(h.N[axis], launch_spec_n, (d_sim, h, axis, op, s, st))
}
cudaError_t fast_mixed4_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st) {
  KWB_MIXED4_SWITCH(h.N[axis], launch_el_n, (h, axis, g, s, st))
}

}  // namespace kwb
