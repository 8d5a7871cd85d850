// Register-FFT kernels for power-of-two line lengths 64 ... 1024 and the cluster plane pass: the
// instantiations and the entry points the launchers call.  The kernel templates live in
// kwb_fast_impl.cuh; the mixed-radix lengths (3 * 2^k, 5 * 2^k) are instantiated in
// kwb_fast_mixed.cu.
#include "kwb_fast_impl.cuh"

namespace kwb {

bool fast_plane_size(int Ny, int Nz) { return Ny == 256 && Nz == 256; }
bool fast_plane_available() {
  static int n = -1;  // clusters that fit on the device at once (checked once per process)
  if (n < 0) n = fast::plane_clusters_per_device();
  return n > 0;
}
// Plane-pass variants usable on this device (1 or 2: the 16-CTA clusters need the non-portable
// cluster size).
int fast_plane_variants() {
  static int v = -1;
  if (v < 0) v = !fast_plane_available() ? 0 : (fast::plane_clusters_of<1>() > 0 ? 2 : 1);
  return v;
}
// Register-order slot -> k_y of the plane pass's y transform (the layout of its multiplier).
void fast_plane_slot_ky(int Ny, int *ky) {
  using F = fast::PlaneFY;
  for (int s = 0; s < Ny; ++s) ky[s] = F::k_of(s % F::G, s / F::G);
}
cudaError_t fast_plane(const SimDev *d_sim, const SimDev &h, long long s, cudaStream_t st) {
  (void)d_sim;
  const int v = h.tile_var[KWB_SLOT_PLANE] == 1 && fast_plane_variants() > 1 ? 1 : 0;
  return v == 1 ? fast::plane_launch<1>(h, s, st) : fast::plane_launch<0>(h, s, st);
}

bool fast_size(int N) {
  return N == 64 || N == 128 || N == 256 || N == 512 || N == 1024 || fast_mixed_size(N) || fast_mixed2_size(N) ||
         fast_mixed3_size(N) || fast_mixed4_size(N) || fast_mixed5_size(N);
}

#define KWB_LINE_SWITCH(N, FN, ARGS)       \
  switch (N) {                             \
    case 64: return fast::FN<64> ARGS;     \
    case 128: return fast::FN<128> ARGS;   \
    case 256: return fast::FN<256> ARGS;   \
    case 512: return fast::FN<512> ARGS;   \
    case 1024: return fast::FN<1024> ARGS; \
    default: return cudaErrorInvalidValue; \
  }

static cudaError_t prime_eos(int N) { KWB_LINE_SWITCH(N, prime_eos_n, ()) }
static cudaError_t prime_line(int N) { KWB_LINE_SWITCH(N, prime_line, ()) }
cudaError_t fast_prime(int N) {
  if (fast_mixed_size(N)) return fast_mixed_prime(N);
  if (fast_mixed2_size(N)) return fast_mixed2_prime(N);
  if (fast_mixed3_size(N)) return fast_mixed3_prime(N);
  if (fast_mixed4_size(N)) return fast_mixed4_prime(N);
  if (fast_mixed5_size(N)) return fast_mixed5_prime(N);
  cudaError_t e = prime_eos(N);
  return e != cudaSuccess ? e : prime_line(N);
}
cudaError_t fast_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                           cudaStream_t st) {
  if (fast_mixed_size(h.N[axis])) return fast_mixed_line_pass(d_sim, h, axis, mode, s, st);
  if (fast_mixed2_size(h.N[axis])) return fast_mixed2_line_pass(d_sim, h, axis, mode, s, st);
  if (fast_mixed3_size(h.N[axis])) return fast_mixed3_line_pass(d_sim, h, axis, mode, s, st);
  if (fast_mixed4_size(h.N[axis])) return fast_mixed4_line_pass(d_sim, h, axis, mode, s, st);
  if (fast_mixed5_size(h.N[axis])) return fast_mixed5_line_pass(d_sim, h, axis, mode, s, st);
  KWB_LINE_SWITCH(h.N[axis], launch_line_n, (d_sim, h, axis, mode, s, st))
}
cudaError_t fast_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  if (fast_mixed_size(h.N[0])) return fast_mixed_eos(d_sim, h, fwd, s, st);
  if (fast_mixed2_size(h.N[0])) return fast_mixed2_eos(d_sim, h, fwd, s, st);
  if (fast_mixed3_size(h.N[0])) return fast_mixed3_eos(d_sim, h, fwd, s, st);
  if (fast_mixed4_size(h.N[0])) return fast_mixed4_eos(d_sim, h, fwd, s, st);
  if (fast_mixed5_size(h.N[0])) return fast_mixed5_eos(d_sim, h, fwd, s, st);
  KWB_LINE_SWITCH(h.N[0], launch_eos_n, (d_sim, h, fwd, s, st))
}
cudaError_t fast_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s, cudaStream_t st) {
  if (fast_mixed_size(h.N[axis])) return fast_mixed_spec(d_sim, h, axis, op, s, st);
  if (fast_mixed2_size(h.N[axis])) return fast_mixed2_spec(d_sim, h, axis, op, s, st);
  if (fast_mixed3_size(h.N[axis])) return fast_mixed3_spec(d_sim, h, axis, op, s, st);
  if (fast_mixed4_size(h.N[axis])) return fast_mixed4_spec(d_sim, h, axis, op, s, st);
  if (fast_mixed5_size(h.N[axis])) return fast_mixed5_spec(d_sim, h, axis, op, s, st);
  KWB_LINE_SWITCH(h.N[axis], launch_spec_n, (d_sim, h, axis, op, s, st))
}
cudaError_t fast_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st) {
  if (fast_mixed_size(h.N[axis])) return fast_mixed_el_grad(h, axis, g, s, st);
  if (fast_mixed2_size(h.N[axis])) return fast_mixed2_el_grad(h, axis, g, s, st);
  if (fast_mixed3_size(h.N[axis])) return fast_mixed3_el_grad(h, axis, g, s, st);
  if (fast_mixed4_size(h.N[axis])) return fast_mixed4_el_grad(h, axis, g, s, st);
  if (fast_mixed5_size(h.N[axis])) return fast_mixed5_el_grad(h, axis, g, s, st);
  KWB_LINE_SWITCH(h.N[axis], launch_el_n, (h, axis, g, s, st))
}

}  // namespace kwb
