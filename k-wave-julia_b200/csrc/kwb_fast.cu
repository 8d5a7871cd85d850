// Register-FFT kernels for power-of-two line lengths 64 ... 1024 and the cluster plane pass: the
// instantiations and the entry points the launchers call.  The kernel templates live in
// kwb_fast_impl.cuh; the mixed-radix lengths (3 * 2^k, 5 * 2^k) are instantiated in
// kwb_fast_mixed.cu.
#include <mutex>

#include "kwb_fast_impl.cuh"

namespace kwb {

bool fast_plane_size(int Ny, int Nz) { return Ny == 256 && Nz == 256; }
bool fast_plane_available() {
  static int n = -1;  // clusters that fit on the device at once (checked once per process)
  if (n < 0) n = fast::plane_clusters_per_device();
  return n > 0;
}
// Plane-pass variants usable on this device, in the order the tuner tries them (their ids in
// ids[]; 16-CTA clusters need the non-portable cluster size).
int fast_plane_variants(int *ids) {
  static int n = -1, v[KWB_PLANE_VARIANTS];
  if (n < 0) {
    int k = 0;
    if (fast_plane_available()) {
      v[k++] = 0;
      if (fast::plane_clusters_of<2>() > 0) v[k++] = 2;
      if (fast::plane_clusters_of<1>() > 0) v[k++] = 1;
      if (fast::plane_clusters_of<3>() > 0) v[k++] = 3;
      if (fast::plane_clusters_of<4>() > 0) v[k++] = 4;
      if (fast::plane_clusters_of<5>() > 0) v[k++] = 5;
    }
    n = k;
  }
  if (ids)
    for (int i = 0; i < n; ++i) ids[i] = v[i];
  return n;
}
// The variant a simulation runs: its measured choice, else slot-major 8 x 512 (108 vs 112 µs per
// 256^3 launch for row-major 8 x 512, 117 and 127 µs for the 16-CTA shapes), else row-major.
static int plane_variant_of(const SimDev &h) {
  int ids[KWB_PLANE_VARIANTS];
  const int n = fast_plane_variants(ids);
  const int want = h.tile_var[KWB_SLOT_PLANE] >= 0 ? h.tile_var[KWB_SLOT_PLANE] : 2;
  for (int i = 0; i < n; ++i)
    if (ids[i] == want) return want;
  return 0;
}
// Shared-memory and cluster-size attributes of the usable variants on the current device (a
// function attribute is set per device).
template <int V>
static cudaError_t plane_prime_one() {
  using P = fast::PlaneVariant<V>;
  const void *fn = fast::plane_fn<V>();
  cudaError_t e = raise_dynamic_smem(fn, fast::plane_smem_of<V>());
  if (e == cudaSuccess && P::CL > 8) e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}
cudaError_t fast_plane_prime() {
  int ids[KWB_PLANE_VARIANTS];
  const int n = fast_plane_variants(ids);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    switch (ids[i]) {
      case 1: e = plane_prime_one<1>(); break;
      case 2: e = plane_prime_one<2>(); break;
      case 3: e = plane_prime_one<3>(); break;
      case 4: e = plane_prime_one<4>(); break;
      case 5: e = plane_prime_one<5>(); break;
      default: e = plane_prime_one<0>(); break;
    }
  }
  return e;
}
bool fast_plane_slot_major(const SimDev &h) { return h.plane && plane_variant_of(h) >= 2; }
// Register-order slot -> k_y of the plane pass's y transform (the layout of its multiplier).
void fast_plane_slot_ky(int Ny, int *ky) {
  using F = fast::PlaneFY;
  for (int s = 0; s < Ny; ++s) ky[s] = F::k_of(s % F::G, s / F::G);
}
// Register position j = t + 32 idx of the slot-major plane pass's z transform -> k_z.
void fast_plane_slot_kz(int Nz, int *kz) {
  using F = fast::PlaneFY;
  for (int j = 0; j < Nz; ++j) kz[j] = F::k_of(j % 32, j / 32);
}
cudaError_t fast_plane(const SimDev *d_sim, const SimDev &h, long long s, cudaStream_t st) {
  (void)d_sim;
  switch (plane_variant_of(h)) {
    case 1: return fast::plane_launch<1>(h, s, st);
    case 2: return fast::plane_launch<2>(h, s, st);
    case 3: return fast::plane_launch<3>(h, s, st);
    case 4: return fast::plane_launch<4>(h, s, st);
    case 5: return fast::plane_launch<5>(h, s, st);
    default: return fast::plane_launch<0>(h, s, st);
  }
}

// cuTensorMapEncodeTiled from the driver, looked up once (the library links only the runtime).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
  });
  return fn;
}

bool encode_strided_maps(SimDev &h, int axis, int cols) {
  const EncodeTiledFn enc = encode_tiled_fn();
  if (!enc || axis < 1 || axis > 2 || cols % 4 != 0 || h.N[0] % 4 != 0) return false;
  const int N = h.N[axis];
  int rows = 0;
  for (int k = (N + 255) / 256; k <= N && !rows; ++k)
    if (N % k == 0) rows = N / k;
  // each box and the second staged tile start on 128-byte boundaries of shared memory
  if (rows <= 0 || rows > 256 || (rows * cols * 4) % 128 != 0 || (N * cols * 4) % 128 != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)h.N[0], (cuuint64_t)h.N[1], (cuuint64_t)h.N[2]};
  const cuuint64_t strides[2] = {(cuuint64_t)h.N[0] * 4, (cuuint64_t)h.N[0] * h.N[1] * 4};
  const cuuint32_t box[3] = {(cuuint32_t)cols, (cuuint32_t)(axis == 1 ? rows : 1), (cuuint32_t)(axis == 2 ? rows : 1)};
  const cuuint32_t unit[3] = {1, 1, 1};
  const float *fields[4] = {h.p, h.rho0, h.u[axis], h.rho[axis]};
  for (int f = 0; f < 4; ++f) {
    if (!fields[f]) continue;
    if (enc(&h.tile_map[f], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(fields[f]), dims, strides, box,
            unit, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  h.tile_box_rows = rows;
  return true;
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
