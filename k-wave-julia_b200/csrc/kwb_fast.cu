// Register-resident FFT kernels for power-of-two line lengths N = E * G (64 ... 1024).
//
// Each line is owned by G threads; thread t holds the E elements x[t + G r] in registers.
// A forward transform is: an E-point DFT in registers (radix-2 decimation in frequency with
// compile-time twiddles), a multiply by exp(-2 pi i t q / N), one shared-memory transpose
// inside the line's thread group, and E/G G-point DFTs in registers.  Thread t then holds
// X[k] for k = t*(E/G) + j + E*m (j < E/G, m < G); the k-space multiplies index that layout
// directly and the inverse transform walks the same steps backwards, returning x[t + G r] to
// the thread that loaded it.  Field operands are loaded straight from HBM into registers
// (coalesced across threads) and prefetched ahead of the transform arithmetic.
//
// Same semantics as the generic shared-memory Stockham kernels (kwb_kernels.cu), which keep
// serving every other line length (radix 3/5/7 sizes) and the :stokes dispersion branch.
#include "kwb_fft.cuh"

namespace kwb {
namespace fast {

// cos(2 pi j/64) and sin(2 pi j/64), j = 0..31 (exact values to 17 significant digits)
__device__ constexpr float kCos64[32] = {
    1.0000000000000000e+00f, 9.9518472667219693e-01f, 9.8078528040323043e-01f, 9.5694033573220882e-01f,
    9.2387953251128674e-01f, 8.8192126434835505e-01f, 8.3146961230254524e-01f, 7.7301045336273699e-01f,
    7.0710678118654757e-01f, 6.3439328416364549e-01f, 5.5557023301960218e-01f, 4.7139673682599764e-01f,
    3.8268343236508978e-01f, 2.9028467725446233e-01f, 1.9509032201612825e-01f, 9.8017140329560604e-02f,
    0.0000000000000000e+00f, -9.8017140329560604e-02f, -1.9509032201612825e-01f, -2.9028467725446233e-01f,
    -3.8268343236508978e-01f, -4.7139673682599764e-01f, -5.5557023301960218e-01f, -6.3439328416364549e-01f,
    -7.0710678118654757e-01f, -7.7301045336273699e-01f, -8.3146961230254524e-01f, -8.8192126434835505e-01f,
    -9.2387953251128674e-01f, -9.5694033573220882e-01f, -9.8078528040323043e-01f, -9.9518472667219693e-01f};
__device__ constexpr float kSin64[32] = {
    0.0000000000000000e+00f, 9.8017140329560604e-02f, 1.9509032201612825e-01f, 2.9028467725446233e-01f,
    3.8268343236508978e-01f, 4.7139673682599764e-01f, 5.5557023301960218e-01f, 6.3439328416364549e-01f,
    7.0710678118654757e-01f, 7.7301045336273699e-01f, 8.3146961230254524e-01f, 8.8192126434835505e-01f,
    9.2387953251128674e-01f, 9.5694033573220882e-01f, 9.8078528040323043e-01f, 9.9518472667219693e-01f,
    1.0000000000000000e+00f, 9.9518472667219693e-01f, 9.8078528040323043e-01f, 9.5694033573220882e-01f,
    9.2387953251128674e-01f, 8.8192126434835505e-01f, 8.3146961230254524e-01f, 7.7301045336273699e-01f,
    7.0710678118654757e-01f, 6.3439328416364549e-01f, 5.5557023301960218e-01f, 4.7139673682599764e-01f,
    3.8268343236508978e-01f, 2.9028467725446233e-01f, 1.9509032201612825e-01f, 9.8017140329560604e-02f};

// x * exp(-+2 pi i j / 64), j a compile-time constant after unrolling
template <bool INV>
__device__ __forceinline__ float2 rot(float2 x, int j) {
  if (j == 0) return x;
  if (j == 16) return mul_mi<INV>(x);
  const float c = kCos64[j];
  const float s = INV ? -kSin64[j] : kSin64[j];
  return make_float2(fmaf(x.x, c, x.y * s), fmaf(x.y, c, -x.x * s));
}

template <int E>
__host__ __device__ constexpr int brev(int q) {
  int r = 0;
  for (int b = 1; b < E; b <<= 1) {
    r = (r << 1) | (q & 1);
    q >>= 1;
  }
  return r;
}

// E-point DFT in registers, natural order in and out (E a power of two, <= 64).
template <int E, bool INV>
__device__ __forceinline__ void dft_reg(float2 (&v)[E]) {
#pragma unroll
  for (int span = E / 2; span >= 1; span >>= 1) {
#pragma unroll
    for (int start = 0; start < E; start += 2 * span) {
#pragma unroll
      for (int k = 0; k < span; ++k) {
        const float2 a = v[start + k], b = v[start + k + span];
        v[start + k] = cadd(a, b);
        v[start + k + span] = rot<INV>(csub(a, b), k * (32 / span));
      }
    }
  }
  float2 t[E];
#pragma unroll
  for (int q = 0; q < E; ++q) t[q] = v[brev<E>(q)];
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = t[q];
}

__device__ __forceinline__ float2 cmul_conj(float2 a, float2 w) {  // a * conj(w)
  return make_float2(fmaf(a.x, w.x, a.y * w.y), fmaf(a.y, w.x, -a.x * w.y));
}

// N = E*G point transform of the line owned by this thread's group.  xs: the line's exchange
// buffer (E rows of pitch G+1); tw2: exp(-2 pi i t q/N) at [q*(G+1) + t].
template <int E, int G, bool WARP>
struct LineFFT {
  static constexpr int N = E * G, J = E / G, RP = G + 1, LP = E * RP + 1;
  static_assert(E % G == 0, "G must divide E");
  __device__ __forceinline__ static void sync() {
    if (WARP) __syncwarp();
    else __syncthreads();
  }
  // in: v[r] = x[t + G r]; out: v[j*G + m] = X[t*J + j + E*m]
  __device__ __forceinline__ static void fwd(float2 (&v)[E], float2 *xs, const float2 *tw2, int t) {
    dft_reg<E, false>(v);
#pragma unroll
    for (int q = 0; q < E; ++q) xs[q * RP + t] = cmul(v[q], tw2[q * RP + t]);
    sync();
#pragma unroll
    for (int j = 0; j < J; ++j) {
      float2 w[G];
#pragma unroll
      for (int u = 0; u < G; ++u) w[u] = xs[(t * J + j) * RP + u];
      dft_reg<G, false>(w);
#pragma unroll
      for (int m = 0; m < G; ++m) v[j * G + m] = w[m];
    }
    sync();
  }
  // in: v[j*G + m] = X[t*J + j + E*m]; out: v[r] = x[t + G r] (unnormalised)
  __device__ __forceinline__ static void inv(float2 (&v)[E], float2 *xs, const float2 *tw2, int t) {
#pragma unroll
    for (int j = 0; j < J; ++j) {
      float2 w[G];
#pragma unroll
      for (int m = 0; m < G; ++m) w[m] = v[j * G + m];
      dft_reg<G, true>(w);
      const int q = t * J + j;
#pragma unroll
      for (int u = 0; u < G; ++u) xs[q * RP + u] = cmul_conj(w[u], tw2[q * RP + u]);
    }
    sync();
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = xs[q * RP + t];
    dft_reg<E, true>(v);
    sync();
  }
  // frequency index held in register idx by thread t
  __device__ __forceinline__ static int k_of(int t, int idx) { return t * J + idx / G + E * (idx % G); }
};

// Build the per-CTA tables: tw2 (and, for line passes, the gradient multipliers in register order).
template <int E, int G>
__device__ __forceinline__ void build_tables(float2 *tw2, float2 *gp2, float2 *gn2, const float2 *tw,
                                             const float2 *gpos, const float2 *gneg) {
  constexpr int RP = G + 1, J = E / G;
  for (int e = threadIdx.x; e < E * G; e += blockDim.x) {
    const int q = e / G, u = e - q * G;
    tw2[q * RP + u] = tw[u * q];
    if (gp2) {
      const int k = u * J + q / G + E * (q % G);
      gp2[q * RP + u] = gpos[k];
      gn2[q * RP + u] = gneg[k];
    }
  }
}

template <int E, int G>
constexpr size_t line_smem(int L) {
  return ((size_t)L * (E * (G + 1) + 1) + 3 * (size_t)E * (G + 1)) * sizeof(float2);
}

// ------------------------------------------------------------------------------------------
// fused per-axis line pass (same algorithm as kwb::k_line_pass)
// ------------------------------------------------------------------------------------------

template <int E, int G, bool CONTIG>
__global__ void __launch_bounds__(KWB_THREADS)
    k_line_fast(const SimDev *__restrict__ sims, int axis, int mode, long long step_s) {
  using F = LineFFT<E, G, CONTIG>;
  constexpr int L = KWB_THREADS / G, RP = F::RP, LP = F::LP;
  extern __shared__ float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  float2 *gp2 = tw2 + E * RP;
  float2 *gn2 = gp2 + E * RP;
  const SimDev &S = sims[0];
  const long long t = *S.t0 + step_s;
  if (mode == KWB_MODE_STEP && t >= S.Nt) return;
  const int tid = threadIdx.x;
  const int tt = CONTIG ? tid % G : tid / L;
  const int l = CONTIG ? tid / G : tid % L;
  const int N = E * G;
  const int Nx = S.N[0];

  // tile geometry (as tile_x / tile_yz of the generic kernel, 2L real lines)
  long long base, stride;
  int cnt, first_line;
  if (CONTIG) {
    const int Ny = S.N[1];
    const int rows = 2 * L, tpp = (Ny + rows - 1) / rows;
    const int z = blockIdx.x / tpp, y0 = (blockIdx.x - z * tpp) * rows;
    cnt = min(rows, Ny - y0);
    base = ((long long)z * Ny + y0) * Nx;
    stride = 1;
    first_line = y0 + Ny * z;
  } else {
    const int cols = 2 * L, tpp = (Nx + cols - 1) / cols;
    const int o = blockIdx.x / tpp, x0 = (blockIdx.x - o * tpp) * cols;
    cnt = min(cols, Nx - x0);
    if (axis == 1) {
      base = (long long)o * Nx * S.N[1] + x0;
      stride = Nx;
    } else {
      base = (long long)o * Nx + x0;
      stride = (long long)Nx * S.N[1];
    }
    first_line = x0 + Nx * o;
  }
  const bool va = 2 * l < cnt, vb = 2 * l + 1 < cnt;
  const bool pair = !CONTIG && vb && ((stride & 1) == 0) && ((base & 1) == 0);
  auto addr = [&](int c, int i) -> long long {
    return CONTIG ? base + (long long)c * Nx + i : base + (long long)i * stride + c;
  };
  auto load_pair = [&](const float *__restrict__ f, int i) -> float2 {
    if (pair) return __ldg(reinterpret_cast<const float2 *>(f + addr(2 * l, i)));
    return make_float2(va ? __ldg(f + addr(2 * l, i)) : 0.f, vb ? __ldg(f + addr(2 * l + 1, i)) : 0.f);
  };
  auto store_pair = [&](float *f, int i, float2 v) {
    if (pair) {
      *reinterpret_cast<float2 *>(f + addr(2 * l, i)) = v;
      return;
    }
    if (va) f[addr(2 * l, i)] = v.x;
    if (vb) f[addr(2 * l + 1, i)] = v.y;
  };

  build_tables<E, G>(tw2, gp2, gn2, S.tw[axis], S.gpos[axis], S.gneg[axis]);
  float2 *xs = sm + l * LP;

  float2 v[E];
#pragma unroll
  for (int r = 0; r < E; ++r) v[r] = load_pair(S.p, tt + G * r);
  float *__restrict__ ud = S.u[axis];
  const float *__restrict__ rho0 = S.rho0;
  // operand prefetch ahead of the transform arithmetic (dropped for E = 32 to stay in registers)
  constexpr bool PF = E <= 16;
  float2 uu[PF ? E : 1];
  if (PF && mode == KWB_MODE_STEP) {
#pragma unroll
    for (int r = 0; r < E; ++r) uu[PF ? r : 0] = load_pair(ud, tt + G * r);
  }
  __syncthreads();  // tables

  // d/dx_d p  (staggered +)
  F::fwd(v, xs, tw2, tt);
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = cmul(v[q], gp2[q * RP + tt]);
  F::inv(v, xs, tw2, tt);

  // velocity update u = pml_sg (pml_sg u - dt/rho_sg dp)
  const float *__restrict__ esg = S.pml_sg_def[axis];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int i = tt + G * r;
    const int inext = (i + 1 == N) ? 0 : i + 1;
    float2 coef;
    if (rho0) {
      const float2 r0 = load_pair(rho0, i), r1 = load_pair(rho0, inext);
      coef = make_float2(S.dt / (0.5f * (r0.x + r1.x)), S.dt / (0.5f * (r0.y + r1.y)));
    } else {
      coef = make_float2(S.dt_over_rho0_s, S.dt_over_rho0_s);
    }
    float2 nv;
    if (mode == KWB_MODE_INIT) {
      nv = make_float2(-0.5f * coef.x * v[r].x, -0.5f * coef.y * v[r].y);
    } else {
      const float es = __ldg(esg + i);
      const float2 u0 = PF ? uu[PF ? r : 0] : load_pair(ud, i);
      float ta = fmaf(-es, u0.x, u0.x), tb = fmaf(-es, u0.y, u0.y);
      ta = fmaf(-coef.x, v[r].x, ta);
      tb = fmaf(-coef.y, v[r].y, tb);
      nv = make_float2(fmaf(-es, ta, ta), fmaf(-es, tb, tb));
    }
    v[r] = make_float2(va ? nv.x : 0.f, vb ? nv.y : 0.f);
  }

  if (mode == KWB_MODE_INIT) {
    float *__restrict__ rd = S.rho[axis];
    const float invD = 1.0f / (float)S.D;
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int i = tt + G * r;
      store_pair(ud, i, v[r]);
      const float2 pp = load_pair(S.p, i);
      float2 cs = S.c0sq ? load_pair(S.c0sq, i) : make_float2(S.c0sq_s, S.c0sq_s);
      store_pair(rd, i, make_float2(pp.x / ((float)S.D * cs.x), pp.y / ((float)S.D * cs.y)));
    }
    (void)invD;
    return;
  }

  // velocity sources on this tile's lines (first_order_steps.jl:586-617, 646-690)
  if (S.u_sig[axis] && S.u_line_ptr[axis]) {
    const int tcol = (int)(min(t + 1, (long long)S.u_cols[axis]) - 1);
    const int q0 = S.u_line_ptr[axis][first_line], q1 = S.u_line_ptr[axis][first_line + cnt];
    for (int q = q0; q < q1; ++q) {
      const SrcEntry se = S.u_entry[axis][q];
      const int c = se.line - first_line;
      if ((c >> 1) != l || (se.pos % G) != tt) continue;
      const int ro = se.pos / G;
      const float val = S.u_sig[axis][(long long)tcol * S.n_u + se.j];
#pragma unroll
      for (int r = 0; r < E; ++r)
        if (r == ro) {
          if (c & 1) v[r].y = (S.u_mode == 0) ? val : v[r].y + val;
          else v[r].x = (S.u_mode == 0) ? val : v[r].x + val;
        }
    }
  }
  float *__restrict__ rd = S.rho[axis];
  float2 rr[PF ? E : 1];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    store_pair(ud, tt + G * r, v[r]);
    if (PF) rr[PF ? r : 0] = load_pair(rd, tt + G * r);
  }

  // d/dx_d u_d  (staggered -)
  F::fwd(v, xs, tw2, tt);
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = cmul(v[q], gn2[q * RP + tt]);
  F::inv(v, xs, tw2, tt);

  // density update rho_d = pml (pml rho_d - dt rho0 du)
  const float *__restrict__ ed = S.pml_def[axis];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int i = tt + G * r;
    const float ei = __ldg(ed + i);
    float2 coef;
    if (rho0) {
      const float2 r0 = load_pair(rho0, i);
      coef = make_float2(S.dt * r0.x, S.dt * r0.y);
    } else {
      coef = make_float2(S.dt_rho0_s, S.dt_rho0_s);
    }
    const float2 r0d = PF ? rr[PF ? r : 0] : load_pair(rd, i);
    float ta = fmaf(-ei, r0d.x, r0d.x), tb = fmaf(-ei, r0d.y, r0d.y);
    ta = fmaf(-coef.x, v[r].x, ta);
    tb = fmaf(-coef.y, v[r].y, tb);
    v[r] = make_float2(fmaf(-ei, ta, ta), fmaf(-ei, tb, tb));
  }
  // pressure (mass) sources (first_order_steps.jl:619-640, 692-715)
  if (S.n_p > 0 && S.p_line_ptr[axis]) {
    const int tcol = (int)(min(t + 1, (long long)S.p_cols) - 1);
    const int q0 = S.p_line_ptr[axis][first_line], q1 = S.p_line_ptr[axis][first_line + cnt];
    for (int q = q0; q < q1; ++q) {
      const SrcEntry se = S.p_entry[axis][q];
      const int c = se.line - first_line;
      if ((c >> 1) != l || (se.pos % G) != tt) continue;
      const int ro = se.pos / G;
      const float val = S.p_sig[(long long)tcol * S.n_p + se.j];
#pragma unroll
      for (int r = 0; r < E; ++r)
        if (r == ro) {
          if (c & 1) v[r].y = (S.p_mode == 0) ? val : v[r].y + val;
          else v[r].x = (S.p_mode == 0) ? val : v[r].x + val;
        }
    }
  }
#pragma unroll
  for (int r = 0; r < E; ++r) store_pair(rd, tt + G * r, v[r]);
}

// ------------------------------------------------------------------------------------------
// equation of state: x R2C, y/z C2C with the multiply innermost, x C2R
// ------------------------------------------------------------------------------------------

template <int E, int G>
__global__ void __launch_bounds__(KWB_THREADS)
    k_eos_fwd_fast(const SimDev *__restrict__ sims, long long step_s) {
  using F = LineFFT<E, G, true>;
  constexpr int L = KWB_THREADS / G, LP = F::LP, N = E * G;
  extern __shared__ float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  const SimDev &S = sims[0];
  const long long t = *S.t0 + step_s;
  if (t >= S.Nt) return;
  const int tid = threadIdx.x, tt = tid % G, l = tid / G;
  const int Ny = S.N[1];
  const int rows = 2 * L, tpp = (Ny + rows - 1) / rows;
  const int z = blockIdx.x / tpp, y0 = (blockIdx.x - z * tpp) * rows;
  const int cnt = min(rows, Ny - y0);
  const long long base = ((long long)z * Ny + y0) * N;
  const bool va = 2 * l < cnt, vb = 2 * l + 1 < cnt;
  build_tables<E, G>(tw2, nullptr, nullptr, S.tw[0], nullptr, nullptr);
  float2 v[E];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int i = tt + G * r;
    float f[2] = {0.f, 0.f};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!(h ? vb : va)) continue;
      const long long a = base + (long long)(2 * l + h) * N + i;
      float rho = __ldg(S.rho[0] + a);
      if (S.D > 1) rho += __ldg(S.rho[1] + a);
      if (S.D > 2) rho += __ldg(S.rho[2] + a);
      if (S.nonlinear) rho = rho * fmaf(S.nlq ? __ldg(S.nlq + a) : S.nlq_s, rho, 1.0f);
      f[h] = S.c0sq ? __ldg(S.c0sq + a) * rho : rho;
    }
    v[r] = make_float2(f[0], f[1]);
  }
  __syncthreads();
  float2 *xs = sm + l * LP;
  F::fwd(v, xs, tw2, tt);
#pragma unroll
  for (int idx = 0; idx < E; ++idx) xs[F::k_of(tt, idx)] = v[idx];
  __syncwarp();
  const int n1 = S.n1;
  const long long rowa = (long long)z * Ny + y0 + 2 * l;
  for (int k = tt; k < n1; k += G) {
    const float2 zz = xs[k];
    const float2 zm = xs[k == 0 ? 0 : N - k];
    if (va) S.spec[rowa * n1 + k] = make_float2(0.5f * (zz.x + zm.x), 0.5f * (zz.y - zm.y));
    if (vb) S.spec[(rowa + 1) * n1 + k] = make_float2(0.5f * (zz.y + zm.y), -0.5f * (zz.x - zm.x));
  }
}

template <int E, int G>
__global__ void __launch_bounds__(KWB_THREADS)
    k_eos_inv_fast(const SimDev *__restrict__ sims, long long step_s) {
  using F = LineFFT<E, G, true>;
  constexpr int L = KWB_THREADS / G, LP = F::LP, N = E * G;
  extern __shared__ float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  const SimDev &S = sims[0];
  const long long t = *S.t0 + step_s;
  if (t >= S.Nt) return;
  const int tid = threadIdx.x, tt = tid % G, l = tid / G;
  const int Ny = S.N[1];
  const int rows = 2 * L, tpp = (Ny + rows - 1) / rows;
  const int z = blockIdx.x / tpp, y0 = (blockIdx.x - z * tpp) * rows;
  const int cnt = min(rows, Ny - y0);
  const long long base = ((long long)z * Ny + y0) * N;
  const bool va = 2 * l < cnt, vb = 2 * l + 1 < cnt;
  build_tables<E, G>(tw2, nullptr, nullptr, S.tw[0], nullptr, nullptr);
  float2 *xs = sm + l * LP;
  const int n1 = S.n1;
  const long long rowa = (long long)z * Ny + y0 + 2 * l;
  for (int k = tt; k < n1; k += G) {
    const float2 A = va ? S.spec[rowa * n1 + k] : make_float2(0.f, 0.f);
    const float2 B = vb ? S.spec[(rowa + 1) * n1 + k] : make_float2(0.f, 0.f);
    if (k == 0 || 2 * k == N) {
      xs[k] = make_float2(A.x, B.x);  // c2r ignores Im of the DC and Nyquist bins
    } else {
      xs[k] = make_float2(A.x - B.y, A.y + B.x);
      xs[N - k] = make_float2(A.x + B.y, B.x - A.y);
    }
  }
  __syncthreads();
  float2 v[E];
#pragma unroll
  for (int idx = 0; idx < E; ++idx) v[idx] = xs[F::k_of(tt, idx)];
  __syncwarp();
  F::inv(v, xs, tw2, tt);
  float *__restrict__ p = S.p;
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int i = tt + G * r;
    if (va) p[base + (long long)(2 * l) * N + i] = v[r].x;
    if (vb) p[base + (long long)(2 * l + 1) * N + i] = v[r].y;
  }
}

template <int E, int G>
__global__ void __launch_bounds__(KWB_THREADS)
    k_spec_fast(const SimDev *__restrict__ sims, int axis, int op, long long step_s) {
  using F = LineFFT<E, G, false>;
  constexpr int L = KWB_THREADS / G, LP = F::LP;
  extern __shared__ float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  const SimDev &S = sims[0];
  const long long t = *S.t0 + step_s;
  if (t >= S.Nt) return;
  const int tid = threadIdx.x, l = tid % L, tt = tid / L;
  const int n1 = S.n1, Ny = S.N[1];
  const int tpp = (n1 + L - 1) / L;
  const int o = blockIdx.x / tpp;
  const int k0 = (blockIdx.x - o * tpp) * L;
  const bool valid = k0 + l < n1;
  long long base, stride;
  if (axis == 1) {
    base = (long long)o * n1 * Ny + k0 + l;
    stride = n1;
  } else {
    base = (long long)o * n1 + k0 + l;
    stride = (long long)n1 * Ny;
  }
  build_tables<E, G>(tw2, nullptr, nullptr, S.tw[axis], nullptr, nullptr);
  float2 *xs = sm + l * LP;
  float2 *__restrict__ spec = S.spec;
  float2 v[E];
  if (op == KWB_SPEC_INV) {
#pragma unroll
    for (int idx = 0; idx < E; ++idx)
      v[idx] = valid ? spec[base + (long long)F::k_of(tt, idx) * stride] : make_float2(0.f, 0.f);
  } else {
#pragma unroll
    for (int r = 0; r < E; ++r) v[r] = valid ? spec[base + (long long)(tt + G * r) * stride] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  if (op == KWB_SPEC_INV) {
    F::inv(v, xs, tw2, tt);
  } else {
    F::fwd(v, xs, tw2, tt);
    if (op == KWB_SPEC_FWD) {
      if (valid) {
#pragma unroll
        for (int idx = 0; idx < E; ++idx) spec[base + (long long)F::k_of(tt, idx) * stride] = v[idx];
      }
      return;
    }
#pragma unroll
    for (int idx = 0; idx < E; ++idx) {
      const int k = F::k_of(tt, idx);
      const long long mi = (axis == 1) ? ((long long)o * Ny + k) * n1 + k0 + l
                                       : ((long long)k * Ny + o) * n1 + k0 + l;
      const float m = valid ? __ldg(S.M + mi) : 0.f;
      v[idx] = cscale(v[idx], m);
    }
    F::inv(v, xs, tw2, tt);
  }
  if (valid) {
#pragma unroll
    for (int r = 0; r < E; ++r) spec[base + (long long)(tt + G * r) * stride] = v[r];
  }
}

// ------------------------------------------------------------------------------------------
// dispatch
// ------------------------------------------------------------------------------------------

static int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

static cudaError_t raise_smem(const void *fn, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (bytes > (size_t)optin) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
}

template <int E, int G>
static cudaError_t prime_size() {
  cudaError_t e;
  const size_t ln = line_smem<E, G>(KWB_THREADS / G);
  if ((e = raise_smem((const void *)k_line_fast<E, G, true>, ln)) != cudaSuccess) return e;
  if ((e = raise_smem((const void *)k_line_fast<E, G, false>, ln)) != cudaSuccess) return e;
  if ((e = raise_smem((const void *)k_eos_fwd_fast<E, G>, ln)) != cudaSuccess) return e;
  if ((e = raise_smem((const void *)k_eos_inv_fast<E, G>, ln)) != cudaSuccess) return e;
  return raise_smem((const void *)k_spec_fast<E, G>, ln);
}

template <int E, int G>
static cudaError_t launch_line(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                               cudaStream_t st) {
  constexpr int L = KWB_THREADS / G;
  const size_t sm = line_smem<E, G>(L);
  if (axis == 0) {
    k_line_fast<E, G, true><<<cdiv(h.N[1], 2 * L) * h.N[2], KWB_THREADS, sm, st>>>(d_sim, axis, mode, s);
  } else {
    const int outer = axis == 1 ? h.N[2] : h.N[1];
    k_line_fast<E, G, false><<<cdiv(h.N[0], 2 * L) * outer, KWB_THREADS, sm, st>>>(d_sim, axis, mode, s);
  }
  return cudaGetLastError();
}

template <int E, int G>
static cudaError_t launch_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  constexpr int L = KWB_THREADS / G;
  const size_t sm = line_smem<E, G>(L);
  const int grid = cdiv(h.N[1], 2 * L) * h.N[2];
  if (fwd) k_eos_fwd_fast<E, G><<<grid, KWB_THREADS, sm, st>>>(d_sim, s);
  else k_eos_inv_fast<E, G><<<grid, KWB_THREADS, sm, st>>>(d_sim, s);
  return cudaGetLastError();
}

template <int E, int G>
static cudaError_t launch_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                               cudaStream_t st) {
  constexpr int L = KWB_THREADS / G;
  const size_t sm = line_smem<E, G>(L);
  const int grid = cdiv(h.n1, L) * (axis == 1 ? h.N[2] : h.N[1]);
  k_spec_fast<E, G><<<grid, KWB_THREADS, sm, st>>>(d_sim, axis, op, s);
  return cudaGetLastError();
}

}  // namespace fast

bool fast_size(int N) { return N == 64 || N == 128 || N == 256 || N == 512 || N == 1024; }

#define KWB_FAST_SWITCH(N, FN, ARGS)                                   \
  switch (N) {                                                         \
    case 64: return fast::FN<8, 8> ARGS;                               \
    case 128: return fast::FN<16, 8> ARGS;                             \
    case 256: return fast::FN<16, 16> ARGS;                            \
    case 512: return fast::FN<32, 16> ARGS;                            \
    case 1024: return fast::FN<32, 32> ARGS;                           \
    default: return cudaErrorInvalidValue;                             \
  }

cudaError_t fast_prime(int N) { KWB_FAST_SWITCH(N, prime_size, ()) }
cudaError_t fast_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                           cudaStream_t st) {
  KWB_FAST_SWITCH(h.N[axis], launch_line, (d_sim, h, axis, mode, s, st))
}
cudaError_t fast_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  KWB_FAST_SWITCH(h.N[0], launch_eos, (d_sim, h, fwd, s, st))
}
cudaError_t fast_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s, cudaStream_t st) {
  KWB_FAST_SWITCH(h.N[axis], launch_spec, (d_sim, h, axis, op, s, st))
}

}  // namespace kwb
