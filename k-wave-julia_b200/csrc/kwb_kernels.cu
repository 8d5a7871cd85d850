// Time-step kernels of libkwb.
//
// One time step of KWave.jl's time_step_{1,2,3}d! (KWave.jl/src/solver/first_order_steps.jl:
// 296-535) is executed as:
//
//   [k_tr_inject]                      time-reversal injection (first_order.jl:450-460, 678-689)
//   k_line_pass(axis) for every axis   fused: d/dx_d p -> u_d update (split PML) -> u source ->
//                                      d/dx_d u_d -> rho_d update (split PML) -> p source
//                                      (first_order_steps.jl:400-428, 489-521, 586-715)
//   k_eos_x_fwd                        EOS prologue (sum rho_d, nonlinearity, c^2) + x R2C
//   k_spec_pass(y [,z])                y/z FFTs of the half spectrum, EOS multiply innermost
//   k_eos_x_inv                        x C2R -> p                  (first_order_steps.jl:214-290)
//   k_sensor_gather per sensor group   record_sensor_data!         (first_order_steps.jl:728-811)
//
// The gradient along axis d is computed on lines along d only: a full N-D rfft, a multiply by
// i k_d e^{+-i k_d d/2} and an N-D irfft (fft_utils.jl:247-303) equal the 1-D transform along
// d, because the multiplier is Hermitian (it is real at the Nyquist bin).  Two real lines are
// transformed as one complex line (a + i b) for the same reason.
#include <algorithm>
#include <map>
#include <mutex>

#include "kwb_fft.cuh"
#include "kwb_tiles.cuh"

namespace kwb {

// ------------------------------------------------------------------------------------------
// fused per-axis line pass
// ------------------------------------------------------------------------------------------

template <bool CONTIG>
__global__ void __launch_bounds__(KWB_PASS_THREADS_MAX)
    k_line_pass(const SimDev *__restrict__ sims, int axis, int mode, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  extern __shared__ float4 smem_raw[];
  float2 *smem = reinterpret_cast<float2 *>(smem_raw);
  const SimDev &S = sims[0];
  const long long t = step_index(S, step_s);
  if (mode == KWB_MODE_STEP && t >= S.Nt) return;

  const int N = S.N[axis];
  const int L = S.L_line[axis];
  const int LS = line_pitch(fft_len(S.plan[axis]));
  const int Nx = S.N[0];
  float2 *X = smem;
  float2 *Y = X + L * LS;
  float2 *tw = Y + L * LS;
  const Tile T = CONTIG ? tile_x(S, 2 * L, blockIdx.x) : tile_yz(S, axis, 2 * L, blockIdx.x);
  auto addr = [&](int c, int i) -> long long {
    return CONTIG ? T.base + (long long)c * Nx + i : T.base + (long long)i * T.stride + c;
  };
  auto decode = [&](int e, int &l, int &i) {
    if (CONTIG) {
      l = e / N;
      i = e - l * N;
    } else {
      i = e / L;
      l = e - i * L;
    }
  };
  const int total = L * N;
  load_twiddles(tw, S.tw[axis], fft_len(S.plan[axis]));
  {
    const float *__restrict__ p = S.p;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int l, i;
      decode(e, l, i);
      const int ca = 2 * l, cb = 2 * l + 1;
      const float a = ca < T.cnt ? p[addr(ca, i)] : 0.f;
      const float b = cb < T.cnt ? p[addr(cb, i)] : 0.f;
      X[l * LS + i] = make_float2(a, b);
    }
  }
  __syncthreads();

  // d/dx_d p  (staggered +)
  float2 *R = fft_lines<false>(X, Y, L, LS, S.plan[axis], tw);
  float2 *F = (R == X) ? Y : X;
  {
    const float2 *__restrict__ g = S.gpos[axis];
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = e / N, i = e - l * N;
      R[l * LS + i] = cmul(R[l * LS + i], g[i]);
    }
  }
  __syncthreads();
  float2 *Dp = fft_lines<true>(R, F, L, LS, S.plan[axis], tw);
  float2 *Fp = (Dp == R) ? F : R;

  // velocity update u = pml_sg (pml_sg u - dt/rho_sg dp), with pml = 1 - deficit
  float *__restrict__ ud = S.u[axis];
  const float *__restrict__ rho0 = S.rho0;
  {
    const float *__restrict__ esg = S.pml_sg_def[axis];
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int l, i;
      decode(e, l, i);
      const float2 g = Dp[l * LS + i];
      const int inext = (i + 1 == N) ? 0 : i + 1;
      const float es = esg[i];
      float out[2] = {0.f, 0.f};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = 2 * l + h;
        if (c >= T.cnt) continue;
        const long long ad = addr(c, i);
        float coef;
        if (rho0) {
          const float rsg = 0.5f * (rho0[ad] + rho0[addr(c, inext)]);
          coef = S.dt / rsg;
        } else {
          coef = S.dt_over_rho0_s;
        }
        const float dp = h ? g.y : g.x;
        float v;
        if (mode == KWB_MODE_INIT) {
          v = -0.5f * coef * dp;  // u(-dt/2) = -dt/(2 rho_sg) dp0  (first_order_steps.jl:128-136)
        } else {
          const float u0 = ud[ad];
          float t1 = fmaf(-es, u0, u0);
          t1 = fmaf(-coef, dp, t1);
          v = fmaf(-es, t1, t1);
        }
        ud[ad] = v;
        out[h] = v;
      }
      Dp[l * LS + i] = make_float2(out[0], out[1]);
    }
  }

  if (mode == KWB_MODE_INIT) {
    // rho_d = p0 / (D c0^2)   (first_order_steps.jl:77, 117-118, 165-167)
    float *__restrict__ rd = S.rho[axis];
    const float *__restrict__ p = S.p;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int l, i;
      decode(e, l, i);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = 2 * l + h;
        if (c >= T.cnt) continue;
        const long long ad = addr(c, i);
        const float csq = S.c0sq ? S.c0sq[ad] : S.c0sq_s;
        rd[ad] = p[ad] / ((float)S.D * csq);
      }
    }
    return;
  }

  // velocity sources on the lines of this tile (first_order_steps.jl:586-617, 646-690)
  const int tcol_u = S.u_sig[axis] ? (int)(min(t + 1, (long long)S.u_cols[axis]) - 1) : 0;
  if (S.u_sig[axis] && S.u_line_ptr[axis]) {
    __syncthreads();
    const int q0 = S.u_line_ptr[axis][T.first_line];
    const int q1 = S.u_line_ptr[axis][T.first_line + T.cnt];
    for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
      const SrcEntry se = S.u_entry[axis][q];
      const int c = se.line - T.first_line;
      float *cell = reinterpret_cast<float *>(&Dp[(c >> 1) * LS + se.pos]) + (c & 1);
      const float val = S.u_sig[axis][(long long)tcol_u * S.n_u + se.j];
      const float nv = (S.u_mode == 0) ? val : *cell + val;
      *cell = nv;
      ud[addr(c, se.pos)] = nv;
    }
  }
  __syncthreads();

  // d/dx_d u_d  (staggered -)
  float2 *R2 = fft_lines<false>(Dp, Fp, L, LS, S.plan[axis], tw);
  float2 *F2 = (R2 == Dp) ? Fp : Dp;
  {
    const float2 *__restrict__ g = S.gneg[axis];
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = e / N, i = e - l * N;
      R2[l * LS + i] = cmul(R2[l * LS + i], g[i]);
    }
  }
  __syncthreads();
  float2 *Du = fft_lines<true>(R2, F2, L, LS, S.plan[axis], tw);

  // density update rho_d = pml (pml rho_d - dt rho0 du)
  float *__restrict__ rd = S.rho[axis];
  {
    const float *__restrict__ ed = S.pml_def[axis];
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int l, i;
      decode(e, l, i);
      const float2 g = Du[l * LS + i];
      const float ei = ed[i];
      float out[2] = {0.f, 0.f};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = 2 * l + h;
        if (c >= T.cnt) continue;
        const long long ad = addr(c, i);
        const float coef = rho0 ? S.dt * rho0[ad] : S.dt_rho0_s;
        const float r0 = rd[ad];
        float du = h ? g.y : g.x;
        if (axis == 1 && S.inv_r) du = fmaf(ud[ad], S.inv_r[i], du);  // + u_r / r (axisymmetric.jl:183)
        float t1 = fmaf(-ei, r0, r0);
        t1 = fmaf(-coef, du, t1);
        const float v = fmaf(-ei, t1, t1);
        rd[ad] = v;
        out[h] = v;
      }
      Du[l * LS + i] = make_float2(out[0], out[1]);
    }
  }

  // pressure (mass) sources: rho_d (+)= p / (D c^2)   (first_order_steps.jl:619-640, 692-715)
  if (S.n_p > 0 && S.p_line_ptr[axis]) {
    __syncthreads();
    const int tcol = (int)(min(t + 1, (long long)S.p_cols) - 1);
    const int q0 = S.p_line_ptr[axis][T.first_line];
    const int q1 = S.p_line_ptr[axis][T.first_line + T.cnt];
    for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
      const SrcEntry se = S.p_entry[axis][q];
      const int c = se.line - T.first_line;
      float *cell = reinterpret_cast<float *>(&Du[(c >> 1) * LS + se.pos]) + (c & 1);
      const float val = S.p_sig[(long long)tcol * S.n_p + se.j];
      const float nv = (S.p_mode == 0) ? val : *cell + val;
      *cell = nv;
      rd[addr(c, se.pos)] = nv;
    }
  }
}

// ------------------------------------------------------------------------------------------
// equation of state
// ------------------------------------------------------------------------------------------

// EOS input per voxel: f = [c0^2] rho_eff, rho_eff = rho (1 + Q rho), Q = BonA / (2 rho0)
// (first_order_steps.jl:236-241, 275-279)
__device__ __forceinline__ float eos_rho_total(const SimDev &S, long long v) {
  float r = S.rho[0][v];
  if (S.D > 1) r += S.rho[1][v];
  if (S.D > 2) r += S.rho[2][v];
  return r;
}

__device__ __forceinline__ float eos_effective(const SimDev &S, long long v, float r) {
  if (S.nonlinear) {
    const float q = S.nlq ? S.nlq[v] : S.nlq_s;
    r = r * fmaf(q, r, 1.0f);
  }
  return r;
}

__global__ void __launch_bounds__(KWB_THREADS)
    k_eos_x_fwd(const SimDev *__restrict__ sims, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  extern __shared__ float4 smem_raw[];
  float2 *smem = reinterpret_cast<float2 *>(smem_raw);
  const SimDev &S = sims[0];
  const long long t = step_index(S, step_s);
  if (t >= S.Nt) return;
  const int N = S.N[0];
  const int L = S.L_eosx;
  const int LS = line_pitch(fft_len(S.plan[0]));
  const int two = S.dispersion;
  const int LL = two ? 2 * L : L;
  float2 *X = smem;
  float2 *Y = X + LL * LS;
  float2 *tw = Y + LL * LS;
  const Tile T = tile_x(S, 2 * L, blockIdx.x);
  const int total = L * N;
  load_twiddles(tw, S.tw[0], fft_len(S.plan[0]));
  const float inv_dt = 1.0f / S.dt;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int l = e / N, i = e - l * N;
    float f[2] = {0.f, 0.f}, f2[2] = {0.f, 0.f};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = 2 * l + h;
      if (c >= T.cnt) continue;
      const long long v = T.base + (long long)c * N + i;
      const float r = eos_rho_total(S, v);
      const float re = eos_effective(S, v, r);
      f[h] = S.c0sq ? S.c0sq[v] * re : re;
      if (two) {
        // dispersion term (rho_eff - rho_eff_prev)/dt; rho_prev keeps plain rho_total
        // (first_order_steps.jl:255-263, 436-440)
        const float rp = S.rho_prev[v];
        f2[h] = (re - eos_effective(S, v, rp)) * inv_dt;
        S.rho_prev[v] = r;
      }
    }
    X[l * LS + i] = make_float2(f[0], f[1]);
    if (two) X[(L + l) * LS + i] = make_float2(f2[0], f2[1]);
  }
  __syncthreads();
  float2 *R = fft_lines<false>(X, Y, LL, LS, S.plan[0], tw);
  // split the two packed real rows: A_k = (Z_k + conj Z_-k)/2, B_k = (Z_k - conj Z_-k)/(2i)
  const int n1 = S.n1;
  const int Ny = S.N[1];
  for (int e = threadIdx.x; e < L * n1; e += blockDim.x) {
    const int l = e / n1, k = e - l * n1;
    const int km = (k == 0) ? 0 : N - k;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      if (s == 1 && !two) break;
      float2 *out = s ? S.spec2 : S.spec;
      const float2 z = R[(s * L + l) * LS + k];
      const float2 zm = R[(s * L + l) * LS + km];
      const float2 A = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
      const float2 B = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
      const int ca = 2 * l, cb = 2 * l + 1;
      const long long rowa = (long long)T.outer * Ny + T.y0 + ca;
      if (ca < T.cnt) out[rowa * n1 + k] = A;
      if (cb < T.cnt) out[(rowa + 1) * n1 + k] = B;
    }
  }
}

__global__ void __launch_bounds__(KWB_THREADS)
    k_eos_x_inv(const SimDev *__restrict__ sims, long long step_s, int mul_x) {
  KWB_STEP_KERNEL_PROLOGUE();
  extern __shared__ float4 smem_raw[];
  float2 *smem = reinterpret_cast<float2 *>(smem_raw);
  const SimDev &S = sims[0];
  const long long t = step_index(S, step_s);
  if (t >= S.Nt) return;
  const int N = S.N[0];
  const int L = S.L_eosx;
  const int LS = line_pitch(fft_len(S.plan[0]));
  float2 *X = smem;
  float2 *Y = X + L * LS;
  float2 *tw = Y + L * LS;
  const Tile T = tile_x(S, 2 * L, blockIdx.x);
  const int n1 = S.n1;
  const int Ny = S.N[1];
  load_twiddles(tw, S.tw[0], fft_len(S.plan[0]));
  const bool even = (N & 1) == 0;
  for (int e = threadIdx.x; e < L * n1; e += blockDim.x) {
    const int l = e / n1, k = e - l * n1;
    const int ca = 2 * l, cb = 2 * l + 1;
    const long long rowa = (long long)T.outer * Ny + T.y0 + ca;
    float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
    if (ca < T.cnt) {
      A = S.spec[rowa * n1 + k];
      if (mul_x) {
        const float m = S.M[rowa * n1 + k];
        A = cscale(A, m);
        if (S.dispersion) {
          const float m2 = S.M2[rowa * n1 + k];
          const float2 A2 = S.spec2[rowa * n1 + k];
          A = make_float2(fmaf(-m2, A2.x, A.x), fmaf(-m2, A2.y, A.y));
        }
      }
    }
    if (cb < T.cnt) {
      B = S.spec[(rowa + 1) * n1 + k];
      if (mul_x) {
        const float m = S.M[(rowa + 1) * n1 + k];
        B = cscale(B, m);
        if (S.dispersion) {
          const float m2 = S.M2[(rowa + 1) * n1 + k];
          const float2 B2 = S.spec2[(rowa + 1) * n1 + k];
          B = make_float2(fmaf(-m2, B2.x, B.x), fmaf(-m2, B2.y, B.y));
        }
      }
    }
    float2 *x = X + l * LS;
    if (k == 0 || (even && 2 * k == N)) {
      // c2r ignores the imaginary part of the DC and Nyquist bins
      x[k] = make_float2(A.x, B.x);
    } else {
      x[k] = make_float2(A.x - B.y, A.y + B.x);
      x[N - k] = make_float2(A.x + B.y, B.x - A.y);
    }
  }
  __syncthreads();
  float2 *R = fft_lines<true>(X, Y, L, LS, S.plan[0], tw);
  float *__restrict__ p = S.p;
  for (int e = threadIdx.x; e < L * N; e += blockDim.x) {
    const int l = e / N, i = e - l * N;
    const float2 z = R[l * LS + i];
    const int ca = 2 * l, cb = 2 * l + 1;
    if (ca < T.cnt) p[T.base + (long long)ca * N + i] = z.x;
    if (cb < T.cnt) p[T.base + (long long)cb * N + i] = z.y;
  }
}

// y- or z-direction FFTs of the half spectrum (complex columns kx0..kx0+L-1)
__global__ void __launch_bounds__(KWB_THREADS)
    k_spec_pass(const SimDev *__restrict__ sims, int axis, int op, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  extern __shared__ float4 smem_raw[];
  float2 *smem = reinterpret_cast<float2 *>(smem_raw);
  const SimDev &S = sims[0];
  const long long t = step_index(S, step_s);
  if (t >= S.Nt) return;
  const int N = S.N[axis];
  const int L = S.L_spec[axis];
  const int LS = line_pitch(fft_len(S.plan[axis]));
  const int two = S.dispersion && op != KWB_SPEC_INV;
  const int LL = two ? 2 * L : L;
  float2 *X = smem;
  float2 *Y = X + LL * LS;
  float2 *tw = Y + LL * LS;
  const int n1 = S.n1, Ny = S.N[1];
  const int tpp = (n1 + L - 1) / L;
  const int o = blockIdx.x / tpp;
  const int k0 = (blockIdx.x - o * tpp) * L;
  const int cnt = min(L, n1 - k0);
  long long base, stride;
  if (axis == 1) {
    base = (long long)o * n1 * Ny + k0;
    stride = n1;
  } else {
    base = (long long)o * n1 + k0;
    stride = (long long)n1 * Ny;
  }
  load_twiddles(tw, S.tw[axis], fft_len(S.plan[axis]));
  const int total = L * N;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int i = e / L, l = e - i * L;
    const long long a = base + (long long)i * stride + l;
    X[l * LS + i] = l < cnt ? S.spec[a] : make_float2(0.f, 0.f);
    if (two) X[(L + l) * LS + i] = l < cnt ? S.spec2[a] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2 *R;
  if (op == KWB_SPEC_INV) {
    R = fft_lines<true>(X, Y, L, LS, S.plan[axis], tw);
  } else {
    R = fft_lines<false>(X, Y, LL, LS, S.plan[axis], tw);
    if (op == KWB_SPEC_FWD_MUL_INV) {
      float2 *F = (R == X) ? Y : X;
      for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int i = e / L, l = e - i * L;
        // multiplier index in [Nz][Ny][n1]
        const long long mi = (axis == 1) ? ((long long)o * Ny + i) * n1 + k0 + l
                                         : ((long long)i * Ny + o) * n1 + k0 + l;
        if (l >= cnt) continue;
        float2 a = cscale(R[l * LS + i], S.M[mi]);
        if (two) {
          const float2 b = R[(L + l) * LS + i];
          const float m2 = S.M2[mi];
          a = make_float2(fmaf(-m2, b.x, a.x), fmaf(-m2, b.y, a.y));
        }
        R[l * LS + i] = a;
      }
      __syncthreads();
      R = fft_lines<true>(R, F, L, LS, S.plan[axis], tw);
    }
  }
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int i = e / L, l = e - i * L;
    if (l >= cnt) continue;
    const long long a = base + (long long)i * stride + l;
    S.spec[a] = R[l * LS + i];
    if (two && op == KWB_SPEC_FWD) S.spec2[a] = R[(L + l) * LS + i];
  }
}

// ------------------------------------------------------------------------------------------
// time reversal, sensors, control
// ------------------------------------------------------------------------------------------

__global__ void k_tr_inject(const SimDev *__restrict__ sims, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  const SimDev &S = sims[0];
  const long long t = step_index(S, step_s);
  if (t >= S.Nt) return;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= S.n_tr) return;
  const long long col = S.Nt - 1 - t;  // tr_t = Nt - t_index + 1 (1-based)
  const float val = S.tr_sig[col * S.n_tr + j];
  const long long v = S.tr_idx[j];
  for (int d = 0; d < S.D; ++d) S.rho[d][v] = val;
}

__global__ void k_sensor_gather(const SimDev *__restrict__ sims, const GroupDev *__restrict__ gp,
                                long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  const SimDev &S = sims[0];
  const long long t = step_index(S, step_s);
  if (t >= S.Nt) return;
  const GroupDev &g = *gp;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.n) return;
  const long long v = g.dense ? j : g.idx[j];
  const unsigned m = g.mask;
  const float pv = S.p[v];
  const bool last = (t == S.Nt - 1);
  if (m & (1u << 0)) g.ser_p[t * g.n + j] = pv;
  if (m & (1u << 1)) g.pmax[j] = fmaxf(g.pmax[j], pv);
  if (m & (1u << 2)) g.pmin[j] = fminf(g.pmin[j], pv);
  if (m & (1u << 3)) g.prms[j] += (double)g.cnt_prms * ((double)pv * (double)pv);
  if ((m & (1u << 4)) && last) g.pfinal[j] = pv;
  const unsigned umask = (7u << 5) | (63u << 8);
  if (m & umask) {
    float uv[3] = {0.f, 0.f, 0.f};
    for (int d = 0; d < S.ndim; ++d) uv[d] = S.u[d][v];
    for (int d = 0; d < S.ndim; ++d)
      if (m & (1u << (5 + d))) g.ser_u[d][t * g.n + j] = uv[d];
    double mag2 = 0.0, i2 = 0.0;
    for (int d = 0; d < S.ndim; ++d) {
      mag2 += (double)uv[d] * (double)uv[d];
      const double pu = (double)pv * (double)uv[d];
      i2 += pu * pu;
    }
    const double mag = sqrt(mag2);
    if (m & (1u << 8)) g.umax[j] = fmax(g.umax[j], mag);
    if (m & (1u << 9)) g.urms[j] += (double)g.cnt_urms * mag2;
    if ((m & (1u << 10)) && last) g.ufinal[j] = mag;
    if (m & ((1u << 11) | (1u << 12))) {
      const double I = sqrt(i2);
      if (m & (1u << 11)) g.iavg[j] += (double)g.cnt_iavg * (I / (double)S.Nt);
      if (m & (1u << 12)) g.imax[j] = fmax(g.imax[j], I);
    }
  }
}

__global__ void k_advance_t0(long long *t0, long long k) {
  KWB_STEP_KERNEL_PROLOGUE();
  if (threadIdx.x == 0 && blockIdx.x == 0) *t0 += k;
}

// ------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------

size_t line_pass_smem(int N, int L) { return ((size_t)2 * L * line_pitch(N) + N) * sizeof(float2); }
size_t spec_pass_smem(int N, int L, int dispersion) {
  return ((size_t)2 * (dispersion ? 2 * L : L) * line_pitch(N) + N) * sizeof(float2);
}

static int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// Threads per CTA of a Stockham line pass: KWB_THREADS, or up to KWB_PASS_THREADS_MAX when the
// pass launches fewer than four CTAs per SM, so that a small grid's few tiles are not each worked
// through by 256 threads in long serial loops (the EOS and spectrum passes, shorter per tile,
// keep 256).
int pass_threads(const SimDev &h, long long tiles, long long elems_per_tile, int axis) {
  if (axis >= 0 && axis < 3 && h.thr_line[axis] > 0) return h.thr_line[axis];
  if (!h.grid_fill || tiles >= 4LL * (h.num_sms > 0 ? h.num_sms : 148)) return KWB_THREADS;
  const long long t = (elems_per_tile / 4 + 31) / 32 * 32;
  return (int)std::min<long long>(KWB_PASS_THREADS_MAX, std::max<long long>(KWB_THREADS, t));
}

// The dynamic shared-memory limit of a kernel is a per-function attribute.  It is raised once to
// the device's opt-in maximum, so simulations of different sizes in one process never lower
// it under one another.
cudaError_t raise_dynamic_smem(const void *fn, size_t bytes) {
  // the limit a kernel was given, per device: later calls that fit it make no API call
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> given;
  int cur = 0;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(cur, fn);
  auto it = given.find(key);
  if (it != given.end() && bytes <= it->second) return cudaSuccess;
  cudaFuncAttributes fa;
  e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  if (bytes + fa.sharedSizeBytes <= 48 * 1024) {
    given[key] = 48 * 1024 - fa.sharedSizeBytes;
    return cudaSuccess;
  }
  int optin = 0;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, cur);
  if (e != cudaSuccess) return e;
  const size_t room = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
  if (bytes > room) return cudaErrorInvalidValue;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)room);
  if (e == cudaSuccess) given[key] = room;
  return e;
}
static cudaError_t set_smem(const void *fn, size_t bytes) { return raise_dynamic_smem(fn, bytes); }

cudaError_t launch_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode,
                             long long step_s, cudaStream_t st) {
  if ((h.fast & 1) && fast_size(h.N[axis]) && (axis == 0 || h.N[0] % 4 == 0)) return fast_line_pass(d_sim, h, axis, mode, step_s, st);
  const int L = h.L_line[axis];
  const size_t sm = line_pass_smem(fft_len(h.plan[axis]), L);
  int tiles;
  if (axis == 0) {
    tiles = cdiv(h.N[1], 2 * L) * h.N[2];
    kwb_launch(k_line_pass<true>, tiles, pass_threads(h, tiles, (long long)L * h.N[0], 0), sm, st, d_sim, axis, mode, step_s);
  } else {
    tiles = cdiv(h.N[0], 2 * L) * (axis == 1 ? h.N[2] : h.N[1]);
    kwb_launch(k_line_pass<false>, tiles, pass_threads(h, tiles, (long long)L * h.N[axis], axis), sm, st, d_sim, axis, mode,
               step_s);
  }
  return cudaGetLastError();
}

cudaError_t launch_eos_x_fwd(const SimDev *d_sim, const SimDev &h, long long step_s,
                             cudaStream_t st) {
  if ((h.fast & 2) && h.ndim >= 2 && !h.dispersion && fast_size(h.N[0])) return fast_eos(d_sim, h, true, step_s, st);
  const int L = h.L_eosx;
  const size_t sm = spec_pass_smem(fft_len(h.plan[0]), L, h.dispersion);
  const int tiles = cdiv(h.N[1], 2 * L) * h.N[2];
  kwb_launch(k_eos_x_fwd, tiles, KWB_THREADS, sm, st, d_sim, step_s);
  return cudaGetLastError();
}

cudaError_t launch_eos_x_inv(const SimDev *d_sim, const SimDev &h, long long step_s,
                             cudaStream_t st) {
  if ((h.fast & 2) && h.ndim >= 2 && !h.dispersion && fast_size(h.N[0])) return fast_eos(d_sim, h, false, step_s, st);
  const int L = h.L_eosx;
  const size_t sm = line_pass_smem(fft_len(h.plan[0]), L);
  const int tiles = cdiv(h.N[1], 2 * L) * h.N[2];
  kwb_launch(k_eos_x_inv, tiles, KWB_THREADS, sm, st, d_sim, step_s, h.ndim == 1 ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_spec_pass(const SimDev *d_sim, const SimDev &h, int axis, int op,
                             long long step_s, cudaStream_t st) {
  if ((h.fast & 2) && !h.dispersion && fast_size(h.N[axis])) return fast_spec(d_sim, h, axis, op, step_s, st);
  const int L = h.L_spec[axis];
  const size_t sm = spec_pass_smem(fft_len(h.plan[axis]), L, h.dispersion && op != KWB_SPEC_INV);
  const int tiles = cdiv(h.n1, L) * (axis == 1 ? h.N[2] : h.N[1]);
  kwb_launch(k_spec_pass, tiles, KWB_THREADS, sm, st, d_sim, axis, op, step_s);
  return cudaGetLastError();
}

cudaError_t launch_tr_inject(const SimDev *d_sim, const SimDev &h, long long step_s,
                             cudaStream_t st) {
  if (h.n_tr <= 0) return cudaSuccess;
  kwb_launch(k_tr_inject, cdiv(h.n_tr, 256), 256, 0, st, d_sim, step_s);
  return cudaGetLastError();
}

cudaError_t launch_sensor_gather(const SimDev *d_sim, const SimDev &h, const GroupDev *d_group,
                                 long long n, long long step_s, cudaStream_t st) {
  (void)h;
  if (n <= 0) return cudaSuccess;
  kwb_launch(k_sensor_gather, cdiv(n, 256), 256, 0, st, d_sim, d_group, step_s);
  return cudaGetLastError();
}

cudaError_t prime_attributes(const SimDev &h) {
  cudaError_t e;
  size_t m = 0;
  if ((e = set_smem((const void *)k_line_pass<true>, line_pass_smem(fft_len(h.plan[0]), h.L_line[0]))) != cudaSuccess) return e;
  for (int a = 1; a < h.ndim; ++a) m = std::max(m, line_pass_smem(fft_len(h.plan[a]), h.L_line[a]));
  if ((e = set_smem((const void *)k_line_pass<false>, m)) != cudaSuccess) return e;
  if ((e = set_smem((const void *)k_eos_x_fwd, spec_pass_smem(fft_len(h.plan[0]), h.L_eosx, h.dispersion))) != cudaSuccess) return e;
  if ((e = set_smem((const void *)k_eos_x_inv, line_pass_smem(fft_len(h.plan[0]), h.L_eosx))) != cudaSuccess) return e;
  m = 0;
  for (int a = 1; a < h.ndim; ++a) m = std::max(m, spec_pass_smem(fft_len(h.plan[a]), h.L_spec[a], h.dispersion));
  if ((e = set_smem((const void *)k_spec_pass, m)) != cudaSuccess) return e;
  if (h.fast)
    for (int a = 0; a < h.ndim; ++a)
      if (fast_size(h.N[a]) && (e = fast_prime(h.N[a])) != cudaSuccess) return e;
  if (h.plane && (e = fast_plane_prime()) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t launch_advance_t0(long long *t0, long long k, cudaStream_t st) {
  kwb_launch(k_advance_t0, 1, 32, 0, st, t0, k);
  return cudaGetLastError();
}

}  // namespace kwb
