// Elastic solver kernels: pstd_elastic_2d / pstd_elastic_3d (KWave.jl/src/solver/elastic.jl:
// 133-366, 386-588) on the line-pass machinery of the fluid solver.
//
// One time step (D = 2 or 3, stresses sigma in slots xx, yy, zz, xy, xz, yz):
//
//   k_el_grad(x), k_el_grad(y)[, k_el_grad(z)]   w_j (+)= d/dx_d sigma_dj, staggered +
//                                                 (elastic.jl:223-231, 448-461); one pass per
//                                                 axis transforms the D stresses on its lines
//   k_el_velocity                                 v_j = pml_sg,j (pml_sg,j v_j + dt/rho_sg,j w_j)
//                                                 (:233-243, 463-476)
//   [k_el_inject(velocity)]                       velocity sources (:245-268, 478-492)
//   k_el_grad(x), k_el_grad(y)[, k_el_grad(z)]   w_dd = dv_d/dx_d, w_{ij} (+)= dv_i/dx_j (i != j),
//                                                 staggered - (:270-279, 494-505)
//   k_el_stress                                   the constitutive update with split PML, then
//                                                 p = -trace(sigma)/D (:281-313, 507-521)
//   [k_el_inject(stress)]                         stress sources, p refreshed at their points
//                                                 (:315-347, 523-545)
//   sensor gathers (kwb_kernels.cu)               record_sensor_data! on p and v (:349-356)
//
// Each directional derivative is the 1-D transform along its axis (the reference's full N-D
// rfft / irfft with a multiplier that varies along one axis only), computed two real lines per
// complex line: power-of-two lines on the register FFTs of kwb_fast.cu (k_el_grad_fast), other
// lengths on the shared-memory Stockham FFTs of kwb_fft.cuh (k_el_grad below).
#include <algorithm>

#include "kwb_fft.cuh"
#include "kwb_tiles.cuh"

namespace kwb {

namespace {

int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// Column-major coordinates of voxel i.
struct Coord {
  int x, y, z;
};
__device__ __forceinline__ Coord coord_of(const SimDev &S, long long i) {
  const int Nx = S.N[0], Ny = S.N[1];
  Coord c;
  const long long row = i / Nx;
  c.x = (int)(i - row * Nx);
  c.z = (int)(row / Ny);
  c.y = (int)(row - (long long)c.z * Ny);
  return c;
}

}  // namespace

// Directional derivatives of g.nf fields along `axis` on one tile of 2L real lines.
template <bool CONTIG>
__global__ void __launch_bounds__(KWB_PASS_THREADS_MAX)
    k_el_grad(const __grid_constant__ SimDev S, int axis, const __grid_constant__ ElGrad g, long long step_s) {
  extern __shared__ float4 smem_raw[];
  const int N = S.N[axis];
  const int L = S.L_line[axis];
  const int LS = line_pitch(fft_len(S.plan[axis]));
  const int Nx = S.N[0];
  float2 *X = reinterpret_cast<float2 *>(smem_raw);
  float2 *Y = X + L * LS;
  float2 *tw = Y + L * LS;
  load_twiddles(tw, S.tw[axis], fft_len(S.plan[axis]));  // set-up-time table: before waiting on the previous kernel
  KWB_STEP_KERNEL_PROLOGUE();
  if (step_index(S, step_s) >= S.Nt) return;
  const Tile T = CONTIG ? tile_x(S, 2 * L, blockIdx.x) : tile_yz(S, axis, 2 * L, blockIdx.x);
  auto addr = [&](int c, int i) -> long long {
    return CONTIG ? T.base + (long long)c * Nx + i : T.base + (long long)i * T.stride + c;
  };
  // element e of the tile: line l, position i (strided tiles keep neighbouring columns adjacent
  // in a warp, so their global accesses coalesce)
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
  const float2 *__restrict__ mult = g.neg ? S.gneg[axis] : S.gpos[axis];
  for (int f = 0; f < g.nf; ++f) {
    const float *__restrict__ src = g.src[f];
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int l, i;
      decode(e, l, i);
      const int ca = 2 * l, cb = 2 * l + 1;
      const float a = ca < T.cnt ? src[addr(ca, i)] : 0.f;
      const float b = cb < T.cnt ? src[addr(cb, i)] : 0.f;
      X[l * LS + i] = make_float2(a, b);
    }
    __syncthreads();
    float2 *R = fft_lines<false>(X, Y, L, LS, S.plan[axis], tw);
    float2 *F = (R == X) ? Y : X;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = e / N, i = e - l * N;
      R[l * LS + i] = cmul(R[l * LS + i], mult[i]);  // i k e^{+-i k d/2} / N
    }
    __syncthreads();
    const float2 *Dv = fft_lines<true>(R, F, L, LS, S.plan[axis], tw);
    float *dst = g.dst[f];
    const bool acc = (g.acc >> f) & 1;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int l, i;
      decode(e, l, i);
      const float2 d = Dv[l * LS + i];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = 2 * l + h;
        if (c >= T.cnt) continue;
        const long long ad = addr(c, i);
        const float dv = h ? d.y : d.x;
        dst[ad] = acc ? dst[ad] + dv : dv;
      }
    }
    __syncthreads();  // X and Y are refilled by the next field
  }
}

// v_j = pml_sg,j (pml_sg,j v_j + dt / rho_sg,j w_j), pml = 1 - deficit; rho_sg,j the periodic
// average of rho0 with its +1 neighbour along j (_stagger_density_{2,3}d, first_order_steps.jl:
// 40-52).
__global__ void __launch_bounds__(KWB_THREADS) k_el_velocity(const __grid_constant__ SimDev S, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  if (step_index(S, step_s) >= S.Nt) return;
  const long long nv = S.nvox;
  const long long plane = (long long)S.N[0] * S.N[1];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const Coord c = coord_of(S, i);
    const int cc[3] = {c.x, c.y, c.z};
    for (int j = 0; j < S.D; ++j) {
      float coef = S.dt_over_rho0_s;
      if (S.rho0) {
        const long long step = j == 0 ? 1 : (j == 1 ? S.N[0] : plane);
        const long long nb = cc[j] + 1 == S.N[j] ? i - (long long)cc[j] * step : i + step;
        coef = (2.0f * S.dt) / (S.rho0[i] + S.rho0[nb]);
      }
      const float e = S.pml_sg_def[j][cc[j]];
      const float v = S.u[j][i];
      float t1 = fmaf(-e, v, v);
      t1 = fmaf(coef, S.el_w[j][i], t1);
      S.u[j][i] = fmaf(-e, t1, t1);
    }
  }
}

// Constitutive update with split PML (elastic.jl:281-313 for 2D, 507-521 for 3D), then
// p = -trace(sigma) / D for the sensors.
__global__ void __launch_bounds__(KWB_THREADS) k_el_stress(const __grid_constant__ SimDev S, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  if (step_index(S, step_s) >= S.Nt) return;
  const long long nv = S.nvox;
  const float dt = S.dt;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const Coord c = coord_of(S, i);
    const float lam = S.el_lam ? S.el_lam[i] : S.el_lam_s;
    const float mu = S.el_mu ? S.el_mu[i] : S.el_mu_s;
    const float l2m = lam + 2.0f * mu;
    const float ex = S.pml_def[0][c.x], ey = S.pml_def[1][c.y];
    // pml * (pml * s + dt a), pml = 1 - e
    auto split = [&](float s, float e, float a) {
      float t1 = fmaf(-e, s, s);
      t1 = fmaf(dt, a, t1);
      return fmaf(-e, t1, t1);
    };
    // pml_i pml_j (s + dt a): 1 - pml_i pml_j = e_i + e_j - e_i e_j
    auto shear = [&](float s, float ei, float ej, float a) {
      const float eij = fmaf(-ei, ej, ei + ej);
      const float t1 = fmaf(dt, a, s);
      return fmaf(-eij, t1, t1);
    };
    if (S.D == 2) {
      const float dxx = S.el_w[0][i], dyy = S.el_w[1][i];
      float axx = fmaf(lam, dyy, l2m * dxx);
      float ayy = fmaf(l2m, dyy, lam * dxx);
      float sh = mu * S.el_w[3][i];
      axx = fmaf(S.el_chi_p, axx, axx);
      ayy = fmaf(S.el_chi_p, ayy, ayy);
      sh = fmaf(S.el_chi_s, sh, sh);
      const float sxx = split(S.el_s[0][i], ex, axx);
      const float syy = split(S.el_s[1][i], ey, ayy);
      S.el_s[0][i] = sxx;
      S.el_s[1][i] = syy;
      S.el_s[3][i] = shear(S.el_s[3][i], ex, ey, sh);
      S.p[i] = -(sxx + syy) / 2.0f;
    } else {
      const float ez = S.pml_def[2][c.z];
      const float dxx = S.el_w[0][i], dyy = S.el_w[1][i], dzz = S.el_w[2][i];
      const float sxx = split(S.el_s[0][i], ex, fmaf(lam, dyy + dzz, l2m * dxx));
      const float syy = split(S.el_s[1][i], ey, fmaf(lam, dxx + dzz, l2m * dyy));
      const float szz = split(S.el_s[2][i], ez, fmaf(lam, dxx + dyy, l2m * dzz));
      S.el_s[0][i] = sxx;
      S.el_s[1][i] = syy;
      S.el_s[2][i] = szz;
      S.el_s[3][i] = shear(S.el_s[3][i], ex, ey, mu * S.el_w[3][i]);
      S.el_s[4][i] = shear(S.el_s[4][i], ex, ez, mu * S.el_w[4][i]);
      S.el_s[5][i] = shear(S.el_s[5][i], ey, ez, mu * S.el_w[5][i]);
      S.p[i] = -(sxx + syy + szz) / 3.0f;
    }
  }
}

// The same two updates on four consecutive x voxels per thread (float4 accesses; Nx a multiple
// of 4 and fewer than 2^31 voxels): item q is x = 4 (q mod Nx/4) of row q div (Nx/4).
__device__ __forceinline__ float4 ld4(const float *p, int i) { return *reinterpret_cast<const float4 *>(p + i); }
__device__ __forceinline__ void st4(float *p, int i, float4 v) { *reinterpret_cast<float4 *>(p + i) = v; }
__device__ __forceinline__ float comp(const float4 &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

__global__ void __launch_bounds__(KWB_THREADS) k_el_velocity4(const __grid_constant__ SimDev S, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  if (step_index(S, step_s) >= S.Nt) return;
  const int Nx = S.N[0], Ny = S.N[1], Nz = S.N[2], qx = Nx / 4;
  const int items = qx * Ny * Nz, plane = Nx * Ny;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < items; q += gridDim.x * blockDim.x) {
    const int row = q / qx, x = 4 * (q - row * qx);
    const int z = row / Ny, y = row - z * Ny;
    const int i = row * Nx + x;
    float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (S.rho0) r0 = ld4(S.rho0, i);
    for (int j = 0; j < S.D; ++j) {
      float4 coef = make_float4(S.dt_over_rho0_s, S.dt_over_rho0_s, S.dt_over_rho0_s, S.dt_over_rho0_s);
      if (S.rho0) {
        // rho_sg,j = (rho0 + rho0 shifted by -e_j, periodic) / 2
        float4 r1;
        if (j == 0) {
          const float nx = S.rho0[x + 4 == Nx ? row * Nx : i + 4];
          r1 = make_float4(r0.y, r0.z, r0.w, nx);
        } else if (j == 1) {
          r1 = ld4(S.rho0, y + 1 == Ny ? i - y * Nx : i + Nx);
        } else {
          r1 = ld4(S.rho0, z + 1 == Nz ? i - z * plane : i + plane);
        }
        const float tdt = 2.0f * S.dt;
        coef = make_float4(tdt / (r0.x + r1.x), tdt / (r0.y + r1.y), tdt / (r0.z + r1.z), tdt / (r0.w + r1.w));
      }
      float4 e;
      if (j == 0) e = ld4(S.pml_sg_def[0], x);
      else {
        const float ej = S.pml_sg_def[j][j == 1 ? y : z];
        e = make_float4(ej, ej, ej, ej);
      }
      const float4 v = ld4(S.u[j], i), w = ld4(S.el_w[j], i);
      // pml (pml v + coef w), pml = 1 - e
      auto upd = [](float e1, float c1, float v1, float w1) {
        const float t1 = fmaf(c1, w1, fmaf(-e1, v1, v1));
        return fmaf(-e1, t1, t1);
      };
      st4(S.u[j], i, make_float4(upd(e.x, coef.x, v.x, w.x), upd(e.y, coef.y, v.y, w.y), upd(e.z, coef.z, v.z, w.z),
                                 upd(e.w, coef.w, v.w, w.w)));
    }
  }
}

__global__ void __launch_bounds__(KWB_THREADS) k_el_stress4(const __grid_constant__ SimDev S, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  if (step_index(S, step_s) >= S.Nt) return;
  const int Nx = S.N[0], Ny = S.N[1], Nz = S.N[2], qx = Nx / 4;
  const int items = qx * Ny * Nz;
  const float dt = S.dt;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < items; q += gridDim.x * blockDim.x) {
    const int row = q / qx, x = 4 * (q - row * qx);
    const int z = row / Ny, y = row - z * Ny;
    const int i = row * Nx + x;
    const float4 lam4 = S.el_lam ? ld4(S.el_lam, i) : make_float4(S.el_lam_s, S.el_lam_s, S.el_lam_s, S.el_lam_s);
    const float4 mu4 = S.el_mu ? ld4(S.el_mu, i) : make_float4(S.el_mu_s, S.el_mu_s, S.el_mu_s, S.el_mu_s);
    const float4 ex4 = ld4(S.pml_def[0], x);
    const float ey = S.pml_def[1][y];
    const float ez = S.D == 3 ? S.pml_def[2][z] : 0.f;
    float4 w[6], sg[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (S.D == 2 && (k == 2 || k > 3)) continue;
      w[k] = ld4(S.el_w[k], i);
      sg[k] = ld4(S.el_s[k], i);
    }
    float out[6][4], pv[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float lam = comp(lam4, c), mu = comp(mu4, c), l2m = lam + 2.0f * mu, ex = comp(ex4, c);
      auto split = [&](float s, float e, float a) {
        float t1 = fmaf(-e, s, s);
        t1 = fmaf(dt, a, t1);
        return fmaf(-e, t1, t1);
      };
      auto shear = [&](float s, float ei, float ej, float a) {
        const float eij = fmaf(-ei, ej, ei + ej);
        const float t1 = fmaf(dt, a, s);
        return fmaf(-eij, t1, t1);
      };
      if (S.D == 2) {
        const float dxx = comp(w[0], c), dyy = comp(w[1], c);
        float axx = fmaf(lam, dyy, l2m * dxx);
        float ayy = fmaf(l2m, dyy, lam * dxx);
        float sh = mu * comp(w[3], c);
        axx = fmaf(S.el_chi_p, axx, axx);
        ayy = fmaf(S.el_chi_p, ayy, ayy);
        sh = fmaf(S.el_chi_s, sh, sh);
        out[0][c] = split(comp(sg[0], c), ex, axx);
        out[1][c] = split(comp(sg[1], c), ey, ayy);
        out[3][c] = shear(comp(sg[3], c), ex, ey, sh);
        pv[c] = -(out[0][c] + out[1][c]) / 2.0f;
      } else {
        const float dxx = comp(w[0], c), dyy = comp(w[1], c), dzz = comp(w[2], c);
        out[0][c] = split(comp(sg[0], c), ex, fmaf(lam, dyy + dzz, l2m * dxx));
        out[1][c] = split(comp(sg[1], c), ey, fmaf(lam, dxx + dzz, l2m * dyy));
        out[2][c] = split(comp(sg[2], c), ez, fmaf(lam, dxx + dyy, l2m * dzz));
        out[3][c] = shear(comp(sg[3], c), ex, ey, mu * comp(w[3], c));
        out[4][c] = shear(comp(sg[4], c), ex, ez, mu * comp(w[4], c));
        out[5][c] = shear(comp(sg[5], c), ey, ez, mu * comp(w[5], c));
        pv[c] = -(out[0][c] + out[1][c] + out[2][c]) / 3.0f;
      }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (S.D == 2 && (k == 2 || k > 3)) continue;
      st4(S.el_s[k], i, make_float4(out[k][0], out[k][1], out[k][2], out[k][3]));
    }
    st4(S.p, i, make_float4(pv[0], pv[1], pv[2], pv[3]));
  }
}

// Point sources: Dirichlet (mode 0) or additive; column min(t, n_cols) of each present component.
// which 0: velocities at u_idx; which 1: stresses at s_idx, then p at those points.
__global__ void k_el_inject(const __grid_constant__ SimDev S, int which, long long step_s) {
  KWB_STEP_KERNEL_PROLOGUE();
  const long long t = step_index(S, step_s);
  if (t >= S.Nt) return;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (which == 0) {
    if (j >= S.n_u) return;
    const long long v = S.u_idx[j];
    for (int d = 0; d < S.D; ++d) {
      if (!S.u_sig[d]) continue;
      const long long col = min(t + 1, (long long)S.u_cols[d]) - 1;
      const float val = S.u_sig[d][col * S.n_u + j];
      S.u[d][v] = S.u_mode == 0 ? val : S.u[d][v] + val;
    }
    return;
  }
  if (j >= S.n_s) return;
  const long long v = S.s_idx[j];
  for (int k = 0; k < 6; ++k) {
    if (!S.s_sig[k] || !S.el_s[k]) continue;
    const long long col = min(t + 1, (long long)S.s_cols[k]) - 1;
    const float val = S.s_sig[k][col * S.n_s + j];
    S.el_s[k][v] = S.s_mode == 0 ? val : S.el_s[k][v] + val;
  }
  if (S.D == 2) S.p[v] = -(S.el_s[0][v] + S.el_s[1][v]) / 2.0f;
  else S.p[v] = -(S.el_s[0][v] + S.el_s[1][v] + S.el_s[2][v]) / 3.0f;
}

// p0: every normal stress starts at -p0 (p holds p0 in FP32).
__global__ void k_el_init(const __grid_constant__ SimDev S) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < S.nvox; i += (long long)gridDim.x * blockDim.x) {
    const float v = -S.p[i];
    for (int d = 0; d < S.D; ++d) S.el_s[d][i] = v;
  }
}

// ------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------

static int elementwise_grid(const SimDev &h) {
  const long long want = cdiv(h.nvox, KWB_THREADS);
  const long long cap = (long long)(h.num_sms > 0 ? h.num_sms : 148) * 8;
  return (int)std::max(1LL, std::min(want, cap));
}

static cudaError_t set_smem_optin(const void *fn, size_t bytes) { return raise_dynamic_smem(fn, bytes); }

// Register-FFT passes serve power-of-two lines (strided ones need Nx a multiple of 4 for their
// 16-byte staging); every other length runs on the Stockham kernel above.
static bool el_fast(const SimDev &h, int axis) {
  return (h.fast & 1) && fast_size(h.N[axis]) && (axis == 0 || h.N[0] % 4 == 0);
}

cudaError_t el_prime(const SimDev &h) {
  cudaError_t e = set_smem_optin((const void *)k_el_grad<true>, line_pass_smem(fft_len(h.plan[0]), h.L_line[0]));
  size_t m = 0;
  for (int a = 1; a < h.ndim; ++a) m = std::max(m, line_pass_smem(fft_len(h.plan[a]), h.L_line[a]));
  if (e == cudaSuccess) e = set_smem_optin((const void *)k_el_grad<false>, m);
  for (int a = 0; a < h.ndim && e == cudaSuccess; ++a)
    if (el_fast(h, a)) e = fast_prime(h.N[a]);
  return e;
}

cudaError_t el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st) {
  if (el_fast(h, axis)) return fast_el_grad(h, axis, g, s, st);
  const int L = h.L_line[axis];
  const size_t sm = line_pass_smem(fft_len(h.plan[axis]), L);
  const long long tiles = axis == 0 ? (long long)cdiv(h.N[1], 2 * L) * h.N[2]
                                    : (long long)cdiv(h.N[0], 2 * L) * (axis == 1 ? h.N[2] : h.N[1]);
  const int threads = pass_threads(h, tiles, (long long)L * h.N[axis]);
  if (axis == 0)
    kwb_launch(k_el_grad<true>, (int)tiles, threads, sm, st, h, axis, g, s);
  else
    kwb_launch(k_el_grad<false>, (int)tiles, threads, sm, st, h, axis, g, s);
  return cudaGetLastError();
}

static bool vec4(const SimDev &h) { return h.N[0] % 4 == 0 && h.nvox < (1LL << 31); }

cudaError_t el_velocity(const SimDev &h, long long s, cudaStream_t st) {
  if (vec4(h)) kwb_launch(k_el_velocity4, elementwise_grid(h), KWB_THREADS, 0, st, h, s);
  else kwb_launch(k_el_velocity, elementwise_grid(h), KWB_THREADS, 0, st, h, s);
  return cudaGetLastError();
}

cudaError_t el_stress(const SimDev &h, long long s, cudaStream_t st) {
  if (vec4(h)) kwb_launch(k_el_stress4, elementwise_grid(h), KWB_THREADS, 0, st, h, s);
  else kwb_launch(k_el_stress, elementwise_grid(h), KWB_THREADS, 0, st, h, s);
  return cudaGetLastError();
}

cudaError_t el_inject(const SimDev &h, int which, long long s, cudaStream_t st) {
  const long long n = which == 0 ? h.n_u : h.n_s;
  if (n <= 0) return cudaSuccess;
  kwb_launch(k_el_inject, cdiv(n, 256), 256, 0, st, h, which, s);
  return cudaGetLastError();
}

cudaError_t el_init(const SimDev &h, cudaStream_t st) {
  k_el_init<<<elementwise_grid(h), KWB_THREADS, 0, st>>>(h);
  return cudaGetLastError();
}

}  // namespace kwb
