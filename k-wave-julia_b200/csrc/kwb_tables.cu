// FP64 operator-table builders.  Every table is computed in double precision on the device and
// rounded once to FP32:
//   * twiddles exp(-2 pi i m/N)                             (the FFT engine, kwb_fft.cuh)
//   * gradient multipliers i k e^{+-i k d/2} / N           (fft_utils.jl:247-303, grid.jl:120-153)
//   * PML deficits 1 - exp(-alpha pos^4 dt)                (pml.jl:25-56)
//   * EOS multiplier [c^2] kappa (1 + tau |k|^y) / Ntot and
//     the dispersion multiplier c^2 kappa eta |k|^(y-1) / Ntot   (solver/first_order.jl:13-42,
//                                                             solver/first_order_steps.jl:243-286)
//   * medium conversions (c0^2, Q = BonA/(2 rho0)) and source signal tables p/(D c^2).
#include "kwb_internal.h"

namespace kwb {

// FFT-order wavenumber index: 0..ceil(N/2)-1, then -(N - m) (grid.jl:120-130)
__device__ __forceinline__ double wavenumber(int m, int N, double d) {
  const double dk = 2.0 * 3.141592653589793238462643 / ((double)N * d);
  const int mm = (m < (N + 1) / 2) ? m : m - N;
  return (double)mm * dk;
}

__global__ void k_build_twiddles(float2 *out, int N) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= N) return;
  double s, c;
  sincospi(2.0 * (double)m / (double)N, &s, &c);
  out[m] = make_float2((float)c, (float)(-s));
}

__global__ void k_build_gradient(float2 *pos, float2 *neg, int N, double d) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= N) return;
  const double k = wavenumber(m, N, d);
  double s, c;
  sincos(k * d / 2.0, &s, &c);
  const double inv = 1.0 / (double)N;
  // i k (c + i s) = (-k s, k c);  i k (c - i s) = (k s, k c)
  pos[m] = make_float2((float)(-k * s * inv), (float)(k * c * inv));
  neg[m] = make_float2((float)(k * s * inv), (float)(k * c * inv));
}

__global__ void k_build_pml_deficit(float *out, int N, int pml_size, double alpha, double dt,
                                    int staggered) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i < N; ++i) out[i] = 0.0f;
  for (int i = 1; i <= pml_size; ++i) {
    const double pos = staggered ? ((double)(pml_size - i) + 0.5) / (double)pml_size
                                 : (double)(pml_size - i + 1) / (double)pml_size;
    const double p2 = pos * pos;
    const double a = alpha * (p2 * p2);
    const float def = (float)(-expm1(-a * dt));
    if (i - 1 < N) out[i - 1] = def;
    if (N - i >= 0) out[N - i] = def;
  }
}

// Layouts: [k_z][k_y][k_x] (slot_ky == nullptr) or, for the cluster plane pass,
// [k_x][k_z][slot] with k_y = slot_ky[slot], or, for its slot-major variant (slot_kz given),
// [k_x][slot][j] with k_z = slot_kz[j].
__global__ void k_build_eos_multiplier(float *M, float *M2, int Nx, int Ny, int Nz, double dx,
                                       double dy, double dz, double c_ref, double dt,
                                       double c_sq_fold, int absorbing, double tau, double eta,
                                       double y, const int *slot_ky, const int *slot_kz) {
  const int n1 = Nx / 2 + 1;
  const long long total = (long long)n1 * Ny * Nz;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  int kx, ky, kz;
  if (slot_kz) {
    kz = slot_kz[(int)(idx % Nz)];
    ky = slot_ky[(int)((idx / Nz) % Ny)];
    kx = (int)(idx / ((long long)Ny * Nz));
  } else if (slot_ky) {
    ky = slot_ky[(int)(idx % Ny)];
    kz = (int)((idx / Ny) % Nz);
    kx = (int)(idx / ((long long)Ny * Nz));
  } else {
    kx = (int)(idx % n1);
    ky = (int)((idx / n1) % Ny);
    kz = (int)(idx / ((long long)n1 * Ny));
  }
  const double a = wavenumber(kx, Nx, dx);
  const double b = Ny > 1 ? wavenumber(ky, Ny, dy) : 0.0;
  const double c = Nz > 1 ? wavenumber(kz, Nz, dz) : 0.0;
  const double kmag = sqrt((a * a + b * b) + c * c);
  const double arg = c_ref * kmag * dt / 2.0;
  const double kappa = (arg == 0.0) ? 1.0 : sin(arg) / arg;
  const double inv_total = 1.0 / ((double)Nx * (double)Ny * (double)Nz);
  double m = c_sq_fold * kappa;
  if (absorbing) m = m * (1.0 + tau * pow(kmag, y));
  M[idx] = (float)(m * inv_total);
  if (M2) M2[idx] = (float)(c_sq_fold * kappa * (eta * pow(kmag, y - 1.0)) * inv_total);
}

// Row-major (x slowest, f fastest: in[(x*Nm + m)*Nf + f]) to column-major
// (out[x + Nx*(m + Nm*f)]) through a 32 x 32 shared tile, so that both sides are coalesced.
// 3-D grids pass (Nx, Ny, Nz); 2-D grids (Nx, 1, Ny).
__global__ void k_transpose_to_column_major(double *out, const double *in, int Nx, int Nm, int Nf) {
  __shared__ double tile[32][33];
  const int f0 = blockIdx.x * 32, x0 = blockIdx.y * 32, m = blockIdx.z;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int x = x0 + j, f = f0 + threadIdx.x;
    if (x < Nx && f < Nf) tile[j][threadIdx.x] = in[((long long)x * Nm + m) * Nf + f];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int f = f0 + j, x = x0 + threadIdx.x;
    if (x < Nx && f < Nf) out[x + (long long)Nx * (m + (long long)Nm * f)] = tile[threadIdx.x][j];
  }
}

// op 0: copy, op 1: square
__global__ void k_convert(float *out, const double *in, long long n, int op) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = in[i];
  out[i] = (float)(op == 1 ? v * v : v);
}

__global__ void k_build_nlq(float *out, const double *bona, int bona_array, double bona_s,
                            const double *rho0, int rho0_array, double rho0_s, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double b = bona_array ? bona[i] : bona_s;
  const double r = rho0_array ? rho0[i] : rho0_s;
  out[i] = (float)((b / 2.0) / r);
}

__global__ void k_build_source_table(float *out, const double *sig, long long n_rows,
                                     long long n_pts, long long n_cols, const double *c_at,
                                     double c_s, int c_array, double divisor, int apply_c) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_pts * n_cols) return;
  const long long col = idx / n_pts;
  const long long j = idx - col * n_pts;
  double v = sig[j + n_rows * col];
  if (apply_c) {
    const double c = c_array ? c_at[j] : c_s;
    v = v / (divisor * (c * c));
  }
  out[idx] = (float)v;
}

static int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

cudaError_t build_twiddles(float2 *out, int N, cudaStream_t st) {
  k_build_twiddles<<<blocks(N, 256), 256, 0, st>>>(out, N);
  return cudaGetLastError();
}
cudaError_t build_gradient(float2 *pos, float2 *neg, int N, double d, cudaStream_t st) {
  k_build_gradient<<<blocks(N, 256), 256, 0, st>>>(pos, neg, N, d);
  return cudaGetLastError();
}
cudaError_t build_pml_deficit(float *out, int N, int pml_size, double alpha, double dt,
                              int staggered, cudaStream_t st) {
  k_build_pml_deficit<<<1, 32, 0, st>>>(out, N, pml_size, alpha, dt, staggered);
  return cudaGetLastError();
}
cudaError_t build_eos_multiplier(float *M, float *M2, const int N[3], const double d[3],
                                 double c_ref, double dt, double c_sq_fold, int absorbing,
                                 double tau, double eta, double y, const int *slot_ky,
                                 const int *slot_kz, cudaStream_t st) {
  const long long total = (long long)(N[0] / 2 + 1) * N[1] * N[2];
  k_build_eos_multiplier<<<blocks(total, 256), 256, 0, st>>>(M, M2, N[0], N[1], N[2], d[0],
                                                             d[1], d[2], c_ref, dt, c_sq_fold,
                                                             absorbing, tau, eta, y, slot_ky, slot_kz);
  return cudaGetLastError();
}
cudaError_t transpose_to_column_major(double *out, const double *in, int ndim, const int N[3],
                                      cudaStream_t st) {
  const int Nx = N[0], Nm = ndim == 3 ? N[1] : 1, Nf = ndim == 3 ? N[2] : N[1];
  if (Nm > 65535) return cudaErrorInvalidValue;
  k_transpose_to_column_major<<<dim3((Nf + 31) / 32, (Nx + 31) / 32, Nm), dim3(32, 8), 0, st>>>(out, in, Nx, Nm, Nf);
  return cudaGetLastError();
}
cudaError_t convert_f64_to_f32(float *out, const double *in, long long n, int op,
                               cudaStream_t st) {
  k_convert<<<blocks(n, 256), 256, 0, st>>>(out, in, n, op);
  return cudaGetLastError();
}
cudaError_t build_nlq(float *out, const double *bona, int bona_array, double bona_s,
                      const double *rho0, int rho0_array, double rho0_s, long long n,
                      cudaStream_t st) {
  k_build_nlq<<<blocks(n, 256), 256, 0, st>>>(out, bona, bona_array, bona_s, rho0, rho0_array,
                                              rho0_s, n);
  return cudaGetLastError();
}
cudaError_t build_source_table(float *out, const double *sig, long long n_rows, long long n_pts,
                               long long n_cols, const double *c_at_pts, double c_s,
                               int c_array, double divisor, int apply_c, cudaStream_t st) {
  const long long total = n_pts * n_cols;
  if (total == 0) return cudaSuccess;
  k_build_source_table<<<blocks(total, 256), 256, 0, st>>>(out, sig, n_rows, n_pts, n_cols,
                                                           c_at_pts, c_s, c_array, divisor,
                                                           apply_c);
  return cudaGetLastError();
}

}  // namespace kwb
