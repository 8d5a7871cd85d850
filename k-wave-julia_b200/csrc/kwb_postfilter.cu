// Post-loop sensor filters on the device: the reference's apply_sensor_directivity! and
// apply_frequency_response! (KWave.jl/src/solver/first_order_steps.jl:836-910).
//
// Both filters replace a recorded pressure series p_j[t] (t < Nt) by real(ifft(fft(p_j) .* H)),
// with a real response H that depends only on |f_k| (f = fftfreq(Nt, 1/dt)):
//   directivity         D_j(f) = sinc(2 pi |f| / d_min * size * sin(theta_j) / 2)  (1 at 0)
//   frequency response  R(f)   = exp(-(|f| - f_c)^2 / (2 bw^2))
// |f_k| = |f_{Nt-k}|, so H is even and the filter equals a circular convolution with the real,
// even kernel h = ifft(H):  p'_j[n] = sum_m h[(n - m) mod Nt] p_j[m].  Here
//   1. k_filter_response builds H per distinct filter in FP64 (the reference's per-bin formula);
//   2. k_filter_kernel takes its inverse DFT in FP64 (a cosine sum, O(Nt^2) per filter) and
//      rounds h to FP32 once;
//   3. k_circulant applies the convolution to the device series [t][j] (sensor points
//      contiguous) as a tiled product: FP32 products summed per 32-term chunk, chunks summed in
//      FP64, so the result keeps FP32 accuracy for any Nt.
// The series never leaves the device before it is filtered.
#include <cmath>

#include "kwb_internal.h"

namespace kwb {
namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

// H[f][k] for k < Nt.  sin_th[f]: sin(theta) of filter f's directivity, or NaN for none.
__global__ void k_filter_response(double *H, int Nt, int nf, const double *sin_th, double dir_size,
                                  double d_min, double fs, int freq, double fc, double bw) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nf * Nt) return;
  const int f = (int)(i / Nt), k = (int)(i - (long long)f * Nt);
  // fftfreq(Nt, 1/fs): k/Nt fs for k < ceil(Nt/2), (k - Nt)/Nt fs after
  const int kk = (k < (Nt + 1) / 2) ? k : k - Nt;
  const double af = fabs((double)kk * fs / (double)Nt);
  double h = 1.0;
  const double st = sin_th[f];
  if (!isnan(st)) {
    const double arg = kTwoPi * af / d_min * dir_size * st / 2.0;
    h = (arg == 0.0) ? 1.0 : sin(arg) / arg;
  }
  if (freq) h *= exp(-((af - fc) * (af - fc)) / (2.0 * bw * bw));
  H[i] = h;
}

// h[f][n] = (1/Nt) sum_k H[f][k] cos(2 pi k n / Nt), from the FP64 table cosT[m] = cos(2 pi m/Nt).
__global__ void k_filter_kernel(float *h, const double *H, const double *cosT, int Nt, int nf) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nf * Nt) return;
  const int f = (int)(i / Nt), n = (int)(i - (long long)f * Nt);
  const double *Hf = H + (long long)f * Nt;
  double s = 0.0;
  int m = 0;  // k n mod Nt
  for (int k = 0; k < Nt; ++k) {
    s = fma(Hf[k], __ldg(cosT + m), s);
    m += n;
    if (m >= Nt) m -= Nt;
  }
  h[i] = (float)(s / (double)Nt);
}

__global__ void k_cos_table(double *cosT, int Nt) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < Nt) cosT[m] = cospi(2.0 * (double)m / (double)Nt);
}

// out[n][j] = sum_m h_{fid[j]}[(n - m) mod Nt] in[m][j], a TN x TJ output tile per CTA.
constexpr int TN = 64, TJ = 32, TM = 32, CT = 256;
__global__ void __launch_bounds__(CT) k_circulant(float *__restrict__ out, const float *__restrict__ in,
                                                  const float *__restrict__ h, const int *__restrict__ fid,
                                                  int Nt, long long n_pts) {
  __shared__ float ps[TM][TJ];
  __shared__ float hs[TJ][TN + TM + 1];  // odd pitch: a warp's 32 points hit 32 banks
  const int tx = threadIdx.x % TJ, ty = threadIdx.x / TJ;  // ty < 8: outputs n0 + ty + 8 i
  const long long j0 = (long long)blockIdx.x * TJ;
  const int n0 = blockIdx.y * TN;
  const long long j = j0 + tx;
  double acc[TN / 8];
#pragma unroll
  for (int i = 0; i < TN / 8; ++i) acc[i] = 0.0;
  for (int m0 = 0; m0 < Nt; m0 += TM) {
    __syncthreads();
    // input chunk rows m0 .. m0 + TM - 1 (zero past Nt or past the last point)
    for (int e = threadIdx.x; e < TM * TJ; e += CT) {
      const int mm = e / TJ, jj = e % TJ;
      const int m = m0 + mm;
      const long long jg = j0 + jj;
      ps[mm][jj] = (m < Nt && jg < n_pts) ? in[(long long)m * n_pts + jg] : 0.f;
    }
    // kernel values h[(n - m) mod Nt] for d = (n - m) - (n0 - m0 - TM + 1) in [0, TN + TM - 1)
    for (int e = threadIdx.x; e < TJ * (TN + TM); e += CT) {
      const int jj = e / (TN + TM), d = e % (TN + TM);
      const long long jg = j0 + jj;
      float v = 0.f;
      if (jg < n_pts && d < TN + TM - 1) {
        int q = (n0 - m0 - TM + 1 + d) % Nt;
        if (q < 0) q += Nt;
        v = h[(long long)fid[jg] * Nt + q];
      }
      hs[jj][d] = v;
    }
    __syncthreads();
    float part[TN / 8];
#pragma unroll
    for (int i = 0; i < TN / 8; ++i) part[i] = 0.f;
#pragma unroll 8
    for (int mm = 0; mm < TM; ++mm) {
      const float x = ps[mm][tx];
#pragma unroll
      for (int i = 0; i < TN / 8; ++i) part[i] = fmaf(hs[tx][ty + 8 * i - mm + TM - 1], x, part[i]);
    }
#pragma unroll
    for (int i = 0; i < TN / 8; ++i) acc[i] += (double)part[i];
  }
  if (j >= n_pts) return;
#pragma unroll
  for (int i = 0; i < TN / 8; ++i) {
    const int n = n0 + ty + 8 * i;
    if (n < Nt) out[(long long)n * n_pts + j] = (float)acc[i];
  }
}

int cdiv_ll(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace

cudaError_t filter_build_kernels(float *h, double *H, double *cosT, int Nt, int nf, const double *sin_th,
                                 double dir_size, double d_min, double dt, int freq, double fc, double bw,
                                 cudaStream_t st) {
  const long long tot = (long long)nf * Nt;
  k_cos_table<<<cdiv_ll(Nt, 256), 256, 0, st>>>(cosT, Nt);
  k_filter_response<<<cdiv_ll(tot, 256), 256, 0, st>>>(H, Nt, nf, sin_th, dir_size, d_min, 1.0 / dt, freq, fc, bw);
  k_filter_kernel<<<cdiv_ll(tot, 128), 128, 0, st>>>(h, H, cosT, Nt, nf);
  return cudaGetLastError();
}

cudaError_t filter_apply(float *out, const float *in, const float *h, const int *fid, int Nt, long long n_pts,
                         cudaStream_t st) {
  if (n_pts <= 0 || Nt <= 0) return cudaSuccess;
  const dim3 grid(cdiv_ll(n_pts, TJ), cdiv_ll(Nt, TN));
  if (grid.y > 65535) return cudaErrorInvalidValue;
  k_circulant<<<grid, CT, 0, st>>>(out, in, h, fid, Nt, n_pts);
  return cudaGetLastError();
}

}  // namespace kwb
