// Batched mixed-radix (2, 3, 4, 5, 7, 8) Stockham FFTs in shared memory.
//
// A CTA holds L complex lines of length N, line stride LS, in shared memory and transforms all
// of them at once: every stage is one pass of radix-R butterflies over L*N/R butterflies
// shared by the CTA's threads, ping-ponging between two buffers.  The Stockham ordering keeps
// the output in natural frequency order, so the k-space multiplies index it directly.
//
// Twiddles exp(-2 pi i m / N) come from a table built in FP64 on the device and rounded once
// to FP32 (kwb_tables.cu); the butterfly constants are the exact values of cos/sin(2 pi k/R)
// written out to 22 digits.  Forward = exp(-i...), inverse = exp(+i...) without 1/N (the
// normalisation is folded into the k-space multipliers).
#pragma once
#include "kwb_internal.h"

namespace kwb {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  __device__ __forceinline__ static void run(float2 (&v)[2]) {
    float2 a = cadd(v[0], v[1]);
    float2 b = csub(v[0], v[1]);
    v[0] = a;
    v[1] = b;
  }
};

template <bool INV>
struct Dft<4, INV> {
  __device__ __forceinline__ static void run(float2 (&v)[4]) {
    float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    float2 t2 = cadd(v[1], v[3]), t3 = mul_mi<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <bool INV>
struct Dft<8, INV> {
  __device__ __forceinline__ static void run(float2 (&v)[8]) {
    const float h = 0.7071067811865475244008f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV>::run(e);
    Dft<4, INV>::run(o);
    // W^1 = (1 -+ i)/sqrt2, W^2 = -+i, W^3 = (-1 -+ i)/sqrt2
    float2 w1 = INV ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                    : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    float2 w2 = mul_mi<INV>(o[2]);
    float2 w3 = INV ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                    : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], w1);
    v[5] = csub(e[1], w1);
    v[2] = cadd(e[2], w2);
    v[6] = csub(e[2], w2);
    v[3] = cadd(e[3], w3);
    v[7] = csub(e[3], w3);
  }
};

template <bool INV>
struct Dft<3, INV> {
  __device__ __forceinline__ static void run(float2 (&v)[3]) {
    const float s3 = 0.8660254037844386467637f;
    float2 t = cadd(v[1], v[2]);
    float2 s = mul_mi<INV>(cscale(csub(v[1], v[2]), s3));
    float2 m = make_float2(fmaf(-0.5f, t.x, v[0].x), fmaf(-0.5f, t.y, v[0].y));
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, s);
    v[2] = csub(m, s);
  }
};

template <bool INV>
struct Dft<5, INV> {
  __device__ __forceinline__ static void run(float2 (&v)[5]) {
    const float c1 = 0.3090169943749474241023f, c2 = -0.8090169943749474241023f;
    const float s1 = 0.9510565162951535721164f, s2 = 0.5877852522924731291687f;
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    float2 b1 = mul_mi<INV>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    float2 b2 = mul_mi<INV>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  }
};

template <bool INV>
struct Dft<7, INV> {
  __device__ __forceinline__ static void run(float2 (&v)[7]) {
    const float c[3] = {0.6234898018587335305251f, -0.2225209339563144042889f,
                        -0.9009688679024191262361f};
    const float s[3] = {0.7818314824680298087084f, 0.9749279121818236070181f,
                        0.4338837391175581204758f};
    float2 t[3], d[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      t[j] = cadd(v[j + 1], v[6 - j]);
      d[j] = csub(v[j + 1], v[6 - j]);
    }
    float2 x0 = v[0];
    v[0] = cadd(x0, cadd(t[0], cadd(t[1], t[2])));
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
      float2 a = x0, b = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 1; j <= 3; ++j) {
        int m = (j * k) % 7;  // cos(2 pi m/7), sin(2 pi m/7) with m in 1..6
        float cm = m <= 3 ? c[m - 1] : c[7 - m - 1];
        float sm = m <= 3 ? s[m - 1] : -s[7 - m - 1];
        a.x = fmaf(cm, t[j - 1].x, a.x);
        a.y = fmaf(cm, t[j - 1].y, a.y);
        b.x = fmaf(sm, d[j - 1].x, b.x);
        b.y = fmaf(sm, d[j - 1].y, b.y);
      }
      b = mul_mi<INV>(b);
      v[k] = cadd(a, b);
      v[7 - k] = csub(a, b);
    }
  }
};

// Line pitch (float2 slots per line) of the Stockham buffers: N elements plus one pad slot per 16
// for the intermediate stages (see spad), plus one.
__host__ __device__ inline int line_pitch(int N) { return N + (N >> 4) + 1; }

// Slot of element m in an intermediate stage buffer: one pad slot after every 16 elements, so
// the strided stores of the early stages (stride R * Ns with Ns < 16) fall in distinct banks.
// The first stage reads, and the last stage writes, the natural (unpadded) order the callers
// use.
__device__ __forceinline__ int spad(int m) { return m + (m >> 4); }

__device__ __forceinline__ int fdiv(int n, FastDiv d) {
  return (int)((__umulhi((unsigned)n, d.mul) + (unsigned)n) >> d.shift);
}

// One Stockham stage of radix R over L lines: X -> Y (pin / pout: X / Y in the padded layout).
// dnr, dns: divisions by N / R and by Ns, precomputed in the plan.
template <int R, bool INV>
__device__ __forceinline__ void stockham_stage(const float2 *__restrict__ X, float2 *__restrict__ Y,
                                               int L, int LS, int N, int Ns,
                                               const float2 *__restrict__ tw, bool pin, bool pout,
                                               FastDiv dnr, FastDiv dns) {
  const int NR = N / R;
  const int total = L * NR;
  const int tstride = N / (Ns * R);
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    const int l = fdiv(b, dnr);
    const int j = b - l * NR;
    const int k = j - fdiv(j, dns) * Ns;
    const float2 *x = X + l * LS;
    float2 *y = Y + l * LS;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int m = j + r * NR;
      v[r] = x[pin ? spad(m) : m];
    }
    if (k != 0) {
      const int ts = k * tstride;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[r * ts];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    Dft<R, INV>::run(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int m = base + r * Ns;
      y[pout ? spad(m) : m] = v[r];
    }
  }
}

// The Stockham stages of `plan` on L lines of fft_len(plan) points held in X (Y is scratch).
template <bool INV>
__device__ float2 *stockham_lines(float2 *X, float2 *Y, int L, int LS, const FftPlan &plan,
                                  const float2 *tw) {
  const int N = fft_len(plan);
  int Ns = 1;
  for (int s = 0; s < plan.nstages; ++s) {
    const int R = plan.radix[s];
    const bool pin = s > 0, pout = s + 1 < plan.nstages;
    const FastDiv dnr = plan.div_nr[s], dns = plan.div_ns[s];
    switch (R) {
      case 2: stockham_stage<2, INV>(X, Y, L, LS, N, Ns, tw, pin, pout, dnr, dns); break;
      case 3: stockham_stage<3, INV>(X, Y, L, LS, N, Ns, tw, pin, pout, dnr, dns); break;
      case 4: stockham_stage<4, INV>(X, Y, L, LS, N, Ns, tw, pin, pout, dnr, dns); break;
      case 5: stockham_stage<5, INV>(X, Y, L, LS, N, Ns, tw, pin, pout, dnr, dns); break;
      case 7: stockham_stage<7, INV>(X, Y, L, LS, N, Ns, tw, pin, pout, dnr, dns); break;
      default: stockham_stage<8, INV>(X, Y, L, LS, N, Ns, tw, pin, pout, dnr, dns); break;
    }
    __syncthreads();
    float2 *t = X;
    X = Y;
    Y = t;
    Ns *= R;
  }
  return X;
}

// Bluestein's algorithm for the n-point DFT of L lines (n = plan.n, first n slots of each line
// in X; X and Y hold plan.m slots per line): with w_j = exp(-i pi j^2/n),
//   X_k = w_k sum_j (x_j w_j) conj(w_{k-j}),
// a circular convolution of length m >= 2n - 1 done as FFT_m, a multiply by the transform of
// the conjugate chirp (chirp_ft, scaled by 1/m), and an inverse FFT_m.  The inverse DFT is the
// conjugate of the forward DFT of the conjugate input.  tw: the m-point twiddles.
template <bool INV>
__device__ float2 *bluestein_lines(float2 *X, float2 *Y, int L, int LS, const FftPlan &plan,
                                   const float2 *tw) {
  const int n = plan.n, m = plan.m;
  const float2 *__restrict__ w = plan.chirp;
  const float2 *__restrict__ B = plan.chirp_ft;
  for (int e = threadIdx.x; e < L * m; e += blockDim.x) {
    const int l = e / m, j = e - l * m;
    float2 a = make_float2(0.f, 0.f);
    if (j < n) {
      float2 x = X[l * LS + j];
      if (INV) x.y = -x.y;
      a = cmul(x, w[j]);
    }
    Y[l * LS + j] = a;
  }
  __syncthreads();
  float2 *R = stockham_lines<false>(Y, X, L, LS, plan, tw);
  float2 *F = (R == Y) ? X : Y;
  for (int e = threadIdx.x; e < L * m; e += blockDim.x) {
    const int l = e / m, j = e - l * m;
    R[l * LS + j] = cmul(R[l * LS + j], B[j]);
  }
  __syncthreads();
  float2 *C = stockham_lines<true>(R, F, L, LS, plan, tw);
  for (int e = threadIdx.x; e < L * n; e += blockDim.x) {
    const int l = e / n, k = e - l * n;
    float2 v = cmul(C[l * LS + k], w[k]);
    if (INV) v.y = -v.y;
    C[l * LS + k] = v;
  }
  __syncthreads();
  return C;
}

// Transform L lines held in X (Y is scratch of the same size; line pitch
// LS >= line_pitch(fft_len(plan))).  Returns the buffer holding the result (X or Y), the first
// plan.n slots of each line in natural order.  Caller must __syncthreads() before (X filled) --
// this function syncs after every stage, so the result is visible to all threads on return.
template <bool INV>
__device__ float2 *fft_lines(float2 *X, float2 *Y, int L, int LS, const FftPlan &plan,
                             const float2 *tw) {
  if (plan.m > 0) return bluestein_lines<INV>(X, Y, L, LS, plan, tw);
  return stockham_lines<INV>(X, Y, L, LS, plan, tw);
}

}  // namespace kwb
