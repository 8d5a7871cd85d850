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
#pragma once
#include <algorithm>

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

// Packed FP32 pairs (FADD2 / FMUL2 / FFMA2): per component the same IEEE round-to-nearest
// result as the scalar operation, in one instruction for both components.
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pair(float x) { return make_float2(x, x); }

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
        v[start + k] = padd(a, b);
        v[start + k + span] = rot<INV>(psub(a, b), k * (32 / span));
      }
    }
  }
  float2 t[E];
#pragma unroll
  for (int q = 0; q < E; ++q) t[q] = v[brev<E>(q)];
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = t[q];
}

// cos(2 pi j/120) and sin(2 pi j/120), j = 0..119: the roots of unity of the 12- and 20-point
// register DFTs (exact values to 18 significant digits)
__device__ constexpr float kCos120[120] = {
    1.00000000000000000e+00f, 9.98629534754573833e-01f, 9.94521895368273290e-01f, 9.87688340595137770e-01f,
    9.78147600733805689e-01f, 9.65925826289068312e-01f, 9.51056516295153531e-01f, 9.33580426497201743e-01f,
    9.13545457642600867e-01f, 8.91006524188367899e-01f, 8.66025403784438708e-01f, 8.38670567945424050e-01f,
    8.09016994374947451e-01f, 7.77145961456970902e-01f, 7.43144825477394244e-01f, 7.07106781186547573e-01f,
    6.69130606358858238e-01f, 6.29320391049837502e-01f, 5.87785252292473137e-01f, 5.44639035015027195e-01f,
    5.00000000000000000e-01f, 4.53990499739546804e-01f, 4.06736643075800375e-01f, 3.58367949545300379e-01f,
    3.09016994374947451e-01f, 2.58819045102520739e-01f, 2.07911690817759232e-01f, 1.56434465040230924e-01f,
    1.04528463267653457e-01f, 5.23359562429437444e-02f, 0.00000000000000000e+00f, -5.23359562429436195e-02f,
    -1.04528463267653332e-01f, -1.56434465040230813e-01f, -2.07911690817759343e-01f, -2.58819045102520628e-01f,
    -3.09016994374947340e-01f, -3.58367949545300268e-01f, -4.06736643075800042e-01f, -4.53990499739546693e-01f,
    -5.00000000000000000e-01f, -5.44639035015026751e-01f, -5.87785252292473026e-01f, -6.29320391049837280e-01f,
    -6.69130606358857905e-01f, -7.07106781186547462e-01f, -7.43144825477394022e-01f, -7.77145961456970902e-01f,
    -8.09016994374947340e-01f, -8.38670567945423939e-01f, -8.66025403784438708e-01f, -8.91006524188367788e-01f,
    -9.13545457642600978e-01f, -9.33580426497201743e-01f, -9.51056516295153531e-01f, -9.65925826289068312e-01f,
    -9.78147600733805689e-01f, -9.87688340595137659e-01f, -9.94521895368273401e-01f, -9.98629534754573833e-01f,
    -1.00000000000000000e+00f, -9.98629534754573833e-01f, -9.94521895368273401e-01f, -9.87688340595137770e-01f,
    -9.78147600733805689e-01f, -9.65925826289068423e-01f, -9.51056516295153642e-01f, -9.33580426497201854e-01f,
    -9.13545457642600867e-01f, -8.91006524188367899e-01f, -8.66025403784438819e-01f, -8.38670567945424050e-01f,
    -8.09016994374947562e-01f, -7.77145961456971013e-01f, -7.43144825477394244e-01f, -7.07106781186547684e-01f,
    -6.69130606358858460e-01f, -6.29320391049837835e-01f, -5.87785252292473248e-01f, -5.44639035015026973e-01f,
    -5.00000000000000000e-01f, -4.53990499739546916e-01f, -4.06736643075800874e-01f, -3.58367949545299880e-01f,
    -3.09016994374947562e-01f, -2.58819045102520628e-01f, -2.07911690817759787e-01f, -1.56434465040231035e-01f,
    -1.04528463267654234e-01f, -5.23359562429434252e-02f, 0.00000000000000000e+00f, 5.23359562429439457e-02f,
    1.04528463267652985e-01f, 1.56434465040230675e-01f, 2.07911690817759426e-01f, 2.58819045102521128e-01f,
    3.09016994374947229e-01f, 3.58367949545299547e-01f, 4.06736643075799764e-01f, 4.53990499739546638e-01f,
    5.00000000000000000e-01f, 5.44639035015026640e-01f, 5.87785252292472915e-01f, 6.29320391049836836e-01f,
    6.69130606358858460e-01f, 7.07106781186547351e-01f, 7.43144825477394244e-01f, 7.77145961456970569e-01f,
    8.09016994374947340e-01f, 8.38670567945423606e-01f, 8.66025403784438819e-01f, 8.91006524188367788e-01f,
    9.13545457642600978e-01f, 9.33580426497201521e-01f, 9.51056516295153531e-01f, 9.65925826289068312e-01f,
    9.78147600733805689e-01f, 9.87688340595137659e-01f, 9.94521895368273290e-01f, 9.98629534754573833e-01f};
__device__ constexpr float kSin120[120] = {
    0.00000000000000000e+00f, 5.23359562429438277e-02f, 1.04528463267653457e-01f, 1.56434465040230869e-01f,
    2.07911690817759315e-01f, 2.58819045102520739e-01f, 3.09016994374947396e-01f, 3.58367949545300268e-01f,
    4.06736643075800153e-01f, 4.53990499739546749e-01f, 5.00000000000000000e-01f, 5.44639035015026973e-01f,
    5.87785252292473137e-01f, 6.29320391049837502e-01f, 6.69130606358858238e-01f, 7.07106781186547462e-01f,
    7.43144825477394133e-01f, 7.77145961456970902e-01f, 8.09016994374947451e-01f, 8.38670567945423939e-01f,
    8.66025403784438597e-01f, 8.91006524188367788e-01f, 9.13545457642600867e-01f, 9.33580426497201743e-01f,
    9.51056516295153531e-01f, 9.65925826289068312e-01f, 9.78147600733805689e-01f, 9.87688340595137770e-01f,
    9.94521895368273290e-01f, 9.98629534754573833e-01f, 1.00000000000000000e+00f, 9.98629534754573833e-01f,
    9.94521895368273401e-01f, 9.87688340595137770e-01f, 9.78147600733805689e-01f, 9.65925826289068312e-01f,
    9.51056516295153642e-01f, 9.33580426497201743e-01f, 9.13545457642600978e-01f, 8.91006524188367899e-01f,
    8.66025403784438708e-01f, 8.38670567945424272e-01f, 8.09016994374947451e-01f, 7.77145961456971013e-01f,
    7.43144825477394466e-01f, 7.07106781186547573e-01f, 6.69130606358858349e-01f, 6.29320391049837391e-01f,
    5.87785252292473248e-01f, 5.44639035015027306e-01f, 5.00000000000000000e-01f, 4.53990499739546860e-01f,
    4.06736643075800042e-01f, 3.58367949545300213e-01f, 3.09016994374947507e-01f, 2.58819045102520573e-01f,
    2.07911690817759315e-01f, 1.56434465040230980e-01f, 1.04528463267653290e-01f, 5.23359562429438069e-02f,
    0.00000000000000000e+00f, -5.23359562429435640e-02f, -1.04528463267653055e-01f, -1.56434465040230730e-01f,
    -2.07911690817759065e-01f, -2.58819045102520351e-01f, -3.09016994374947285e-01f, -3.58367949545299991e-01f,
    -4.06736643075800208e-01f, -4.53990499739546693e-01f, -5.00000000000000000e-01f, -5.44639035015027084e-01f,
    -5.87785252292473026e-01f, -6.29320391049837169e-01f, -6.69130606358858238e-01f, -7.07106781186547462e-01f,
    -7.43144825477394022e-01f, -7.77145961456970569e-01f, -8.09016994374947340e-01f, -8.38670567945424050e-01f,
    -8.66025403784438375e-01f, -8.91006524188367788e-01f, -9.13545457642600534e-01f, -9.33580426497201854e-01f,
    -9.51056516295153531e-01f, -9.65925826289068312e-01f, -9.78147600733805578e-01f, -9.87688340595137659e-01f,
    -9.94521895368273290e-01f, -9.98629534754573944e-01f, -1.00000000000000000e+00f, -9.98629534754573833e-01f,
    -9.94521895368273401e-01f, -9.87688340595137770e-01f, -9.78147600733805578e-01f, -9.65925826289068201e-01f,
    -9.51056516295153642e-01f, -9.33580426497202076e-01f, -9.13545457642601089e-01f, -8.91006524188368010e-01f,
    -8.66025403784438597e-01f, -8.38670567945424272e-01f, -8.09016994374947562e-01f, -7.77145961456971346e-01f,
    -7.43144825477394022e-01f, -7.07106781186547684e-01f, -6.69130606358858127e-01f, -6.29320391049837835e-01f,
    -5.87785252292473359e-01f, -5.44639035015027750e-01f, -5.00000000000000000e-01f, -4.53990499739546971e-01f,
    -4.06736643075800153e-01f, -3.58367949545300768e-01f, -3.09016994374947618e-01f, -2.58819045102520684e-01f,
    -2.07911690817758982e-01f, -1.56434465040231119e-01f, -1.04528463267653415e-01f, -5.23359562429443689e-02f};

// x * exp(-+2 pi i m/E) for compile-time m and E (E divides 120)
template <int E, bool INV>
__device__ __forceinline__ float2 rotE(float2 x, int m) {
  m %= E;
  if (m == 0) return x;
  const int j = m * (120 / E);
  if (j == 30) return mul_mi<INV>(x);
  if (j == 60) return make_float2(-x.x, -x.y);
  if (j == 90) return mul_mi<!INV>(x);
  const float c = kCos120[j];
  const float s = INV ? -kSin120[j] : kSin120[j];
  return make_float2(fmaf(x.x, c, x.y * s), fmaf(x.y, c, -x.x * s));
}

// E-point DFT in registers, natural order in and out, for E = 2^a (dft_reg), 3, 5, or an odd
// prime P in {3, 5} times a smaller such length Q (one Cooley-Tukey step, n = Q n1 + n2,
// k = k1 + P k2: P-point DFTs over n1, twiddles exp(-2 pi i n2 k1/E), Q-point DFTs over n2).
template <int E, bool INV>
__device__ __forceinline__ void dft_mixed(float2 (&v)[E]) {
  if constexpr ((E & (E - 1)) == 0) {
    dft_reg<E, INV>(v);
  } else if constexpr (E == 3 || E == 5) {
    Dft<E, INV>::run(v);
  } else {
    constexpr int P = (E % 3 == 0) ? 3 : 5;
    constexpr int Q = E / P;
    static_assert(P * Q == E && 120 % E == 0, "register DFT length");
    float2 a[E];
#pragma unroll
    for (int n2 = 0; n2 < Q; ++n2) {
      float2 w[P];
#pragma unroll
      for (int n1 = 0; n1 < P; ++n1) w[n1] = v[Q * n1 + n2];
      Dft<P, INV>::run(w);
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) a[n2 * P + k1] = rotE<E, INV>(w[k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      float2 w[Q];
#pragma unroll
      for (int n2 = 0; n2 < Q; ++n2) w[n2] = a[n2 * P + k1];
      dft_mixed<Q, INV>(w);
#pragma unroll
      for (int k2 = 0; k2 < Q; ++k2) v[k1 + P * k2] = w[k2];
    }
  }
}

__device__ __forceinline__ float2 cmul_conj(float2 a, float2 w) {  // a * conj(w)
  return make_float2(fmaf(a.x, w.x, a.y * w.y), fmaf(a.y, w.x, -a.x * w.y));
}

// N = E*G point transform of the line owned by this thread's group.  xs: the line's exchange
// buffer (E rows of pitch G+1); tw2: exp(-2 pi i t q/N) at [q*(G+1) + t].
template <int E_, int G_, bool WARP>
struct LineFFT {
  static constexpr int E = E_, G = G_;
  static constexpr int N = E * G, J = E / G, RP = G + 1, LP = E * RP + 1;
  static_assert(E % G == 0, "G must divide E");
  static constexpr bool WARP_SYNC = WARP;  // one line per warp: exchanges need only __syncwarp
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
  __host__ __device__ __forceinline__ static int k_of(int t, int idx) { return t * J + idx / G + E * (idx % G); }
  __device__ __forceinline__ static int nat(int k) { return k; }  // natural-order spectrum slot
  __device__ __forceinline__ static int nat_of(int t, int idx) { return k_of(t, idx); }
  // per-CTA twiddle table: exp(-2 pi i t q/N) at [q*(G+1) + t]
  static constexpr int TW = E * RP;
  __device__ __forceinline__ static void build_tw(float2 *tw2, const float2 *tw) {
    for (int e = threadIdx.x; e < E * G; e += blockDim.x) {
      const int q = e / G, u = e - q * G;
      tw2[q * RP + u] = tw[u * q];
    }
  }
};

// N = R1 * A * B point transform of one line owned by G = A*B threads, each holding E = R1
// elements (three levels, two shared-memory exchanges): an R1-point DFT in registers over
// x[t + G r]; twiddle exp(-2 pi i t q1/N); exchange; for each (q1, a) a B-point DFT over b of
// the values at t = a + A b, twiddle exp(-2 pi i a m_b/G); exchange; for each (q1, m_b) an
// A-point DFT over a, giving X[q1 + R1 (m_b + B m_a)].  Fewer registers per thread than the
// two-level form (E = 8 for N = 128..512), so twice the resident warps.
template <int R1, int A, int B, bool WARP>
struct LineFFT3 {
  static constexpr int E = R1, G = A * B, N = R1 * A * B;
  static constexpr int P2 = R1 / B, P3 = R1 / A;  // (q1, a) and (q1, m_b) pairs per thread
  static_assert(R1 % A == 0 && R1 % B == 0, "A and B must divide R1");
  static constexpr int RP = G + 1;                 // pitch of the level-1 twiddle table
  static constexpr int AP = A + 1;                 // pitch of the level-2 twiddle table
  // Exchange layouts.  Each is a sum of one term per index (affine in the parts), so every
  // access is a per-thread base plus a compile-time offset, and the pads are chosen so that the
  // exchanges of a line held by one warp (contiguous passes) hit distinct banks in every stage:
  //   level 1  [q][u]          q * RP1 + u
  //   level 2  [q1][m_b][a]    q1 * Q2 + beta2(m_b) + a
  //   natural  k = q1 + R1 (m_b + B m_a)  ->  q1 + beta3(m_b) + m_a * ZS   (EOS pair split)
  // A line occupies LP (odd) slots, so lines held by one warp in strided passes, which all use
  // the same offset within their line, also hit distinct banks.
  static constexpr int PI = R1 == 16 ? 3 : A == 2 ? 0 : A == 4 ? 1 : 2;
  static constexpr int RP1 = PI == 3 ? 65 : G + A;
  static constexpr int M2 = PI == 0 ? 2 : PI == 1 ? 4 : PI == 2 ? 9 : 8, X2 = PI == 1 || PI == 3 ? 1 : 0;
  static constexpr int Z2 = PI == 0 ? 1 : 0, Q2 = PI == 0 ? 18 : PI == 1 ? 36 : PI == 2 ? 72 : 68;
  static constexpr int M3 = PI == 3 ? 16 : 8, X3 = PI == 2 ? 2 : 4, ZS = PI == 3 ? 140 : PI == 2 ? 70 : 76;
  __host__ __device__ static constexpr int beta2(int mb) { return mb * M2 + (mb >> 1) * X2 + (mb >> 2) * Z2; }
  __host__ __device__ static constexpr int beta3(int mb) { return mb * M3 + (mb >> 1) * X3; }
  static constexpr int S1 = (R1 - 1) * RP1 + G, S2 = (R1 - 1) * Q2 + beta2(B - 1) + A;
  static constexpr int S3 = R1 + beta3(B - 1) + (A - 1) * ZS;
  static constexpr int SM = S1 > S2 ? (S1 > S3 ? S1 : S3) : (S2 > S3 ? S2 : S3);
  static constexpr int LP = SM | 1;
  static constexpr int TW = R1 * RP + B * AP;      // level-1 then level-2 twiddles
  __device__ __forceinline__ static int i1(int q, int u) { return q * RP1 + u; }
  __device__ __forceinline__ static int i2(int q1, int mb, int a) { return q1 * Q2 + beta2(mb) + a; }
  __device__ __forceinline__ static int nat3(int q1, int mb, int ma) { return q1 + beta3(mb) + ma * ZS; }
  __device__ __forceinline__ static int nat(int k) { return nat3(k % R1, (k / R1) % B, k / (R1 * B)); }
  // slot of register idx of thread t (the k_of position) in the natural-order layout
  __device__ __forceinline__ static int nat_of(int t, int idx) {
    const int p0 = t * P3, q1 = p0 / B, mb = p0 - q1 * B + idx / A;  // B is a multiple of P3
    return nat3(q1, mb, idx % A);
  }
  static constexpr bool WARP_SYNC = WARP;  // one line per warp: exchanges need only __syncwarp
  __device__ __forceinline__ static void sync() {
    if (WARP) __syncwarp();
    else __syncthreads();
  }
  __device__ __forceinline__ static void build_tw(float2 *tw, const float2 *g) {
    for (int e = threadIdx.x; e < R1 * G; e += blockDim.x) {
      const int q = e / G, u = e - q * G;
      tw[q * RP + u] = g[u * q];  // exp(-2 pi i u q / N)
    }
    for (int e = threadIdx.x; e < A * B; e += blockDim.x) {
      const int mb = e / A, a = e - mb * A;
      tw[R1 * RP + mb * AP + a] = g[a * mb * R1];  // exp(-2 pi i a m_b / G)
    }
  }
  // in: v[r] = x[t + G r]; out: v[j*A + m_a] = X[q1 + R1 (m_b + B m_a)], (q1, m_b) = pair t*P3 + j
  __device__ __forceinline__ static void fwd(float2 (&v)[E], float2 *xs, const float2 *tw, int t) {
    dft_reg<R1, false>(v);
#pragma unroll
    for (int q = 0; q < R1; ++q) xs[i1(q, t)] = q == 0 ? v[q] : cmul(v[q], tw[q * RP + t]);
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / A, a = p - q1 * A;
      float2 w[B];
#pragma unroll
      for (int b = 0; b < B; ++b) w[b] = xs[i1(q1, a + A * b)];
      dft_reg<B, false>(w);
#pragma unroll
      for (int mb = 0; mb < B; ++mb) v[j * B + mb] = mb == 0 ? w[mb] : cmul(w[mb], tw[R1 * RP + mb * AP + a]);
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / A, a = p - q1 * A;
#pragma unroll
      for (int mb = 0; mb < B; ++mb) xs[i2(q1, mb, a)] = v[j * B + mb];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P3; ++j) {
      const int p = t * P3 + j, q1 = p / B, mb = p - q1 * B;
      float2 w[A];
#pragma unroll
      for (int a = 0; a < A; ++a) w[a] = xs[i2(q1, mb, a)];
      dft_reg<A, false>(w);
#pragma unroll
      for (int ma = 0; ma < A; ++ma) v[j * A + ma] = w[ma];
    }
    sync();
  }
  // exact reverse of fwd with conjugate twiddles (unnormalised); out: v[r] = x[t + G r]
  __device__ __forceinline__ static void inv(float2 (&v)[E], float2 *xs, const float2 *tw, int t) {
#pragma unroll
    for (int j = 0; j < P3; ++j) {
      const int p = t * P3 + j, q1 = p / B, mb = p - q1 * B;
      float2 w[A];
#pragma unroll
      for (int ma = 0; ma < A; ++ma) w[ma] = v[j * A + ma];
      dft_reg<A, true>(w);
#pragma unroll
      for (int a = 0; a < A; ++a) xs[i2(q1, mb, a)] = w[a];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / A, a = p - q1 * A;
      float2 w[B];
#pragma unroll
      for (int mb = 0; mb < B; ++mb) w[mb] = mb == 0 ? xs[i2(q1, mb, a)] : cmul_conj(xs[i2(q1, mb, a)], tw[R1 * RP + mb * AP + a]);
      dft_reg<B, true>(w);
#pragma unroll
      for (int b = 0; b < B; ++b) v[j * B + b] = w[b];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / A, a = p - q1 * A;
#pragma unroll
      for (int b = 0; b < B; ++b) xs[i1(q1, a + A * b)] = v[j * B + b];
    }
    sync();
#pragma unroll
    for (int q = 0; q < R1; ++q) v[q] = q == 0 ? xs[i1(q, t)] : cmul_conj(xs[i1(q, t)], tw[q * RP + t]);
    dft_reg<R1, true>(v);
    sync();
  }
  __host__ __device__ __forceinline__ static int k_of(int t, int idx) {
    const int p = t * P3 + idx / A, q1 = p / B, mb = p - q1 * B, ma = idx % A;
    return q1 + R1 * (mb + B * ma);
  }
};

// LineFFT3 for mixed-radix lengths: N = R1 * A * B with R1 = 12 or 20 (a register DFT of 3 or 5
// times a power of two) and A, B dividing R1 (register DFTs of 2, 3, 4, 5, 6, 10 or 12 points),
// e.g. 96 = 12*2*4, 192 = 12*4*4, 160 = 20*2*4, 320 = 20*4*4, 288 = 12*4*6, 1000 = 20*5*10.
// Same three levels and the same register layouts as LineFFT3; the exchange buffers use generic
// padding (odd pitches) instead of LineFFT3's tuned offsets, and the natural-order slots pad one
// per 32.  With G = A*B not dividing 32, a line's threads span warps and WARP must be false.
template <int R1, int A, int B, bool WARP>
struct LineFFT3G {
  static constexpr int E = R1, G = A * B, N = R1 * A * B;
  static constexpr int P2 = R1 / B, P3 = R1 / A;
  static_assert(R1 % A == 0 && R1 % B == 0, "LineFFT3G shape: A and B divide R1");
  static constexpr int RP = G + 1;   // level-1 twiddle pitch
  static constexpr int AP = A + 1;   // level-2 twiddle pitch
  static constexpr int RP1 = G + 1;  // level-1 exchange [q][u]
  static constexpr int M2 = A + 1, Q2 = B * M2 + 1;  // level-2 exchange [q1][mb][a]
  __host__ __device__ static constexpr int nat(int k) { return k + (k >> 5); }
  static constexpr int S1 = (R1 - 1) * RP1 + G, S2 = (R1 - 1) * Q2 + (B - 1) * M2 + A, S3 = N + (N >> 5);
  static constexpr int SM = S1 > S2 ? (S1 > S3 ? S1 : S3) : (S2 > S3 ? S2 : S3);
  static constexpr int LP = SM | 1;
  static constexpr int TW = R1 * RP + B * AP;
  __device__ __forceinline__ static int i1(int q, int u) { return q * RP1 + u; }
  __device__ __forceinline__ static int i2(int q1, int mb, int a) { return q1 * Q2 + mb * M2 + a; }
  static constexpr bool WARP_SYNC = WARP;
  __device__ __forceinline__ static void sync() {
    if (WARP) __syncwarp();
    else __syncthreads();
  }
  __host__ __device__ __forceinline__ static int k_of(int t, int idx) {
    const int p = t * P3 + idx / A, q1 = p / B, mb = p - q1 * B, ma = idx % A;
    return q1 + R1 * (mb + B * ma);
  }
  __device__ __forceinline__ static int nat_of(int t, int idx) { return nat(k_of(t, idx)); }
  __device__ __forceinline__ static void build_tw(float2 *tw, const float2 *g) {
    for (int e = threadIdx.x; e < R1 * G; e += blockDim.x) {
      const int q = e / G, u = e - q * G;
      tw[q * RP + u] = g[u * q];  // exp(-2 pi i u q / N)
    }
    for (int e = threadIdx.x; e < A * B; e += blockDim.x) {
      const int mb = e / A, a = e - mb * A;
      tw[R1 * RP + mb * AP + a] = g[a * mb * R1];  // exp(-2 pi i a m_b / G)
    }
  }
  // in: v[r] = x[t + G r]; out: v[j*A + m_a] = X[q1 + R1 (m_b + B m_a)], (q1, m_b) = pair t*P3 + j
  __device__ __forceinline__ static void fwd(float2 (&v)[E], float2 *xs, const float2 *tw, int t) {
    dft_mixed<R1, false>(v);
#pragma unroll
    for (int q = 0; q < R1; ++q) xs[i1(q, t)] = q == 0 ? v[q] : cmul(v[q], tw[q * RP + t]);
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / A, a = p - q1 * A;
      float2 w[B];
#pragma unroll
      for (int b = 0; b < B; ++b) w[b] = xs[i1(q1, a + A * b)];
      dft_mixed<B, false>(w);
#pragma unroll
      for (int mb = 0; mb < B; ++mb) v[j * B + mb] = mb == 0 ? w[mb] : cmul(w[mb], tw[R1 * RP + mb * AP + a]);
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / A, a = p - q1 * A;
#pragma unroll
      for (int mb = 0; mb < B; ++mb) xs[i2(q1, mb, a)] = v[j * B + mb];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P3; ++j) {
      const int p = t * P3 + j, q1 = p / B, mb = p - q1 * B;
      float2 w[A];
#pragma unroll
      for (int a = 0; a < A; ++a) w[a] = xs[i2(q1, mb, a)];
      dft_mixed<A, false>(w);
#pragma unroll
      for (int ma = 0; ma < A; ++ma) v[j * A + ma] = w[ma];
    }
    sync();
  }
  // exact reverse of fwd with conjugate twiddles (unnormalised); out: v[r] = x[t + G r]
  __device__ __forceinline__ static void inv(float2 (&v)[E], float2 *xs, const float2 *tw, int t) {
#pragma unroll
    for (int j = 0; j < P3; ++j) {
      const int p = t * P3 + j, q1 = p / B, mb = p - q1 * B;
      float2 w[A];
#pragma unroll
      for (int ma = 0; ma < A; ++ma) w[ma] = v[j * A + ma];
      dft_mixed<A, true>(w);
#pragma unroll
      for (int a = 0; a < A; ++a) xs[i2(q1, mb, a)] = w[a];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / A, a = p - q1 * A;
      float2 w[B];
#pragma unroll
      for (int mb = 0; mb < B; ++mb) w[mb] = mb == 0 ? xs[i2(q1, mb, a)] : cmul_conj(xs[i2(q1, mb, a)], tw[R1 * RP + mb * AP + a]);
      dft_mixed<B, true>(w);
#pragma unroll
      for (int b = 0; b < B; ++b) v[j * B + b] = w[b];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / A, a = p - q1 * A;
#pragma unroll
      for (int b = 0; b < B; ++b) xs[i1(q1, a + A * b)] = v[j * B + b];
    }
    sync();
#pragma unroll
    for (int q = 0; q < R1; ++q) v[q] = q == 0 ? xs[i1(q, t)] : cmul_conj(xs[i1(q, t)], tw[q * RP + t]);
    dft_mixed<R1, true>(v);
    sync();
  }
};

// Four levels for longer mixed-radix lines: N = R1 * A * B * C with A, B, C powers of two
// dividing R1 (384 = 12*4*4*2, 768 = 12*4*4*4), G = A*B*C threads per line.  The G-point DFT
// over u = a + A (b + B c) is split three ways (m = m_c + C (m_b + B m_a)):
//   Y[m] = sum_a w_A^{a m_a} w_G^{a (m_c + C m_b)} sum_b w_B^{b m_b} w_BC^{b m_c} sum_c w_C^{c m_c} y[u],
// so after the R1-point register DFT and its twiddles, level 2 takes C-point DFTs over c (twiddle
// w_BC^{b m_c}), level 3 B-point DFTs over b (twiddle w_G^{a (m_c + C m_b)}) and level 4
// A-point DFTs over a; thread t then holds X[q1 + R1 (m_c + C (m_b + B m_a))].  Exchanges use
// generic odd pitches.
template <int R1, int A, int B, int C, bool WARP>
struct LineFFT4G {
  static constexpr int E = R1, G = A * B * C, N = R1 * A * B * C;
  static constexpr int P2 = R1 / C, P3 = R1 / B, P4 = R1 / A;
  static_assert(R1 % A == 0 && R1 % B == 0 && R1 % C == 0, "LineFFT4G shape");
  static constexpr int RP = G + 1;  // level-1 twiddle pitch and exchange pitch
  // exchange layouts: level 1 [q][u]; level 2 [q1][a][m_c][b]; level 3 [q1][m_b][m_c][a]
  static constexpr int Q2 = A * (C * (B + 1)) + 1, Q3 = B * (C * (A + 1)) + 1;
  __host__ __device__ static constexpr int nat(int k) { return k + (k >> 5); }
  __device__ __forceinline__ static int i1(int q, int u) { return q * RP + u; }
  __device__ __forceinline__ static int i2(int q1, int a, int mc, int b) { return q1 * Q2 + (a * C + mc) * (B + 1) + b; }
  __device__ __forceinline__ static int i3(int q1, int mb, int mc, int a) { return q1 * Q3 + (mb * C + mc) * (A + 1) + a; }
  static constexpr int S1 = (R1 - 1) * RP + G, S2 = R1 * Q2, S3 = R1 * Q3, S4 = N + (N >> 5);
  static constexpr int SA = S1 > S2 ? S1 : S2, SB = S3 > S4 ? S3 : S4, SM = SA > SB ? SA : SB;
  static constexpr int LP = SM | 1;
  // twiddles: level 1 exp(-2 pi i u q/N) [q][u]; level 2 w_BC^{b m_c} [m_c][b];
  // level 3 w_G^{a (m_c + C m_b)} [m_b][m_c][a]
  static constexpr int T2 = R1 * RP, T3 = T2 + C * (B + 1);
  static constexpr int TW = T3 + B * C * (A + 1);
  static constexpr bool WARP_SYNC = WARP;
  __device__ __forceinline__ static void sync() {
    if (WARP) __syncwarp();
    else __syncthreads();
  }
  // level-4 work item p = t P4 + j -> (q1, m_b, m_c) = p in [R1][B][C] order
  __host__ __device__ __forceinline__ static int k_of(int t, int idx) {
    const int p = t * P4 + idx / A, q1 = p / (B * C), r = p - q1 * B * C, mb = r / C, mc = r - mb * C;
    return q1 + R1 * (mc + C * (mb + B * (idx % A)));
  }
  __device__ __forceinline__ static int nat_of(int t, int idx) { return nat(k_of(t, idx)); }
  __device__ __forceinline__ static void build_tw(float2 *tw, const float2 *g) {
    for (int e = threadIdx.x; e < R1 * G; e += blockDim.x) {
      const int q = e / G, u = e - q * G;
      tw[q * RP + u] = g[u * q];
    }
    constexpr int NG = N / G;  // g[j NG] = exp(-2 pi i j/G)
    for (int e = threadIdx.x; e < C * B; e += blockDim.x) {
      const int mc = e / B, b = e - mc * B;
      tw[T2 + mc * (B + 1) + b] = g[NG * A * b * mc];  // w_BC^{b m_c} = w_G^{A b m_c}
    }
    for (int e = threadIdx.x; e < B * C * A; e += blockDim.x) {
      const int mb = e / (C * A), r = e - mb * C * A, mc = r / A, a = r - mc * A;
      tw[T3 + (mb * C + mc) * (A + 1) + a] = g[NG * ((a * (mc + C * mb)) % G)];
    }
  }
  __device__ __forceinline__ static void fwd(float2 (&v)[E], float2 *xs, const float2 *tw, int t) {
    dft_mixed<R1, false>(v);
#pragma unroll
    for (int q = 0; q < R1; ++q) xs[i1(q, t)] = q == 0 ? v[q] : cmul(v[q], tw[q * RP + t]);
    sync();
    // level 2: (q1, a, b) = t P2 + j in [R1][A][B] order; C-point DFT over c
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / (A * B), r = p - q1 * A * B, a = r / B, b = r - a * B;
      float2 w[C];
#pragma unroll
      for (int c = 0; c < C; ++c) w[c] = xs[i1(q1, a + A * (b + B * c))];
      dft_reg<C, false>(w);
#pragma unroll
      for (int mc = 0; mc < C; ++mc) v[j * C + mc] = (mc == 0 || b == 0) ? w[mc] : cmul(w[mc], tw[T2 + mc * (B + 1) + b]);
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / (A * B), r = p - q1 * A * B, a = r / B, b = r - a * B;
#pragma unroll
      for (int mc = 0; mc < C; ++mc) xs[i2(q1, a, mc, b)] = v[j * C + mc];
    }
    sync();
    // level 3: (q1, a, m_c) = t P3 + j in [R1][A][C] order; B-point DFT over b
#pragma unroll
    for (int j = 0; j < P3; ++j) {
      const int p = t * P3 + j, q1 = p / (A * C), r = p - q1 * A * C, a = r / C, mc = r - a * C;
      float2 w[B];
#pragma unroll
      for (int b = 0; b < B; ++b) w[b] = xs[i2(q1, a, mc, b)];
      dft_reg<B, false>(w);
#pragma unroll
      for (int mb = 0; mb < B; ++mb) v[j * B + mb] = a == 0 ? w[mb] : cmul(w[mb], tw[T3 + (mb * C + mc) * (A + 1) + a]);
    }
    sync();
#pragma unroll
    for (int j = 0; j < P3; ++j) {
      const int p = t * P3 + j, q1 = p / (A * C), r = p - q1 * A * C, a = r / C, mc = r - a * C;
#pragma unroll
      for (int mb = 0; mb < B; ++mb) xs[i3(q1, mb, mc, a)] = v[j * B + mb];
    }
    sync();
    // level 4: (q1, m_b, m_c) = t P4 + j in [R1][B][C] order; A-point DFT over a
#pragma unroll
    for (int j = 0; j < P4; ++j) {
      const int p = t * P4 + j, q1 = p / (B * C), r = p - q1 * B * C, mb = r / C, mc = r - mb * C;
      float2 w[A];
#pragma unroll
      for (int a = 0; a < A; ++a) w[a] = xs[i3(q1, mb, mc, a)];
      dft_reg<A, false>(w);
#pragma unroll
      for (int ma = 0; ma < A; ++ma) v[j * A + ma] = w[ma];
    }
    sync();
  }
  // exact reverse of fwd with conjugate twiddles (unnormalised); out: v[r] = x[t + G r]
  __device__ __forceinline__ static void inv(float2 (&v)[E], float2 *xs, const float2 *tw, int t) {
#pragma unroll
    for (int j = 0; j < P4; ++j) {
      const int p = t * P4 + j, q1 = p / (B * C), r = p - q1 * B * C, mb = r / C, mc = r - mb * C;
      float2 w[A];
#pragma unroll
      for (int ma = 0; ma < A; ++ma) w[ma] = v[j * A + ma];
      dft_reg<A, true>(w);
#pragma unroll
      for (int a = 0; a < A; ++a) xs[i3(q1, mb, mc, a)] = w[a];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P3; ++j) {
      const int p = t * P3 + j, q1 = p / (A * C), r = p - q1 * A * C, a = r / C, mc = r - a * C;
      float2 w[B];
#pragma unroll
      for (int mb = 0; mb < B; ++mb)
        w[mb] = a == 0 ? xs[i3(q1, mb, mc, a)] : cmul_conj(xs[i3(q1, mb, mc, a)], tw[T3 + (mb * C + mc) * (A + 1) + a]);
      dft_reg<B, true>(w);
#pragma unroll
      for (int b = 0; b < B; ++b) v[j * B + b] = w[b];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P3; ++j) {
      const int p = t * P3 + j, q1 = p / (A * C), r = p - q1 * A * C, a = r / C, mc = r - a * C;
#pragma unroll
      for (int b = 0; b < B; ++b) xs[i2(q1, a, mc, b)] = v[j * B + b];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / (A * B), r = p - q1 * A * B, a = r / B, b = r - a * B;
      float2 w[C];
#pragma unroll
      for (int mc = 0; mc < C; ++mc)
        w[mc] = (mc == 0 || b == 0) ? xs[i2(q1, a, mc, b)] : cmul_conj(xs[i2(q1, a, mc, b)], tw[T2 + mc * (B + 1) + b]);
      dft_reg<C, true>(w);
#pragma unroll
      for (int c = 0; c < C; ++c) v[j * C + c] = w[c];
    }
    sync();
#pragma unroll
    for (int j = 0; j < P2; ++j) {
      const int p = t * P2 + j, q1 = p / (A * B), r = p - q1 * A * B, a = r / B, b = r - a * B;
#pragma unroll
      for (int c = 0; c < C; ++c) xs[i1(q1, a + A * (b + B * c))] = v[j * C + c];
    }
    sync();
#pragma unroll
    for (int q = 0; q < R1; ++q) v[q] = q == 0 ? xs[i1(q, t)] : cmul_conj(xs[i1(q, t)], tw[q * RP + t]);
    dft_mixed<R1, true>(v);
    sync();
  }
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

// Line-pass tables for an FFT policy F: twiddles, then the gradient multipliers i k e^{+-ikd/2}/N
// in register order [idx][t] (pitch G+1).
template <class F>
__device__ __forceinline__ void build_line_tables(float2 *tw, float2 *gp2, float2 *gn2, const float2 *g,
                                                  const float2 *gpos, const float2 *gneg) {
  F::build_tw(tw, g);
  constexpr int RP = F::G + 1;
  for (int e = threadIdx.x; e < F::E * F::G; e += blockDim.x) {
    const int q = e / F::G, u = e - q * F::G;
    const int k = F::k_of(u, q);
    gp2[q * RP + u] = gpos[k];
    gn2[q * RP + u] = gneg[k];
  }
}
// Register line pass: exchange buffers, twiddles and gradient tables, then the two staged operand
// tiles, 128-byte aligned (destinations of tiled TMA copies).
template <class F>
__host__ __device__ constexpr size_t pline_offset(int L) {
  return (((size_t)L * F::LP + F::TW + 2 * (size_t)F::E * (F::G + 1)) * sizeof(float2) + 127) & ~size_t(127);
}
template <class F>
__host__ __device__ constexpr size_t pline_smem(int L) {
  return pline_offset<F>(L) + 2 * (size_t)(2 * L) * F::N * sizeof(float);
}

template <int E, int G>
__host__ __device__ constexpr size_t line_smem(int L) {
  return ((size_t)L * (E * (G + 1) + 1) + 3 * (size_t)E * (G + 1)) * sizeof(float2);
}
// Line pass: the exchange buffers and tables, then two staged operand tiles (p and rho0) of
// 2L real lines x N floats each, 16-byte aligned.
template <int E, int G>
__host__ __device__ constexpr size_t line_stage_offset(int L) {
  return (line_smem<E, G>(L) + 15) & ~size_t(15);
}
template <int E, int G>
__host__ __device__ constexpr size_t line_smem_staged(int L) {
  return line_stage_offset<E, G>(L) + 2 * (size_t)(2 * L) * (E * G) * sizeof(float);
}

// 16-byte asynchronous global->shared copy; bytes beyond src_bytes are zero-filled.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Bulk (TMA) copies global -> shared completing on an mbarrier (no multicast).
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
// order this thread's earlier generic-proxy accesses of shared memory before async-proxy writes
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *m, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(m))
               : "memory");
}
// Tiled tensor copy (TMA) of one box of a 3-D tensor map into shared memory, completing on the
// mbarrier with the box's byte count.  The map lives in the kernel's parameter space; x is the
// innermost coordinate (a multiple of 4 FP32 elements, 16 bytes); no multicast.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *m) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(m))
      : "memory");
}
// Bulk prefetch of a contiguous block into L2 (16-byte aligned address and size).
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *m, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for phase `parity` of an mbarrier, giving up after about 2^30 SM clocks (half a second):
// false means the copies it tracks did not complete, which the caller reports instead of hanging.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *m, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(m, parity))
    if (clock64() - t0 > (1LL << 30)) return false;
  return true;
}

// ------------------------------------------------------------------------------------------
// fused per-axis line pass (same algorithm as kwb::k_line_pass)
// ------------------------------------------------------------------------------------------

// XEOS (x axis, time steps only): the pass ends with the equation of state's x R2C for its tile,
// as k_eos_fwd_fast does, starting from rho_x still in registers (rho_y and rho_z are final:
// the x pass runs last).
// STMA (strided passes): the instantiation that can stage its tiles by tiled TMA copies; the
// other one is the plain 16-byte cp.async pass.
template <class F, bool CONTIG, int LT, int MINB, bool XEOS, bool STMA = false>
__global__ void __launch_bounds__(LT * F::G, MINB)
    k_line_fast(const __grid_constant__ SimDev S, int axis, int mode, long long step_s) {
  constexpr int E = F::E, G = F::G;
  constexpr int RP = G + 1, LP = F::LP;
  constexpr int L = LT;  // complex lines per tile
  extern __shared__ __align__(128) float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  float2 *gp2 = tw2 + F::TW;
  float2 *gn2 = gp2 + E * RP;
  // Contiguous tiles are 2L whole consecutive rows, so each field's tile is one block of
  // memory: one bulk (TMA) copy per field.  Strided tiles (2L columns of N rows) are boxes of
  // the field's tensor map: N / tile_box_rows tiled TMA copies per field.  Each field's copies
  // complete on its own mbarrier (0 p, 1 rho0, 2 u_d, 3 rho_d; each used for one phase).
  // Tiled copies need 16-byte box rows and x offsets (2L a multiple of 4) and 128-byte aligned
  // destinations (the staged tiles and each box within them; the host checks the box sizes).
  constexpr bool TMA_S_OK = STMA && !CONTIG && (2 * LT) % 4 == 0;
  const bool tma = CONTIG ? (S.tma_line[axis] >= 0 ? S.tma_line[axis] : S.tile_tma) != 0
                          : (TMA_S_OK && S.tile_tma_s != 0 && S.tile_box_rows > 0 && F::N % S.tile_box_rows == 0 &&
                             ((smem_u32(smem_raw) + (unsigned)pline_offset<F>(LT)) & 127u) == 0);
  __shared__ __align__(8) unsigned long long tile_bar[4];
  if (tma && threadIdx.x == 0) {
#pragma unroll
    for (int b = 0; b < 4; ++b) mbar_init(&tile_bar[b], 1);
  }
  // the tables are written once at set-up: built before waiting on the previous kernel
  build_line_tables<F>(tw2, gp2, gn2, S.tw[axis], S.gpos[axis], S.gneg[axis]);
  if (tma) __syncthreads();  // the mbarriers are initialised for every thread
  KWB_STEP_KERNEL_PROLOGUE();
  const long long t = *S.t0 + step_s;
  if (mode == KWB_MODE_STEP && t >= S.Nt) return;
  // once a wait has given up, the simulation is failed: later tiles exit at once instead of each
  // waiting out its budget (uniform over the CTA: one load before any thread diverges)
  if (tma && *reinterpret_cast<volatile const int *>(S.err) != 0) return;
  const int tid = threadIdx.x;
  const int tt = CONTIG ? tid % G : tid / L;
  const int l = CONTIG ? tid / G : tid % L;
  constexpr int N = E * G, THREADS = LT * G;
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
  // Element (column c, position i) sits at off(c, i) from `base`; 32-bit offsets (grids are
  // limited to 2^31 voxels).  Strided tiles read the two columns of a pair as one float2 (the
  // row pitch is even on this path), zero-filling a pair that lies past the grid edge.
  const int st32 = (int)stride;
  auto off = [&](int c, int i) -> int { return CONTIG ? c * Nx + i : i * st32 + c; };
  auto load_pair = [&](const float *__restrict__ f, int i) -> float2 {
    const float *fb = f + base;
    if (!CONTIG) return vb ? __ldg(reinterpret_cast<const float2 *>(fb + off(2 * l, i))) : make_float2(0.f, 0.f);
    return make_float2(va ? __ldg(fb + off(2 * l, i)) : 0.f, vb ? __ldg(fb + off(2 * l + 1, i)) : 0.f);
  };
  auto store_pair = [&](float *f, int i, float2 v) {
    float *fb = f + base;
    if (!CONTIG) {
      if (vb) *reinterpret_cast<float2 *>(fb + off(2 * l, i)) = v;
      return;
    }
    if (va) fb[off(2 * l, i)] = v.x;
    if (vb) fb[off(2 * l + 1, i)] = v.y;
  };

  // Stage the p tile (and the rho0 tile when density varies) into shared memory with
  // asynchronous 16-byte copies: every load of the tile is in flight at once, overlapping the
  // table set-up and, for rho0, the first transform.  Staged layout: CONTIG [row][i],
  // strided [i][column] (the tile's own global layout, compacted).
  float *st_p = reinterpret_cast<float *>(reinterpret_cast<char *>(smem_raw) + pline_offset<F>(L));
  float *st_r = st_p + 2 * L * N;
  // Chunk assignments are compile-time strides from a per-thread start, so the addresses of a
  // thread's chunks differ by constants.
  auto stage = [&](float *dst, const float *f, int slot) {
    const float *fb = f + base;
    if (CONTIG && tma) {
      // rows contiguous in memory: one bulk copy of cnt rows (16-byte aligned: N % 4 == 0)
      if (tid == 0) {
        const unsigned bytes = (unsigned)cnt * N * 4u;
        fence_proxy_async_smem();
        mbar_expect_tx(&tile_bar[slot], bytes);
        if (!(S.test_drop_copy && slot == 0 && blockIdx.x == 0)) bulk_copy_g2s(dst, fb, bytes, &tile_bar[slot]);
      }
      return;
    } else if (!CONTIG && tma) {
      // the tile is a box of the field's tensor map, N / BR boxes of BR positions: columns past
      // the grid edge arrive as zeros (the map's out-of-bounds fill)
      if (tid == 0) {
        // the tile's first column and its fixed (z or y) index, recomputed here rather than kept
        // live through the transforms
        const int tpp = (Nx + 2 * L - 1) / (2 * L);
        const int to = blockIdx.x / tpp, tx0 = (blockIdx.x - to * tpp) * 2 * L;
        const int BR = S.tile_box_rows;
        fence_proxy_async_smem();
        mbar_expect_tx(&tile_bar[slot], (unsigned)(2 * L * N * 4));
        if (!(S.test_drop_copy && slot == 0 && blockIdx.x == 0)) {
          for (int c = 0; c * BR < N; ++c) {
            if (axis == 1) tma_load_3d(dst + c * BR * 2 * L, &S.tile_map[slot], tx0, c * BR, to, &tile_bar[slot]);
            else tma_load_3d(dst + c * BR * 2 * L, &S.tile_map[slot], tx0, to, c * BR, &tile_bar[slot]);
          }
        }
      }
      return;
    } else if (CONTIG) {
      constexpr int CH = 2 * L * N / 4, PER = (CH + THREADS - 1) / THREADS;  // rows contiguous in memory
      const int chunks = cnt * N / 4;
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int q = tid + k * THREADS;
        if (q < chunks) cp_async16(dst + 4 * q, fb + 4 * q, 16);
      }
    } else {
      constexpr int CPR = (2 * L) / 4;  // 16-byte chunks per tile row (strided tiles have L >= 2)
      static_assert(THREADS % CPR == 0 && (CPR * N) % THREADS == 0, "strided staging");
      constexpr int RSTEP = THREADS / CPR, PER = CPR * N / THREADS;
      const int ch = tid % CPR, i0 = tid / CPR;
      const int valid = min(4, cnt - 4 * ch);
      const int bytes = valid > 0 ? 4 * valid : 0;
      float *d0 = dst + i0 * 2 * L + 4 * ch;
      const float *s0 = fb + i0 * st32 + 4 * ch;
      const int sstep = RSTEP * st32;
#pragma unroll
      for (int k = 0; k < PER; ++k) cp_async16(d0 + k * RSTEP * 2 * L, s0 + k * sstep, bytes);
    }
    cp_async_commit();
  };
  // Contiguous tiles: wait (bounded) for the bulk copies of the given slots, uniformly over the
  // CTA.  On a timeout the error word is set and the tile is abandoned: the remaining waits drain
  // any copy still in flight before the CTA exits.
  bool issued[4] = {false, false, false, false};
  auto tile_wait = [&](int s0, int s1) -> bool {
    if (!tma) {  // 16-byte cp.async staging: the p tile alone first, then everything
      if (s0 == 0 && s1 < 0) cp_async_wait<1>();
      else cp_async_wait<0>();
      __syncthreads();
      return true;
    }
    bool ok = true;
    if (s0 >= 0) ok = mbar_wait_bounded(&tile_bar[s0], 0) && ok;
    if (s1 >= 0) ok = mbar_wait_bounded(&tile_bar[s1], 0) && ok;
    ok = __syncthreads_and(ok);
    if (!ok) {
      if (tid == 0) atomicOr(S.err, 1);
      for (int b = 0; b < 4; ++b)
        if (issued[b]) mbar_wait_bounded(&tile_bar[b], 0);
    }
    return ok;
  };
  auto staged = [&](const float *st, int i) -> float2 {
    if (CONTIG) return make_float2(va ? st[(2 * l) * N + i] : 0.f, vb ? st[(2 * l + 1) * N + i] : 0.f);
    return *reinterpret_cast<const float2 *>(st + i * 2 * L + 2 * l);
  };
  const float *__restrict__ rho0 = S.rho0;
  stage(st_p, S.p, 0);
  issued[0] = true;
  if (rho0) {
    stage(st_r, rho0, 1);
    issued[1] = true;
  } else if (!tma) {
    cp_async_commit();
  }
  float2 *xs = sm + l * LP;
  float *__restrict__ ud = S.u[axis];
  // the p tile has landed (rho0 may still be in flight), for every thread; tables too
  if (!tile_wait(0, -1)) return;
  float2 v[E];
#pragma unroll
  for (int r = 0; r < E; ++r) v[r] = staged(st_p, tt + G * r);
  // time steps: the velocity tile takes the p tile's slot while d/dx_d p is transformed
  // (INIT keeps p staged: it is read again below)
  if (mode == KWB_MODE_STEP) {
    __syncthreads();  // every thread has its p values
    stage(st_p, ud, 2);
    issued[2] = true;
  }

  // d/dx_d p  (staggered +)
  F::fwd(v, xs, tw2, tt);
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = cmul(v[q], gp2[q * RP + tt]);
  F::inv(v, xs, tw2, tt);
  // the rho0 and velocity tiles have landed
  if (!tile_wait(rho0 ? 1 : -1, mode == KWB_MODE_STEP ? 2 : -1)) return;

  // velocity update u = pml_sg (pml_sg u - dt/rho_sg dp)
  const float *__restrict__ esg = S.pml_sg_def[axis];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int i = tt + G * r;
    const int inext = (r == E - 1 && tt == G - 1) ? 0 : i + 1;  // periodic neighbour
    float2 coef;
    if (rho0) {
      const float2 r0 = staged(st_r, i), r1 = staged(st_r, inext);
      coef = make_float2(__fdividef(2.0f * S.dt, r0.x + r1.x), __fdividef(2.0f * S.dt, r0.y + r1.y));
    } else {
      coef = make_float2(S.dt_over_rho0_s, S.dt_over_rho0_s);
    }
    float2 nv;
    if (mode == KWB_MODE_INIT) {
      nv = make_float2(-0.5f * coef.x * v[r].x, -0.5f * coef.y * v[r].y);
    } else {
      const float2 nes = pair(-__ldg(esg + i));
      const float2 u0 = staged(st_p, i);
      const float2 tu = pfma(make_float2(-coef.x, -coef.y), v[r], pfma(nes, u0, u0));
      nv = pfma(nes, tu, tu);
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
      const float2 pp = staged(st_p, i);
      float2 cs = S.c0sq ? load_pair(S.c0sq, i) : make_float2(S.c0sq_s, S.c0sq_s);
      store_pair(rd, i, make_float2(pp.x / ((float)S.D * cs.x), pp.y / ((float)S.D * cs.y)));
    }
    (void)invD;
    return;
  }

  // the split density rho_d takes the slot while d/dx_d u is transformed
  __syncthreads();  // every thread is done with the velocity tile
  stage(st_p, S.rho[axis], 3);
  issued[3] = true;
  if constexpr (XEOS) {
    // the equation-of-state operands of this tile (rho_y, rho_z, the B/A term, c^2) are read
    // after the density update; each is one contiguous block, prefetched into L2 now so that
    // those loads hit L2 instead of waiting on HBM
    if (S.eos_prefetch && tid == 0) {
      const unsigned bytes = (unsigned)cnt * N * 4u;
      const float *ops[4] = {S.D > 1 ? S.rho[1] : nullptr, S.D > 2 ? S.rho[2] : nullptr,
                             S.nonlinear ? S.nlq : nullptr, S.c0sq};
#pragma unroll
      for (int f = 0; f < 4; ++f)
        if (ops[f]) bulk_prefetch_l2(ops[f] + base, bytes);
    }
  }

  // velocity sources on this tile's lines (first_order_steps.jl:586-617, 646-690)
  // (entries are sorted by line: a thread scans only its own two lines)
  if (S.u_sig[axis] && S.u_line_ptr[axis] && va) {
    const int tcol = (int)(min(t + 1, (long long)S.u_cols[axis]) - 1);
    const int la = first_line + 2 * l;
    const int q0 = S.u_line_ptr[axis][la], q1 = S.u_line_ptr[axis][la + (vb ? 2 : 1)];
    for (int q = q0; q < q1; ++q) {
      const SrcEntry se = S.u_entry[axis][q];
      const int c = se.line - la;
      if ((se.pos % G) != tt) continue;
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
#pragma unroll
  for (int r = 0; r < E; ++r) store_pair(ud, tt + G * r, v[r]);

  // d/dx_d u_d  (staggered -)
  F::fwd(v, xs, tw2, tt);
#pragma unroll
  for (int q = 0; q < E; ++q) v[q] = cmul(v[q], gn2[q * RP + tt]);
  F::inv(v, xs, tw2, tt);

  if (!tile_wait(3, -1)) return;  // the rho_d tile has landed
  // density update rho_d = pml (pml rho_d - dt rho0 du)
  const float *__restrict__ ed = S.pml_def[axis];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int i = tt + G * r;
    const float2 nei = pair(-__ldg(ed + i));
    const float2 ncoef = rho0 ? pmul(pair(-S.dt), staged(st_r, i)) : pair(-S.dt_rho0_s);
    const float2 r0d = staged(st_p, i);
    float2 du = v[r];
    if (!CONTIG && axis == 1 && S.inv_r) {  // + u_r / r, the axisymmetric radial term (axisymmetric.jl:183)
      // u_r as stored above by this thread: an ordinary (coherent) load, not the read-only path
      const float2 ur = vb ? *reinterpret_cast<const float2 *>(ud + base + off(2 * l, i)) : make_float2(0.f, 0.f);
      du = pfma(ur, pair(__ldg(S.inv_r + i)), du);
    }
    const float2 tr = pfma(ncoef, du, pfma(nei, r0d, r0d));
    v[r] = pfma(nei, tr, tr);
  }
  // pressure (mass) sources (first_order_steps.jl:619-640, 692-715)
  if (S.n_p > 0 && S.p_line_ptr[axis] && va) {
    const int tcol = (int)(min(t + 1, (long long)S.p_cols) - 1);
    const int la = first_line + 2 * l;
    const int q0 = S.p_line_ptr[axis][la], q1 = S.p_line_ptr[axis][la + (vb ? 2 : 1)];
    for (int q = q0; q < q1; ++q) {
      const SrcEntry se = S.p_entry[axis][q];
      const int c = se.line - la;
      if ((se.pos % G) != tt) continue;
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
  if constexpr (XEOS) {
    // equation of state, x R2C (k_eos_fwd_fast): sum of the split densities, nonlinearity, c^2
#pragma unroll
    for (int r = 0; r < E; ++r) v[r] = make_float2(va ? v[r].x : 0.f, vb ? v[r].y : 0.f);
    if (S.D > 1) {
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const float2 b = load_pair(S.rho[1], tt + G * r);
        v[r] = padd(v[r], b);
      }
    }
    if (S.D > 2) {
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const float2 b = load_pair(S.rho[2], tt + G * r);
        v[r] = padd(v[r], b);
      }
    }
    if (S.nonlinear) {
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const float2 q = S.nlq ? load_pair(S.nlq, tt + G * r) : make_float2(S.nlq_s, S.nlq_s);
        v[r] = pmul(v[r], pfma(q, v[r], pair(1.0f)));
      }
    }
    if (S.c0sq) {
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const float2 c = load_pair(S.c0sq, tt + G * r);
        v[r] = pmul(c, v[r]);
      }
    }
    F::fwd(v, xs, tw2, tt);
#pragma unroll
    for (int idx = 0; idx < E; ++idx) xs[F::nat_of(tt, idx)] = v[idx];
    {
      const int n1 = S.n1, Ny = S.N[1];
      const int rows = 2 * L, tpp = (Ny + rows - 1) / rows;
      const int z = blockIdx.x / tpp, y0 = (blockIdx.x - z * tpp) * rows;
      if (S.plane) {
        __syncthreads();
        const int lp = tid % L;
        const float2 *xl = sm + lp * LP;
        float2 *dst = S.spec + ((long long)z * n1 + tid / L) * Ny + y0 + 2 * lp;
        const long long kstep = (long long)G * Ny;  // THREADS / L = G values of kx per sweep
        for (int k = tid / L; k < n1 && 2 * lp < cnt; k += G, dst += kstep) {
          const float2 zz = xl[F::nat(k)], zm = xl[F::nat(k == 0 ? 0 : N - k)];
          const float2 A = make_float2(0.5f * (zz.x + zm.x), 0.5f * (zz.y - zm.y));
          const float2 B = make_float2(0.5f * (zz.y + zm.y), -0.5f * (zz.x - zm.x));
          if (2 * lp + 1 < cnt) *reinterpret_cast<float4 *>(dst) = make_float4(A.x, A.y, B.x, B.y);
          else *dst = A;
        }
      } else {
        F::sync();
        const long long rowa = (long long)z * Ny + y0 + 2 * l;
        for (int k = tt; k < n1; k += G) {
          const float2 zz = xs[F::nat(k)];
          const float2 zm = xs[F::nat(k == 0 ? 0 : N - k)];
          if (va) S.spec[rowa * n1 + k] = make_float2(0.5f * (zz.x + zm.x), 0.5f * (zz.y - zm.y));
          if (vb) S.spec[(rowa + 1) * n1 + k] = make_float2(0.5f * (zz.y + zm.y), -0.5f * (zz.x - zm.x));
        }
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// equation of state: x R2C, y/z C2C with the multiply innermost, x C2R
// ------------------------------------------------------------------------------------------

// PLANE: write the half spectrum as [z][kx][y] (rows of y for the cluster y-z pass), instead of
// [z][y][kx].
template <class F, int LT, int MINB, bool PLANE>
__global__ void __launch_bounds__(LT * F::G, MINB)
    k_eos_fwd_fast(const __grid_constant__ SimDev S, long long step_s) {
  constexpr int E = F::E, G = F::G;
  constexpr int LP = F::LP, N = E * G, L = LT;
  extern __shared__ __align__(128) float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  // the twiddles are written once at set-up: built before waiting on the previous kernel
  F::build_tw(tw2, S.tw[0]);
  KWB_STEP_KERNEL_PROLOGUE();
  const long long t = *S.t0 + step_s;
  if (t >= S.Nt) return;
  const int tid = threadIdx.x, tt = tid % G, l = tid / G;
  const int Ny = S.N[1];
  const int rows = 2 * L, tpp = (Ny + rows - 1) / rows;
  const int z = blockIdx.x / tpp, y0 = (blockIdx.x - z * tpp) * rows;
  const int cnt = min(rows, Ny - y0);
  const long long base = ((long long)z * Ny + y0) * N;
  const bool va = 2 * l < cnt, vb = 2 * l + 1 < cnt;
  // One field at a time over all E positions: each loop issues 2E independent loads, so
  // every thread keeps many requests in flight (the sum, nonlinearity and c^2 follow).
  auto ld = [&](const float *__restrict__ f, int i) -> float2 {
    const float *fb = f + base + (long long)(2 * l) * N + i;
    return make_float2(va ? __ldg(fb) : 0.f, vb ? __ldg(fb + N) : 0.f);
  };
  float2 v[E];
#pragma unroll
  for (int r = 0; r < E; ++r) v[r] = ld(S.rho[0], tt + G * r);
  if (S.D > 1) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const float2 b = ld(S.rho[1], tt + G * r);
      v[r] = padd(v[r], b);
    }
  }
  if (S.D > 2) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const float2 b = ld(S.rho[2], tt + G * r);
      v[r] = padd(v[r], b);
    }
  }
  if (S.nonlinear) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const float2 q = S.nlq ? ld(S.nlq, tt + G * r) : make_float2(S.nlq_s, S.nlq_s);
      v[r] = pmul(v[r], pfma(q, v[r], pair(1.0f)));
    }
  }
  if (S.c0sq) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const float2 c = ld(S.c0sq, tt + G * r);
      v[r] = pmul(c, v[r]);
    }
  }
  __syncthreads();
  float2 *xs = sm + l * LP;
  F::fwd(v, xs, tw2, tt);
#pragma unroll
  for (int idx = 0; idx < E; ++idx) xs[F::nat_of(tt, idx)] = v[idx];
  const int n1 = S.n1;
  if (PLANE) {
    // one (kx, line pair) per thread, pairs fastest: the pair's two rows are adjacent in y, so
    // each thread writes A and B as one 16-byte store and each kx gets 2L consecutive y
    __syncthreads();
    const int lp = tid % L;
    const float2 *xl = sm + lp * LP;
    float2 *dst = S.spec + ((long long)z * n1 + tid / L) * Ny + y0 + 2 * lp;
    const long long kstep = (long long)G * Ny;  // THREADS / L = G values of kx per sweep
    for (int k = tid / L; k < n1 && 2 * lp < cnt; k += G, dst += kstep) {
      const float2 zz = xl[F::nat(k)], zm = xl[F::nat(k == 0 ? 0 : N - k)];
      const float2 A = make_float2(0.5f * (zz.x + zm.x), 0.5f * (zz.y - zm.y));
      const float2 B = make_float2(0.5f * (zz.y + zm.y), -0.5f * (zz.x - zm.x));
      if (2 * lp + 1 < cnt) *reinterpret_cast<float4 *>(dst) = make_float4(A.x, A.y, B.x, B.y);
      else *dst = A;
    }
    return;
  }
  F::sync();
  const long long rowa = (long long)z * Ny + y0 + 2 * l;
  for (int k = tt; k < n1; k += G) {
    const float2 zz = xs[F::nat(k)];
    const float2 zm = xs[F::nat(k == 0 ? 0 : N - k)];
    if (va) S.spec[rowa * n1 + k] = make_float2(0.5f * (zz.x + zm.x), 0.5f * (zz.y - zm.y));
    if (vb) S.spec[(rowa + 1) * n1 + k] = make_float2(0.5f * (zz.y + zm.y), -0.5f * (zz.x - zm.x));
  }
}

template <class F, int LT, int MINB, bool PLANE>
__global__ void __launch_bounds__(LT * F::G, MINB)
    k_eos_inv_fast(const __grid_constant__ SimDev S, long long step_s) {
  constexpr int E = F::E, G = F::G;
  constexpr int LP = F::LP, N = E * G, L = LT;
  extern __shared__ __align__(128) float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  // the twiddles are written once at set-up: built before waiting on the previous kernel
  F::build_tw(tw2, S.tw[0]);
  KWB_STEP_KERNEL_PROLOGUE();
  const long long t = *S.t0 + step_s;
  if (t >= S.Nt) return;
  const int tid = threadIdx.x, tt = tid % G, l = tid / G;
  const int Ny = S.N[1];
  const int rows = 2 * L, tpp = (Ny + rows - 1) / rows;
  const int z = blockIdx.x / tpp, y0 = (blockIdx.x - z * tpp) * rows;
  const int cnt = min(rows, Ny - y0);
  const long long base = ((long long)z * Ny + y0) * N;
  const bool va = 2 * l < cnt, vb = 2 * l + 1 < cnt;
  float2 *xs = sm + l * LP;
  const int n1 = S.n1;
  if (PLANE) {
    // one (kx, line pair) per thread, pairs fastest: the pair's rows are adjacent in y, so A and
    // B arrive as one 16-byte load and each kx reads 2L consecutive y
    const int lp = tid % L;
    float2 *xl = sm + lp * LP;
    const float2 *srcp = S.spec + ((long long)z * n1 + tid / L) * Ny + y0 + 2 * lp;
    const long long kstep = (long long)G * Ny;  // THREADS / L = G values of kx per sweep
    for (int k = tid / L; k < n1; k += G, srcp += kstep) {
      float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
      if (2 * lp + 1 < cnt) {
        const float4 ab = *reinterpret_cast<const float4 *>(srcp);
        A = make_float2(ab.x, ab.y);
        B = make_float2(ab.z, ab.w);
      } else if (2 * lp < cnt) {
        A = *srcp;
      }
      if (k == 0 || 2 * k == N) {
        xl[F::nat(k)] = make_float2(A.x, B.x);  // c2r ignores Im of the DC and Nyquist bins
      } else {
        xl[F::nat(k)] = make_float2(A.x - B.y, A.y + B.x);
        xl[F::nat(N - k)] = make_float2(A.x + B.y, B.x - A.y);
      }
    }
  } else {
    const long long rowa = (long long)z * Ny + y0 + 2 * l;
    for (int k = tt; k < n1; k += G) {
      const float2 A = va ? S.spec[rowa * n1 + k] : make_float2(0.f, 0.f);
      const float2 B = vb ? S.spec[(rowa + 1) * n1 + k] : make_float2(0.f, 0.f);
      if (k == 0 || 2 * k == N) {
        xs[F::nat(k)] = make_float2(A.x, B.x);  // c2r ignores Im of the DC and Nyquist bins
      } else {
        xs[F::nat(k)] = make_float2(A.x - B.y, A.y + B.x);
        xs[F::nat(N - k)] = make_float2(A.x + B.y, B.x - A.y);
      }
    }
  }
  __syncthreads();
  float2 v[E];
#pragma unroll
  for (int idx = 0; idx < E; ++idx) v[idx] = xs[F::nat_of(tt, idx)];
  // dense pressure sensor (record_sensor_data!, first_order_steps.jl:732-752): prefetch the
  // running max (or, without one, the running min) before the transform, update all fields as p
  // is written.  One prefetched field keeps the kernel within its register budget.
  const GroupDev *gd = S.dense_p;
  const unsigned gm = gd ? gd->mask : 0u;
  constexpr bool PFS = E <= 16;  // prefetch only while it fits in registers
  float2 pm[PFS ? E : 1];
  const bool pf_max = PFS && (gm & (1u << 1)), pf_min = PFS && !pf_max && (gm & (1u << 2));
  const long long ra = base + (long long)(2 * l) * N, rb = ra + N;
  if (pf_max || pf_min) {
    const float *pa = pf_max ? gd->pmax : gd->pmin;
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int i = tt + G * r;
      pm[PFS ? r : 0] = make_float2(va ? pa[ra + i] : 0.f, vb ? pa[rb + i] : 0.f);
    }
  }
  F::sync();
  F::inv(v, xs, tw2, tt);
  // p and the dense sensor fields: one pass per field over this thread's two rows (ra, ra + N)
  auto put = [&](float *a) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if (va) a[tt + G * r] = v[r].x;
      if (vb) a[N + tt + G * r] = v[r].y;
    }
  };
  put(S.p + ra);
  if (gm) {
    if (gm & (1u << 0)) put(gd->ser_p + t * gd->n + ra);
    if (gm & (1u << 1)) {
      float *a = gd->pmax + ra;
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const int i = tt + G * r;
        if (va) a[i] = fmaxf(pf_max ? pm[PFS ? r : 0].x : a[i], v[r].x);
        if (vb) a[N + i] = fmaxf(pf_max ? pm[PFS ? r : 0].y : a[N + i], v[r].y);
      }
    }
    if (gm & (1u << 2)) {
      float *a = gd->pmin + ra;
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const int i = tt + G * r;
        if (va) a[i] = fminf(pf_min ? pm[PFS ? r : 0].x : a[i], v[r].x);
        if (vb) a[N + i] = fminf(pf_min ? pm[PFS ? r : 0].y : a[N + i], v[r].y);
      }
    }
    if (gm & (1u << 3)) {
      double *a = gd->prms + ra;
      const double w = (double)gd->cnt_prms;
#pragma unroll
      for (int r = 0; r < E; ++r) {
        const int i = tt + G * r;
        if (va) a[i] += w * ((double)v[r].x * (double)v[r].x);
        if (vb) a[N + i] += w * ((double)v[r].y * (double)v[r].y);
      }
    }
    if ((gm & (1u << 4)) && t == S.Nt - 1) put(gd->pfinal + ra);
  }
  // sparse pressure sensor (record_sensor_data!, first_order_steps.jl:732-752): this thread's
  // p values go to its line's exchange buffer (x order, the two rows as one pair), then the
  // points on the line pair are recorded from there through the group's per-x-line index
  const GroupDev *gs = S.sparse_p;
  if (gs) {
    const int line0 = z * Ny + y0 + 2 * l;
    const int qa = va ? gs->line_ptr[line0] : 0;
    const int qb = va ? gs->line_ptr[line0 + 1] : 0;
    const int qc = vb ? gs->line_ptr[line0 + 2] : qb;
    // most lines hold no point: skip the exchange unless some line of the group (the warp for
    // one-warp lines, else the block) does
    bool any = qc > qa;
    if (F::WARP_SYNC) any = __any_sync(0xffffffffu, any);
    else any = __syncthreads_or(any);
    if (!any) return;
#pragma unroll
    for (int r = 0; r < E; ++r) xs[tt + G * r] = v[r];
    F::sync();
    const unsigned sm_ = gs->mask;
    const bool last = (t == S.Nt - 1);
    for (int c = 0; c < 2; ++c) {
      if (!(c ? vb : va)) continue;
      const int q0 = c ? qb : qa, q1 = c ? qc : qb;
      for (int q = q0 + tt; q < q1; q += G) {
        const int2 e = gs->line_ent[q];
        const float2 pp = xs[e.x];
        const float pv = c ? pp.y : pp.x;
        const long long j = e.y;
        if (sm_ & (1u << 0)) gs->ser_p[t * gs->n + j] = pv;
        if (sm_ & (1u << 1)) gs->pmax[j] = fmaxf(gs->pmax[j], pv);
        if (sm_ & (1u << 2)) gs->pmin[j] = fminf(gs->pmin[j], pv);
        if (sm_ & (1u << 3)) gs->prms[j] += (double)gs->cnt_prms * ((double)pv * (double)pv);
        if ((sm_ & (1u << 4)) && last) gs->pfinal[j] = pv;
      }
    }
  }
}

template <class F, int LT, int MINB>
__global__ void __launch_bounds__(LT * F::G, MINB)
    k_spec_fast(const __grid_constant__ SimDev S, int axis, int op, long long step_s) {
  constexpr int E = F::E, G = F::G;
  constexpr int LP = F::LP, L = LT;
  extern __shared__ __align__(128) float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  // the twiddles are written once at set-up: built before waiting on the previous kernel
  F::build_tw(tw2, S.tw[axis]);
  KWB_STEP_KERNEL_PROLOGUE();
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
// y and z transforms of the equation of state, one kx plane per thread-block cluster
// ------------------------------------------------------------------------------------------

#define KWB_PLANE_THREADS 512

// Distributed shared memory: 32-bit shared::cluster addresses of the same offset in another CTA.
__device__ __forceinline__ unsigned cta_smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned cluster_map(unsigned addr, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ float2 cluster_ld(unsigned addr) {
  float2 v;
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ void cluster_st(unsigned addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};\n" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}

// Plane pass: the spectrum is [z][kx][y] (k_eos_fwd_fast<PLANE>), so plane kx is NZ rows of NY
// contiguous values.  The CL CTAs of a cluster share plane kx: CTA r holds z rows
// [r RZ, (r+1) RZ) in shared memory and
//   1. transforms its rows along y (contiguous lines, one warp per line) and keeps each row in
//      register order: slot s = t + G idx holds k_y = FY::k_of(t, idx);
//   2. after a cluster barrier, transforms along z the slots [r CY, (r+1) CY) of every row of
//      the plane (lines spread over the warps as in the strided line passes, so that a warp's
//      loads cover consecutive slots of one row), loading element z of a slot from the CTA that
//      holds row z (distributed shared memory), multiplies by M[kx][k_z][slot] and transforms
//      back, storing each element to the CTA it came from;
//   3. after a second barrier, transforms its rows back along y and writes them to the plane.
// The spectrum crosses HBM once in and once out per step, with the multiplier read once.
// The cluster shape is set at launch (CL CTAs of THREADS threads: 8 x 512, or 16 x 256 with half
// the rows per CTA so that four CTAs fit an SM); element z of a z line sits in row z % RZ of
// cluster CTA z / RZ.
template <class FY, class FZ, int CL, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_plane_fast(const __grid_constant__ SimDev S, long long step_s) {
  constexpr int NY = FY::N, NZ = FZ::N, RZ = NZ / CL, CY = NY / CL;
  constexpr int LY = THREADS / FY::G, LZ = THREADS / FZ::G;
  static_assert(RZ == 2 * LY && CY % LZ == 0 && NZ % RZ == 0, "plane tiling");
  constexpr int XS = (LY * FY::LP > LZ * FZ::LP) ? LY * FY::LP : LZ * FZ::LP;
  extern __shared__ __align__(128) float4 smem_raw[];
  float2 *data = reinterpret_cast<float2 *>(smem_raw);  // [RZ][NY]
  float2 *xsb = data + RZ * NY;
  float2 *twy = xsb + XS;
  float2 *twz = twy + FY::TW;
  // the twiddles are written once at set-up: built before waiting on the previous kernel
  FY::build_tw(twy, S.tw[1]);
  FZ::build_tw(twz, S.tw[2]);
  KWB_STEP_KERNEL_PROLOGUE();
  const long long t = *S.t0 + step_s;
  if (t >= S.Nt) return;  // uniform over the cluster
  const unsigned rank = cluster_rank();
  const int kx = blockIdx.x / CL;
  const int tid = threadIdx.x;
  // the multiplier of plane kx is read in the z phase; each CTA prefetches its slice of it (rows
  // k_z in [rank RZ, (rank+1) RZ), contiguous) into L2 now, so that the cluster holds all of it
  if (S.eos_prefetch && tid == 0)
    bulk_prefetch_l2(S.M + ((long long)kx * NZ + (long long)rank * RZ) * NY, (unsigned)(RZ * NY * 4));
  const long long rstride = (long long)S.n1 * NY;  // between consecutive z rows of the plane
  float2 *plane = S.spec + (long long)rank * RZ * rstride + (long long)kx * NY;
  // rows in two groups, so that the first transforms start while the second group lands
  constexpr int CPR = NY / 2;  // 16-byte chunks per row
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    for (int q = tid; q < LY * CPR; q += THREADS) {
      const int r = g * LY + q / CPR, c = q % CPR;
      cp_async16(data + r * NY + 2 * c, plane + r * rstride + 2 * c, 16);
    }
    cp_async_commit();
  }

  // 1. forward along y
  {
    const int tt = tid % FY::G, l = tid / FY::G;
    float2 *xs = xsb + l * FY::LP;
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      if (g == 0) cp_async_wait<1>();
      else cp_async_wait<0>();
      __syncthreads();
      float2 *row = data + (g * LY + l) * NY;
      float2 v[FY::E];
#pragma unroll
      for (int r = 0; r < FY::E; ++r) v[r] = row[tt + FY::G * r];
      FY::fwd(v, xs, twy, tt);
#pragma unroll
      for (int idx = 0; idx < FY::E; ++idx) row[tt + FY::G * idx] = v[idx];
    }
  }
  cluster_barrier();

  // 2. along z, multiply, back along z
  {
    const int l = tid % LZ, tt = tid / LZ;
    float2 *xs = xsb + l * FZ::LP;
    const float *__restrict__ Mp = S.M + (long long)kx * NZ * NY;
#pragma unroll 1
    for (int c0 = 0; c0 < CY; c0 += LZ) {
      const int sl = (int)rank * CY + c0 + l;  // slot (register-order k_y) of this line
      // element z = tt + G r is row z % RZ of CTA z / RZ
      float2 v[FZ::E];
#pragma unroll
      for (int r = 0; r < FZ::E; ++r) {
        const int z = tt + FZ::G * r;
        v[r] = cluster_ld(cluster_map(cta_smem_addr(data + (z % RZ) * NY + sl), (unsigned)(z / RZ)));
      }
      FZ::fwd(v, xs, twz, tt);
      // the multiplier is loaded after the transform: held across it, it spilled
#pragma unroll
      for (int idx = 0; idx < FZ::E; ++idx) {
        const float m = __ldg(Mp + (long long)FZ::k_of(tt, idx) * NY + sl);
        v[idx] = make_float2(v[idx].x * m, v[idx].y * m);
      }
      FZ::inv(v, xs, twz, tt);
#pragma unroll
      for (int r = 0; r < FZ::E; ++r) {
        const int z = tt + FZ::G * r;
        cluster_st(cluster_map(cta_smem_addr(data + (z % RZ) * NY + sl), (unsigned)(z / RZ)), v[r]);
      }
    }
  }
  cluster_barrier();

  // 3. back along y, straight to the plane
  {
    const int tt = tid % FY::G, l = tid / FY::G;
    float2 *xs = xsb + l * FY::LP;
#pragma unroll 1
    for (int g = 0; g < 2; ++g) {
      const float2 *row = data + (g * LY + l) * NY;
      float2 v[FY::E];
#pragma unroll
      for (int idx = 0; idx < FY::E; ++idx) v[idx] = row[tt + FY::G * idx];
      FY::inv(v, xs, twy, tt);
      float2 *out = plane + (g * LY + l) * rstride;
#pragma unroll
      for (int r = 0; r < FY::E; ++r) out[tt + FY::G * r] = v[r];
    }
  }
}

// Plane pass with slot-major rows: the same three steps and the same arithmetic as k_plane_fast,
// with one warp per line throughout and no block-wide barriers.  After its y transforms a CTA
// stores its rows slot-major, cols[slot][z row] with an odd pitch RZ + 1, so the part of the z
// line of one slot that a cluster CTA holds is RZ consecutive values: the warp that owns the line
// gathers it with contiguous distributed-shared-memory reads (lane t takes z = t + 32 r from CTA
// z / RZ, row z % RZ), transforms it, multiplies, transforms back and scatters it to the same
// places.  Each slot column of a CTA is touched by exactly one warp of the cluster between the
// two cluster barriers, so nothing else orders the z step.  Rows are read from and written to
// the plane directly (lane t holds x[t + 32 r]: coalesced 256-byte row segments).  The multiplier
// is laid out [kx][slot][j] with k_z = F::k_of(j % 32, j / 32), so a line's 256 values are
// contiguous (the table builder writes that layout when this variant runs).
template <class F, int CL, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_plane_cols(const __grid_constant__ SimDev S, long long step_s) {
  constexpr int NY = F::N, NZ = F::N, RZ = NZ / CL, CY = NY / CL, W = THREADS / 32;
  constexpr int RP = RZ + 1;  // pitch of a slot column (odd: conflict-free row stores)
  static_assert(F::G == 32 && F::WARP_SYNC, "one warp per line");
  static_assert(RZ % W == 0 && CY % W == 0 && NZ % RZ == 0, "plane tiling");
  extern __shared__ __align__(128) float4 smem_raw[];
  float2 *cols = reinterpret_cast<float2 *>(smem_raw);  // [NY][RP]
  float2 *xsb = cols + NY * RP;                          // one exchange buffer per warp
  float2 *twy = xsb + W * F::LP;
  float2 *twz = twy + F::TW;
  F::build_tw(twy, S.tw[1]);
  F::build_tw(twz, S.tw[2]);
  KWB_STEP_KERNEL_PROLOGUE();
  const long long t = *S.t0 + step_s;
  if (t >= S.Nt) return;  // uniform over the cluster
  const unsigned rank = cluster_rank();
  const int kx = blockIdx.x / CL;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float2 *xs = xsb + w * F::LP;
  const float *__restrict__ Mk = S.M + (long long)kx * NY * NZ;
  if (S.eos_prefetch && threadIdx.x == 0) bulk_prefetch_l2(Mk + (long long)rank * CY * NZ, (unsigned)(CY * NZ * 4));
  const long long rstride = (long long)S.n1 * NY;  // between consecutive z rows of the plane
  float2 *plane = S.spec + (long long)rank * RZ * rstride + (long long)kx * NY;
  __syncthreads();  // twiddles

  // 1. forward along y, rows to slot-major columns
#pragma unroll 1
  for (int zl = w; zl < RZ; zl += W) {
    const float2 *row = plane + zl * rstride;
    float2 v[F::E];
#pragma unroll
    for (int r = 0; r < F::E; ++r) v[r] = row[lane + 32 * r];
    F::fwd(v, xs, twy, lane);
#pragma unroll
    for (int idx = 0; idx < F::E; ++idx) cols[(lane + 32 * idx) * RP + zl] = v[idx];
  }
  cluster_barrier();

  // 2. the z lines of this CTA's slots: gather, forward, multiply, back, scatter
  const unsigned cbase = cta_smem_addr(cols);
#pragma unroll 1
  for (int c = w; c < CY; c += W) {
    const int sl = (int)rank * CY + c;
    float2 v[F::E];
#pragma unroll
    for (int r = 0; r < F::E; ++r) {
      const int z = lane + 32 * r;
      v[r] = cluster_ld(cluster_map(cbase + (unsigned)((sl * RP + z % RZ) * 8), (unsigned)(z / RZ)));
    }
    F::fwd(v, xs, twz, lane);
    const float *m = Mk + (long long)sl * NZ + lane;
#pragma unroll
    for (int idx = 0; idx < F::E; ++idx) {
      const float mm = __ldg(m + 32 * idx);
      v[idx] = make_float2(v[idx].x * mm, v[idx].y * mm);
    }
    F::inv(v, xs, twz, lane);
#pragma unroll
    for (int r = 0; r < F::E; ++r) {
      const int z = lane + 32 * r;
      cluster_st(cluster_map(cbase + (unsigned)((sl * RP + z % RZ) * 8), (unsigned)(z / RZ)), v[r]);
    }
  }
  cluster_barrier();

  // 3. back along y, straight to the plane
#pragma unroll 1
  for (int zl = w; zl < RZ; zl += W) {
    float2 v[F::E];
#pragma unroll
    for (int idx = 0; idx < F::E; ++idx) v[idx] = cols[(lane + 32 * idx) * RP + zl];
    F::inv(v, xs, twy, lane);
    float2 *out = plane + zl * rstride;
#pragma unroll
    for (int r = 0; r < F::E; ++r) out[lane + 32 * r] = v[r];
  }
}


// ------------------------------------------------------------------------------------------
// dispatch
// ------------------------------------------------------------------------------------------

static inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

static inline cudaError_t raise_smem(const void *fn, size_t bytes) { return raise_dynamic_smem(fn, bytes); }

// Two compile-time tile sizes per line length: full tiles of 256/G complex lines for large
// grids, and small tiles (one warp, >= 2 lines) when full tiles would leave SMs idle.
template <int G>
struct Tiles {
  static constexpr int BIG = KWB_THREADS / G;
  static constexpr int SMALL = (32 / G > 2 ? 32 / G : 2);
};

static inline bool want_small(const SimDev &h, long long tiles_big) {
  return tiles_big < 2LL * (h.num_sms > 0 ? h.num_sms : 148);
}

// Tile variant per pass: 0 = big (THREADS per CTA), 1 = mid (128 threads), 2 = small (one warp).
static inline int tile_variant(const SimDev &h, int slot, long long tiles_big) {
  if (h.tile_override >= 0) return h.tile_override;
  if (slot >= 0 && h.tile_var[slot] >= 0) return h.tile_var[slot];
  return want_small(h, tiles_big) ? 2 : 0;
}

// Line-pass configurations: FFT policy, threads per CTA and CTAs per SM to target.  The
// three-level policy (8 registers-worth of elements per thread) is used for 128..1024, the
// two-level one for 64.
template <int N>
struct LinePolicy;
template <>
struct LinePolicy<64> {
  template <bool C> using F = LineFFT<8, 8, C>;
  static constexpr int THREADS = 256, MINB = 2;
};
template <>
struct LinePolicy<128> {
  template <bool C> using F = LineFFT3<8, 2, 8, C>;
  static constexpr int THREADS = 512, MINB = 2;
};
template <>
struct LinePolicy<256> {
  template <bool C> using F = LineFFT3<8, 4, 8, C>;
  static constexpr int THREADS = 512, MINB = 2;
};
template <>
struct LinePolicy<512> {
  template <bool C> using F = LineFFT3<8, 8, 8, false>;  // 64 threads per line: block-level sync
  static constexpr int THREADS = 512, MINB = 2;
};
template <>
struct LinePolicy<1024> {
  template <bool C> using F = LineFFT3<16, 8, 8, false>;
  static constexpr int THREADS = 512, MINB = 1;
};

// Mixed-radix lengths (LineFFT3G): 12 or 20 registers' worth of elements per thread, 256
// threads per CTA so that two CTAs with their staged tiles fit an SM.
template <>
struct LinePolicy<96> {
  template <bool C> using F = LineFFT3G<12, 2, 4, C>;
  static constexpr int THREADS = 256, MINB = 2;
};
template <>
struct LinePolicy<160> {
  template <bool C> using F = LineFFT3G<20, 2, 4, C>;
  static constexpr int THREADS = 256, MINB = 2;
};
template <>
struct LinePolicy<192> {
  template <bool C> using F = LineFFT3G<12, 4, 4, C>;
  static constexpr int THREADS = 256, MINB = 2;
};
template <>
struct LinePolicy<320> {
  template <bool C> using F = LineFFT3G<20, 4, 4, C>;
  static constexpr int THREADS = 256, MINB = 2;
};

template <>
struct LinePolicy<80> {
  template <bool C> using F = LineFFT3G<20, 2, 2, C>;
  static constexpr int THREADS = 128, MINB = 2;
};
template <>
struct LinePolicy<640> {
  template <bool C> using F = LineFFT4G<20, 4, 4, 2, C>;
  static constexpr int THREADS = 256, MINB = 2;
};
// Threads per line not a power of two (block-level exchanges); THREADS keeps the full-width tile
// at an even number of lines.
template <>
struct LinePolicy<144> {
  template <bool C> using F = LineFFT3G<12, 3, 4, false>;
  static constexpr int THREADS = 192, MINB = 2;
};
template <>
struct LinePolicy<288> {
  template <bool C> using F = LineFFT3G<12, 4, 6, false>;
  static constexpr int THREADS = 192, MINB = 2;
};
template <>
struct LinePolicy<432> {
  template <bool C> using F = LineFFT3G<12, 6, 6, false>;
  static constexpr int THREADS = 288, MINB = 2;
};
template <>
struct LinePolicy<576> {
  template <bool C> using F = LineFFT3G<12, 4, 12, false>;
  static constexpr int THREADS = 192, MINB = 2;
};
template <>
struct LinePolicy<864> {
  template <bool C> using F = LineFFT3G<12, 6, 12, false>;
  static constexpr int THREADS = 288, MINB = 2;
};
template <>
struct LinePolicy<400> {
  template <bool C> using F = LineFFT3G<20, 4, 5, false>;
  static constexpr int THREADS = 160, MINB = 2;
};
template <>
struct LinePolicy<500> {
  template <bool C> using F = LineFFT3G<20, 5, 5, false>;
  static constexpr int THREADS = 200, MINB = 2;
};
template <>
struct LinePolicy<800> {
  template <bool C> using F = LineFFT3G<20, 4, 10, false>;
  static constexpr int THREADS = 160, MINB = 2;
};
template <>
struct LinePolicy<1000> {
  template <bool C> using F = LineFFT3G<20, 5, 10, false>;
  static constexpr int THREADS = 200, MINB = 2;
};
template <>
struct LinePolicy<384> {
  template <bool C> using F = LineFFT4G<12, 4, 4, 2, C>;
  static constexpr int THREADS = 256, MINB = 2;
};
template <>
struct LinePolicy<768> {
  template <bool C> using F = LineFFT4G<12, 4, 4, 4, false>;  // 64 threads per line: block-level sync
  static constexpr int THREADS = 256, MINB = 2;
};

// elastic gradient pass (defined below), primed with the line-pass variants of the same tiles
template <class F, bool CONTIG, int LT, int MINB>
__global__ void __launch_bounds__(LT * F::G, MINB)
    k_el_grad_fast(const __grid_constant__ SimDev S, int axis, const __grid_constant__ ElGrad g, long long step_s);

template <int N, bool C, int LT>
static inline cudaError_t prime_line_variant() {
  using P = LinePolicy<N>;
  using F = typename P::template F<C>;
  cudaError_t e = raise_smem((const void *)k_line_fast<F, C, LT, P::MINB, false>, pline_smem<F>(LT));
  if (e == cudaSuccess) e = raise_smem((const void *)k_el_grad_fast<F, C, LT, P::MINB>, pline_smem<F>(LT));
  if constexpr (C) {
    if (e == cudaSuccess) e = raise_smem((const void *)k_line_fast<F, C, LT, P::MINB, true>, pline_smem<F>(LT));
  } else {
    if (e == cudaSuccess) e = raise_smem((const void *)k_line_fast<F, C, LT, P::MINB, false, true>, pline_smem<F>(LT));
  }
  return e;
}

template <int N>
static inline cudaError_t prime_line() {
  using P = LinePolicy<N>;
  constexpr int G = P::template F<true>::G;
  constexpr int BIG = P::THREADS / G, SMALL = (32 / G > 2 ? 32 / G : 2);
  cudaError_t e;
  if ((e = prime_line_variant<N, true, BIG>()) != cudaSuccess) return e;
  if ((e = prime_line_variant<N, false, BIG>()) != cudaSuccess) return e;
  if ((e = prime_line_variant<N, true, SMALL>()) != cudaSuccess) return e;
  if ((e = prime_line_variant<N, false, SMALL>()) != cudaSuccess) return e;
  constexpr int MID = ((128 / G) & ~1) > SMALL ? ((128 / G) & ~1) : SMALL;  // even line counts
  if ((e = prime_line_variant<N, true, MID>()) != cudaSuccess) return e;
  return prime_line_variant<N, false, MID>();
}

template <int N, int LT>
static inline void line_go(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s, cudaStream_t st) {
  using P = LinePolicy<N>;
  if (axis == 0) {
    using F = typename P::template F<true>;
    const int grid = cdiv(h.N[1], 2 * LT) * h.N[2];
    if (h.fuse_xeos && mode == KWB_MODE_STEP)
      kwb_launch(k_line_fast<F, true, LT, P::MINB, true>, grid, LT * F::G, pline_smem<F>(LT), st, h, axis, mode, s);
    else
      kwb_launch(k_line_fast<F, true, LT, P::MINB, false>, grid, LT * F::G, pline_smem<F>(LT), st, h, axis, mode, s);
  } else {
    using F = typename P::template F<false>;
    const int grid = cdiv(h.N[0], 2 * LT) * (axis == 1 ? h.N[2] : h.N[1]);
    const bool want = (h.tma_line[axis] >= 0 ? h.tma_line[axis] : h.tile_tma) != 0;
    if (want && (2 * LT) % 4 == 0) {
      // strided tiles by tiled TMA: this launch's copy of the descriptor carries the fields'
      // tensor maps for its tile width (16-byte rows and offsets only)
      SimDev hs = h;
      if (encode_strided_maps(hs, axis, 2 * LT)) {
        hs.tile_tma_s = 1;
        kwb_launch(k_line_fast<F, false, LT, P::MINB, false, true>, grid, LT * F::G, pline_smem<F>(LT), st, hs, axis, mode, s);
        return;
      }
    }
    kwb_launch(k_line_fast<F, false, LT, P::MINB, false>, grid, LT * F::G, pline_smem<F>(LT), st, h, axis, mode, s);
  }
}

template <int N>
static inline cudaError_t launch_line_n(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                 cudaStream_t st) {
  using P = LinePolicy<N>;
  constexpr int G = P::template F<true>::G;
  constexpr int BIG = P::THREADS / G, SMALL = (32 / G > 2 ? 32 / G : 2);
  constexpr int MID = ((128 / G) & ~1) > SMALL ? ((128 / G) & ~1) : SMALL;  // even line counts
  const long long tiles = axis == 0 ? (long long)cdiv(h.N[1], 2 * BIG) * h.N[2]
                                    : (long long)cdiv(h.N[0], 2 * BIG) * (axis == 1 ? h.N[2] : h.N[1]);
  switch (tile_variant(h, KWB_SLOT_LINE0 + axis, tiles)) {
    case 1: line_go<N, MID>(d_sim, h, axis, mode, s, st); break;
    case 2: line_go<N, SMALL>(d_sim, h, axis, mode, s, st); break;
    default: line_go<N, BIG>(d_sim, h, axis, mode, s, st); break;
  }
  return cudaGetLastError();
}

template <class F>
__host__ __device__ constexpr size_t eos_smem(int L) {
  return ((size_t)L * F::LP + F::TW) * sizeof(float2);
}

template <int N, int LT>
static inline cudaError_t prime_eos_variant() {
  using P = LinePolicy<N>;
  using FC = typename P::template F<true>;
  using FS = typename P::template F<false>;
  cudaError_t e;
  if ((e = raise_smem((const void *)k_eos_fwd_fast<FC, LT, P::MINB, false>, eos_smem<FC>(LT))) != cudaSuccess) return e;
  if ((e = raise_smem((const void *)k_eos_inv_fast<FC, LT, P::MINB, false>, eos_smem<FC>(LT))) != cudaSuccess) return e;
  if ((e = raise_smem((const void *)k_eos_fwd_fast<FC, LT, P::MINB, true>, eos_smem<FC>(LT))) != cudaSuccess) return e;
  if ((e = raise_smem((const void *)k_eos_inv_fast<FC, LT, P::MINB, true>, eos_smem<FC>(LT))) != cudaSuccess) return e;
  return raise_smem((const void *)k_spec_fast<FS, LT, P::MINB>, eos_smem<FS>(LT));
}

template <int N>
static inline cudaError_t prime_eos_n() {
  using P = LinePolicy<N>;
  constexpr int G = P::template F<true>::G;
  constexpr int BIG = P::THREADS / G, SMALL = (32 / G > 2 ? 32 / G : 2);
  constexpr int MID = ((128 / G) & ~1) > SMALL ? ((128 / G) & ~1) : SMALL;  // even line counts
  cudaError_t e = prime_eos_variant<N, BIG>();
  if (e == cudaSuccess) e = prime_eos_variant<N, MID>();
  return e != cudaSuccess ? e : prime_eos_variant<N, SMALL>();
}

template <int N, int LT>
static inline void eos_go(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  using P = LinePolicy<N>;
  using F = typename P::template F<true>;
  const int grid = cdiv(h.N[1], 2 * LT) * h.N[2];
  if (h.plane) {
    if (fwd) kwb_launch(k_eos_fwd_fast<F, LT, P::MINB, true>, grid, LT * F::G, eos_smem<F>(LT), st, h, s);
    else kwb_launch(k_eos_inv_fast<F, LT, P::MINB, true>, grid, LT * F::G, eos_smem<F>(LT), st, h, s);
  } else {
    if (fwd) kwb_launch(k_eos_fwd_fast<F, LT, P::MINB, false>, grid, LT * F::G, eos_smem<F>(LT), st, h, s);
    else kwb_launch(k_eos_inv_fast<F, LT, P::MINB, false>, grid, LT * F::G, eos_smem<F>(LT), st, h, s);
  }
}

template <int N>
static inline cudaError_t launch_eos_n(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st) {
  using P = LinePolicy<N>;
  constexpr int G = P::template F<true>::G;
  constexpr int BIG = P::THREADS / G, SMALL = (32 / G > 2 ? 32 / G : 2);
  constexpr int MID = ((128 / G) & ~1) > SMALL ? ((128 / G) & ~1) : SMALL;  // even line counts
  switch (tile_variant(h, fwd ? KWB_SLOT_EOS_FWD : KWB_SLOT_EOS_INV, (long long)cdiv(h.N[1], 2 * BIG) * h.N[2])) {
    case 1: eos_go<N, MID>(d_sim, h, fwd, s, st); break;
    case 2: eos_go<N, SMALL>(d_sim, h, fwd, s, st); break;
    default: eos_go<N, BIG>(d_sim, h, fwd, s, st); break;
  }
  return cudaGetLastError();
}

template <int N, int LT>
static inline void spec_go(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s, cudaStream_t st) {
  using P = LinePolicy<N>;
  using F = typename P::template F<false>;
  const int grid = cdiv(h.n1, LT) * (axis == 1 ? h.N[2] : h.N[1]);
  kwb_launch(k_spec_fast<F, LT, P::MINB>, grid, LT * F::G, eos_smem<F>(LT), st, h, axis, op, s);
}

template <int N>
static inline cudaError_t launch_spec_n(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                                 cudaStream_t st) {
  using P = LinePolicy<N>;
  constexpr int G = P::template F<true>::G;
  constexpr int BIG = P::THREADS / G, SMALL = (32 / G > 2 ? 32 / G : 2);
  constexpr int MID = ((128 / G) & ~1) > SMALL ? ((128 / G) & ~1) : SMALL;  // even line counts
  switch (tile_variant(h, KWB_SLOT_SPEC1 + axis - 1, (long long)cdiv(h.n1, BIG) * (axis == 1 ? h.N[2] : h.N[1]))) {
    case 1: spec_go<N, MID>(d_sim, h, axis, op, s, st); break;
    case 2: spec_go<N, SMALL>(d_sim, h, axis, op, s, st); break;
    default: spec_go<N, BIG>(d_sim, h, axis, op, s, st); break;
  }
  return cudaGetLastError();
}

// Cluster plane pass for Ny = Nz = 256.  Variants: 0 -- k_plane_fast with 8 CTAs of 512 threads
// per kx plane (32 rows each); 1 -- k_plane_fast with 16 CTAs of 256 threads (16 rows each; a
// non-portable cluster size); 2 and 3 -- k_plane_cols with the same two cluster shapes (its
// multiplier in the slot-major layout); 4 and 5 -- k_plane_cols with 1024-thread CTAs in
// clusters of 4 or 8.
using PlaneFY = LinePolicy<256>::F<true>;
using PlaneFZ = LinePolicy<256>::F<false>;
template <int V> struct PlaneVariant;
template <> struct PlaneVariant<0> {
  static constexpr int CL = 8, THREADS = 512, MINB = 2;
  static constexpr bool COLS = false;
};
template <> struct PlaneVariant<1> {
  static constexpr int CL = 16, THREADS = 256, MINB = 4;
  static constexpr bool COLS = false;
};
template <> struct PlaneVariant<2> {
  static constexpr int CL = 8, THREADS = 512, MINB = 2;
  static constexpr bool COLS = true;
};
template <> struct PlaneVariant<3> {
  static constexpr int CL = 16, THREADS = 256, MINB = 3;
  static constexpr bool COLS = true;
};
// one 1024-thread CTA per SM: clusters of 4 (64 rows each) or of 8 (32 rows, one per warp)
template <> struct PlaneVariant<4> {
  static constexpr int CL = 4, THREADS = 1024, MINB = 1;
  static constexpr bool COLS = true;
};
template <> struct PlaneVariant<5> {
  static constexpr int CL = 8, THREADS = 1024, MINB = 1;
  static constexpr bool COLS = true;
};
template <int V>
constexpr size_t plane_smem_of() {
  using P = PlaneVariant<V>;
  constexpr int RZ = 256 / P::CL;
  if (P::COLS) {
    constexpr int W = P::THREADS / 32;
    return ((size_t)256 * (RZ + 1) + W * PlaneFY::LP + 2 * PlaneFY::TW) * sizeof(float2);
  }
  constexpr int LY = P::THREADS / PlaneFY::G, LZ = P::THREADS / PlaneFZ::G;
  constexpr int XS = (LY * PlaneFY::LP > LZ * PlaneFZ::LP) ? LY * PlaneFY::LP : LZ * PlaneFZ::LP;
  return ((size_t)RZ * 256 + XS + PlaneFY::TW + PlaneFZ::TW) * sizeof(float2);
}
template <int V>
inline auto plane_kernel() {
  using P = PlaneVariant<V>;
  if constexpr (P::COLS)
    return k_plane_cols<PlaneFY, P::CL, P::THREADS, P::MINB>;
  else
    return k_plane_fast<PlaneFY, PlaneFZ, P::CL, P::THREADS, P::MINB>;
}
template <int V>
inline const void *plane_fn() {
  return (const void *)plane_kernel<V>();
}
template <int V>
inline cudaLaunchConfig_t plane_cfg(int n1, cudaStream_t st, cudaLaunchAttribute *at, bool pdl) {
  using P = PlaneVariant<V>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(n1 * P::CL);
  cfg.blockDim = dim3(P::THREADS);
  cfg.dynamicSmemBytes = plane_smem_of<V>();
  cfg.stream = st;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = P::CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 2 : 1;
  return cfg;
}
// Clusters of variant V that fit on the device at once (0: the variant is unavailable).
template <int V>
inline int plane_clusters_of() {
  using P = PlaneVariant<V>;
  const void *fn = plane_fn<V>();
  if (raise_smem(fn, plane_smem_of<V>()) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (P::CL > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchAttribute at[2];
  cudaLaunchConfig_t cfg = plane_cfg<V>(16, nullptr, at, false);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
static inline int plane_clusters_per_device() { return plane_clusters_of<0>(); }
template <int V>
inline cudaError_t plane_launch(const SimDev &h, long long s, cudaStream_t st) {
  cudaLaunchAttribute at[2];
  cudaLaunchConfig_t cfg = plane_cfg<V>(h.n1, st, at, true);
  return cudaLaunchKernelEx(&cfg, plane_kernel<V>(), h, s);
}

// ------------------------------------------------------------------------------------------
// elastic solver: directional derivatives of up to three fields in one line pass (the step
// sequence and the generic shared-memory version are in kwb_elastic.cu)
// ------------------------------------------------------------------------------------------

// The fields go through the two staging slots in turn: field f + 1 lands while field f is
// transformed, and field f + 2 takes field f's slot once every thread holds field f.  Each
// derivative is written, or added to the destination (bit f of g.acc).
template <class F, bool CONTIG, int LT, int MINB>
__global__ void __launch_bounds__(LT * F::G, MINB)
    k_el_grad_fast(const __grid_constant__ SimDev S, int axis, const __grid_constant__ ElGrad g, long long step_s) {
  constexpr int E = F::E, G = F::G;
  constexpr int RP = G + 1, LP = F::LP;
  constexpr int L = LT;
  extern __shared__ __align__(128) float4 smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw2 = sm + L * LP;
  float2 *gp2 = tw2 + F::TW;
  float2 *gn2 = gp2 + E * RP;
  build_line_tables<F>(tw2, gp2, gn2, S.tw[axis], S.gpos[axis], S.gneg[axis]);
  KWB_STEP_KERNEL_PROLOGUE();
  if (*S.t0 + step_s >= S.Nt) return;
  const int tid = threadIdx.x;
  const int tt = CONTIG ? tid % G : tid / L;
  const int l = CONTIG ? tid / G : tid % L;
  constexpr int N = E * G, THREADS = LT * G;
  const int Nx = S.N[0];
  long long base;
  int cnt;
  int st32 = 1;
  if (CONTIG) {
    const int Ny = S.N[1];
    const int rows = 2 * L, tpp = (Ny + rows - 1) / rows;
    const int z = blockIdx.x / tpp, y0 = (blockIdx.x - z * tpp) * rows;
    cnt = min(rows, Ny - y0);
    base = ((long long)z * Ny + y0) * Nx;
  } else {
    const int cols = 2 * L, tpp = (Nx + cols - 1) / cols;
    const int o = blockIdx.x / tpp, x0 = (blockIdx.x - o * tpp) * cols;
    cnt = min(cols, Nx - x0);
    if (axis == 1) {
      base = (long long)o * Nx * S.N[1] + x0;
      st32 = Nx;
    } else {
      base = (long long)o * Nx + x0;
      st32 = Nx * S.N[1];
    }
  }
  const bool va = 2 * l < cnt, vb = 2 * l + 1 < cnt;
  auto off = [&](int c, int i) -> int { return CONTIG ? c * Nx + i : i * st32 + c; };
  float *st0 = reinterpret_cast<float *>(reinterpret_cast<char *>(smem_raw) + pline_offset<F>(L));
  float *st1 = st0 + 2 * L * N;
  auto stage = [&](float *dst, const float *f) {
    const float *fb = f + base;
    if (CONTIG) {
      constexpr int CH = 2 * L * N / 4, PER = (CH + THREADS - 1) / THREADS;
      const int chunks = cnt * N / 4;
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int q = tid + k * THREADS;
        if (q < chunks) cp_async16(dst + 4 * q, fb + 4 * q, 16);
      }
    } else {
      constexpr int CPR = (2 * L) / 4;
      static_assert(THREADS % CPR == 0 && (CPR * N) % THREADS == 0, "strided staging");
      constexpr int RSTEP = THREADS / CPR, PER = CPR * N / THREADS;
      const int ch = tid % CPR, i0 = tid / CPR;
      const int valid = min(4, cnt - 4 * ch);
      const int bytes = valid > 0 ? 4 * valid : 0;
      float *d0 = dst + i0 * 2 * L + 4 * ch;
      const float *s0 = fb + i0 * st32 + 4 * ch;
      const int sstep = RSTEP * st32;
#pragma unroll
      for (int k = 0; k < PER; ++k) cp_async16(d0 + k * RSTEP * 2 * L, s0 + k * sstep, bytes);
    }
    cp_async_commit();
  };

  auto staged = [&](const float *st, int i) -> float2 {
    if (CONTIG) return make_float2(va ? st[(2 * l) * N + i] : 0.f, vb ? st[(2 * l + 1) * N + i] : 0.f);
    return *reinterpret_cast<const float2 *>(st + i * 2 * L + 2 * l);
  };
  // the destination as this kernel may already have written it: ordinary (coherent) loads
  auto load_cur = [&](const float *f, int i) -> float2 {
    const float *fb = f + base;
    if (!CONTIG) return vb ? *reinterpret_cast<const float2 *>(fb + off(2 * l, i)) : make_float2(0.f, 0.f);
    return make_float2(va ? fb[off(2 * l, i)] : 0.f, vb ? fb[off(2 * l + 1, i)] : 0.f);
  };
  auto store_pair = [&](float *f, int i, float2 v) {
    float *fb = f + base;
    if (!CONTIG) {
      if (vb) *reinterpret_cast<float2 *>(fb + off(2 * l, i)) = v;
      return;
    }
    if (va) fb[off(2 * l, i)] = v.x;
    if (vb) fb[off(2 * l + 1, i)] = v.y;
  };
  const float2 *mul = g.neg ? gn2 : gp2;
  stage(st0, g.src[0]);
  if (g.nf > 1) stage(st1, g.src[1]);
  else cp_async_commit();
  float2 *xs = sm + l * LP;
  for (int f = 0; f < g.nf; ++f) {
    float *slot = (f & 1) ? st1 : st0;
    if (f == g.nf - 1) cp_async_wait<0>();
    else cp_async_wait<1>();
    __syncthreads();  // field f has landed for every thread; the tables too
    float2 v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) v[r] = staged(slot, tt + G * r);
    if (f + 2 < g.nf) {
      __syncthreads();  // every thread holds field f
      stage(slot, g.src[f + 2]);
    }
    F::fwd(v, xs, tw2, tt);
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = cmul(v[q], mul[q * RP + tt]);
    float *dst = g.dst[f];
    const bool acc = (g.acc >> f) & 1;
    // the running sum is loaded while the inverse transform runs
    float2 prev[E];
#pragma unroll
    for (int r = 0; r < E; ++r) prev[r] = acc ? load_cur(dst, tt + G * r) : make_float2(0.f, 0.f);
    F::inv(v, xs, tw2, tt);
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int i = tt + G * r;
      store_pair(dst, i, acc ? padd(prev[r], v[r]) : v[r]);
    }
  }
}

template <int N, int LT>
static inline void el_go(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st) {
  using P = LinePolicy<N>;
  if (axis == 0) {
    using F = typename P::template F<true>;
    kwb_launch(k_el_grad_fast<F, true, LT, P::MINB>, cdiv(h.N[1], 2 * LT) * h.N[2], LT * F::G, pline_smem<F>(LT),
               st, h, axis, g, s);
  } else {
    using F = typename P::template F<false>;
    kwb_launch(k_el_grad_fast<F, false, LT, P::MINB>, cdiv(h.N[0], 2 * LT) * (axis == 1 ? h.N[2] : h.N[1]),
               LT * F::G, pline_smem<F>(LT), st, h, axis, g, s);
  }
}

template <int N>
static inline cudaError_t launch_el_n(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st) {
  using P = LinePolicy<N>;
  constexpr int G = P::template F<true>::G;
  constexpr int BIG = P::THREADS / G, SMALL = (32 / G > 2 ? 32 / G : 2);
  constexpr int MID = ((128 / G) & ~1) > SMALL ? ((128 / G) & ~1) : SMALL;  // even line counts
  const long long tiles = axis == 0 ? (long long)cdiv(h.N[1], 2 * BIG) * h.N[2]
                                    : (long long)cdiv(h.N[0], 2 * BIG) * (axis == 1 ? h.N[2] : h.N[1]);
  switch (tile_variant(h, KWB_SLOT_LINE0 + axis, tiles)) {
    case 1: el_go<N, MID>(h, axis, g, s, st); break;
    case 2: el_go<N, SMALL>(h, axis, g, s, st); break;
    default: el_go<N, BIG>(h, axis, g, s, st); break;
  }
  return cudaGetLastError();
}

}  // namespace fast
}  // namespace kwb
