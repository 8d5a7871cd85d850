// C ABI of libkwb: context, validation, device admission, simulation set-up, stepping
// (eager or CUDA-graph replay), output read-back and per-kernel profiling.
//
// The set-up restates the allocation and pre-computation half of kspace_first_order
// (KWave.jl/src/solver/first_order.jl:92-441 for 1D/2D, 505-669 for 3D); the stepping restates
// its time loop (first_order.jl:232-266, 448-484, 677-713) with the kernels of kwb_fast.cu and
// kwb_kernels.cu; elastic problems step through elastic_step (kernels in kwb_elastic.cu).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <sys/stat.h>

#include "../../include/kwb.h"
#include "kwb_internal.h"

struct KwbServer;  // kwb_serve.cu

struct kwb_ctx {
  int device = 0;
  std::string err;
  KwbServer *server = nullptr;  // started by the first kwb_submit
  // pinned staging for device -> host read-back (two halves), allocated on first use
  float *pin = nullptr;
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  // Device memory pool of this context's simulations: stream-ordered allocation, and freed
  // blocks stay in the pool for the next simulation (no unmapping between simulations).
  cudaMemPool_t pool = nullptr;
  // The continuous-batching scheduler's private context: its simulations share the GPU with
  // one another, so they keep full-width tiles (kwb_sim_create, grid_fill).
  bool batched = false;
  ~kwb_ctx() {
    if (pool) cudaMemPoolDestroy(pool);  // released once outstanding blocks are freed
    if (pin) cudaFreeHost(pin);
    for (cudaEvent_t e : pin_ev)
      if (e) cudaEventDestroy(e);
  }
};

size_t estimate_device_bytes(const kwb_problem *P);
void kwb_server_shutdown(kwb_ctx *ctx);

static std::string g_create_err;
static const double kPi = 3.141592653589793238462643;

namespace {

using namespace kwb;

int set_err(kwb_ctx *ctx, int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return code;
}

// Split [0, n) over host threads (one thread below 256K elements per thread).
template <class Fn>
void parallel_range(long long n, Fn fn) {
  const long long hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
  const long long T = std::min(hw, (n + (1 << 18) - 1) >> 18);
  if (T <= 1) {
    fn(0LL, n);
    return;
  }
  const long long per = (n + T - 1) / T;
  std::vector<std::thread> th;
  for (long long k = 1; k < T; ++k) {
    const long long lo = k * per, hi = std::min(n, lo + per);
    if (lo < hi) th.emplace_back(fn, lo, hi);
  }
  fn(0LL, std::min(n, per));
  for (auto &x : th) x.join();
}

#define CU(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return set_err(ctx, KWB_E_DEVICE, "CUDA error %s at %s:%d (%s)",                  \
                     cudaGetErrorString(e_), __FILE__, __LINE__, #call);                \
  } while (0)

// Device FP32 array -> caller's FP64 array in chunks through the context's pinned buffer: the
// next chunk's copy (on `st`) overlaps this chunk's conversion, which runs on host threads (and
// so also takes the first-touch page faults of a freshly allocated destination in parallel).
constexpr long long kPinFloats = 8LL << 20;  // floats per half of the pinned buffer (32 MB)
int read_f32_as_f64(kwb_ctx *ctx, cudaStream_t st, const float *src, long long cnt, double *dst) {
  if (cnt <= 0) return KWB_OK;
  if (!ctx->pin) {
    CU(cudaMallocHost(&ctx->pin, 2 * kPinFloats * sizeof(float)));
    for (cudaEvent_t &e : ctx->pin_ev) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const long long nch = (cnt + kPinFloats - 1) / kPinFloats;
  auto issue = [&](long long c) -> cudaError_t {
    const long long lo = c * kPinFloats, len = std::min(kPinFloats, cnt - lo);
    cudaError_t e = cudaMemcpyAsync(ctx->pin + (c & 1) * kPinFloats, src + lo, len * 4, cudaMemcpyDeviceToHost, st);
    return e == cudaSuccess ? cudaEventRecord(ctx->pin_ev[c & 1], st) : e;
  };
  CU(issue(0));
  for (long long c = 0; c < nch; ++c) {
    CU(cudaEventSynchronize(ctx->pin_ev[c & 1]));
    if (c + 1 < nch) CU(issue(c + 1));
    const long long lo = c * kPinFloats, len = std::min(kPinFloats, cnt - lo);
    const float *sp = ctx->pin + (c & 1) * kPinFloats;
    double *dp = dst + lo;
    parallel_range(len, [sp, dp](long long a, long long b) {
      for (long long i = a; i < b; ++i) dp[i] = (double)sp[i];
    });
  }
  return KWB_OK;
}

// Julia's mean() sums pairwise; a pairwise sum keeps c_ref at FP64 round-off as well.  The top
// `par` levels of the same halving tree run on separate threads (the sum is the same, bit for
// bit, as the sequential recursion).
double pairwise_sum(const double *x, long long n, int par = 0) {
  if (n <= 128) {
    double s = 0.0;
    for (long long i = 0; i < n; ++i) s += x[i];
    return s;
  }
  const long long h = n / 2;
  if (par > 0 && n >= (1LL << 20)) {
    double left = 0.0;
    std::thread t([&] { left = pairwise_sum(x, h, par - 1); });
    const double right = pairwise_sum(x + h, n - h, par - 1);
    t.join();
    return left + right;
  }
  return pairwise_sum(x, h) + pairwise_sum(x + h, n - h);
}

}  // namespace

namespace kwb {

// Stockham stage radices of a line of N points: 8s first, then 4 or 2, then 3, 5, 7.
bool make_plan_order(int N, FftPlan &pl, int order) {
  pl.n = N;
  pl.nstages = 0;
  int n = N, a = 0;
  while (n % 2 == 0) {
    n /= 2;
    ++a;
  }
  int odd[KWB_MAX_STAGES], nodd = 0;
  for (int p : {3, 5, 7}) {
    while (n % p == 0) {
      if (nodd >= KWB_MAX_STAGES) return false;
      odd[nodd++] = p;
      n /= p;
    }
  }
  if (n != 1) return false;
  auto push = [&](int r) {
    if (pl.nstages >= KWB_MAX_STAGES) return false;
    pl.radix[pl.nstages++] = r;
    return true;
  };
  if (order == 2)
    for (int i = 0; i < nodd; ++i)
      if (!push(odd[i])) return false;
  const int big = order == 1 ? 2 : 3;  // log2 of the largest power-of-two radix
  while (a >= big)
    if (!push(1 << big)) return false;
    else a -= big;
  if (a == 2 && !push(4)) return false;
  if (a == 1 && !push(2)) return false;
  if (order != 2)
    for (int i = 0; i < nodd; ++i)
      if (!push(odd[i])) return false;
  // the stages' divisions by the butterflies per line and by the sub-transform length so far
  int ns = 1;
  for (int st = 0; st < pl.nstages; ++st) {
    pl.div_nr[st] = make_fastdiv((unsigned)(N / pl.radix[st]));
    pl.div_ns[st] = make_fastdiv((unsigned)ns);
    ns *= pl.radix[st];
  }
  return true;
}

bool make_plan(int N, FftPlan &pl) { return make_plan_order(N, pl, 0); }

bool plan_line(int N, FftPlan &pl, int order) {
  const float2 *chirp = pl.chirp, *chirp_ft = pl.chirp_ft;  // tables built by the caller
  pl.m = 0;
  if (!make_plan_order(N, pl, order)) {
    if (N > KWB_BLUESTEIN_MAX_N) return false;
    int M = 1;
    while (M < 2 * N - 1) M *= 2;
    if (!make_plan_order(M, pl, order)) return false;
    pl.n = N;
    pl.m = M;
  }
  pl.chirp = chirp;
  pl.chirp_ft = chirp_ft;
  return true;
}

// Bluestein tables of an n-point line with inner length m (FP64, rounded once): the chirp
// w_j = exp(-i pi j^2/n) (j^2 reduced mod 2n exactly, in integers) and FFT_m of its conjugate
// wrapped to length m (b_j = b_{m-j} = conj(w_j), j < n), scaled by 1/m.
void bluestein_tables(int n, int m, std::vector<float2> &chirp, std::vector<float2> &chirp_ft) {
  const double pi = 3.141592653589793238462643;
  std::vector<double> wr(n), wi(n);
  for (int j = 0; j < n; ++j) {
    const long long q = ((long long)j * j) % (2LL * n);
    const double th = pi * (double)q / (double)n;
    wr[j] = std::cos(th);
    wi[j] = -std::sin(th);
  }
  std::vector<double> br(m, 0.0), bi(m, 0.0);
  for (int j = 0; j < n; ++j) {
    br[j] = wr[j];
    bi[j] = -wi[j];
    if (j > 0) {
      br[m - j] = wr[j];
      bi[m - j] = -wi[j];
    }
  }
  // iterative radix-2 FFT (forward, exp(-2 pi i jk/m)), m a power of two
  for (int i = 1, j = 0; i < m; ++i) {
    int bit = m >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      std::swap(br[i], br[j]);
      std::swap(bi[i], bi[j]);
    }
  }
  for (int len = 2; len <= m; len <<= 1) {
    for (int k = 0; k < len / 2; ++k) {
      const double a = -2.0 * pi * (double)k / (double)len;
      const double cr = std::cos(a), ci = std::sin(a);
      for (int i = 0; i < m; i += len) {
        const int u = i + k, v = i + k + len / 2;
        const double tr = br[v] * cr - bi[v] * ci, ti = br[v] * ci + bi[v] * cr;
        br[v] = br[u] - tr;
        bi[v] = bi[u] - ti;
        br[u] += tr;
        bi[u] += ti;
      }
    }
  }
  chirp.resize(n);
  chirp_ft.resize(m);
  for (int j = 0; j < n; ++j) chirp[j] = make_float2((float)wr[j], (float)wi[j]);
  for (int k = 0; k < m; ++k) chirp_ft[k] = make_float2((float)(br[k] / m), (float)(bi[k] / m));
}

int choose_L(int N, int want, int cap_lines, int dispersion, bool spec) {
  int L = want;
  if (L < 1) L = 1;
  while (L > 1 && (spec ? spec_pass_smem(N, L, dispersion) : line_pass_smem(N, L)) > 200 * 1024)
    L /= 2;
  if (cap_lines > 0 && L > cap_lines) L = cap_lines;
  if (L < 1) L = 1;
  return L;
}

}  // namespace kwb

namespace {

// Stream-ordered device scratch for simulation set-up (FP64 staging of the medium): freed on
// the set-up stream when the creating call returns, so it holds no memory afterwards.
struct TempBuf {
  cudaStream_t st = nullptr;
  cudaMemPool_t pool = nullptr;
  std::vector<void *> ptrs;
  TempBuf(cudaStream_t s, cudaMemPool_t p) : st(s), pool(p) {}
  ~TempBuf() {
    for (void *p : ptrs) cudaFreeAsync(p, st);
  }
  template <class T>
  cudaError_t alloc(T **out, size_t count) {
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, (count ? count : 1) * sizeof(T), pool, st);
    if (e != cudaSuccess) return e;
    ptrs.push_back(p);
    *out = static_cast<T *>(p);
    return cudaSuccess;
  }
};

// A simulation's device buffers, allocated and released in stream order on its stream (`st`):
// releasing them does not wait for the rest of the device, unlike cudaFree, so retiring one of
// many concurrent simulations does not stall the others.
struct DevBuf {
  std::vector<void *> ptrs;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  cudaMemPool_t pool = nullptr;
  void release() {
    for (void *p : ptrs) {
      if (st) cudaFreeAsync(p, st);
      else cudaFree(p);
    }
    ptrs.clear();
  }
  ~DevBuf() { release(); }
  template <class T>
  cudaError_t alloc(T **out, size_t count) {
    void *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = st ? cudaMallocFromPoolAsync(&p, count * sizeof(T), pool, st) : cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) return e;
    ptrs.push_back(p);
    bytes += count * sizeof(T);
    *out = static_cast<T *>(p);
    return cudaSuccess;
  }
};

}  // namespace

__global__ void kwb_k_fill_f32(float *p, long long n, float v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
__global__ void kwb_k_fill_f64(double *p, long long n, double v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

struct GroupHost {
  kwb_sensor_group spec;
  GroupDev dev{};
  GroupDev *d_dev = nullptr;
  long long n = 0;
  bool fused = false;  // updated inside the x C2R pass
  // post-loop filters of the p series: distinct filters (sin(theta) of their directivity, NaN
  // for none) and the filter of each point; empty when the group has no filter
  std::vector<double> filt_sin;
  std::vector<int> filt_of;
};

struct kwb_sim {
  kwb_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  DevBuf mem;
  SimDev h{};
  SimDev *d_sim = nullptr;
  long long *d_t0 = nullptr;
  long long t0_host = 0;
  long long Nt_loop = 0;
  long long Nt_grid = 0;
  long long steps_done = 0;
  double d[3] = {1.0, 1.0, 1.0};  // grid spacing and time step (post-loop filters)
  double dt = 0.0;
  std::string schedule_src = "heuristic";  // where the FFT schedule came from (kwb_sim_schedule)
  std::vector<GroupHost> groups;
  bool tr = false;
  kwb_progress_fn progress = nullptr;
  void *progress_user = nullptr;
  float *p_host = nullptr;  // pinned, progress callback
  cudaGraphExec_t graph = nullptr;
  int graph_K = 0;
  int launches_per_step = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~kwb_sim() {
    if (graph) cudaGraphExecDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (p_host) cudaFreeHost(p_host);
    mem.release();  // stream-ordered, before the stream goes
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

int validate_index(kwb_ctx *ctx, const int64_t *idx, int64_t n, int64_t nvox, const char *what) {
  if (n < 0) return set_err(ctx, KWB_E_INVALID, "%s: negative point count", what);
  if (n > 0 && !idx) return set_err(ctx, KWB_E_INVALID, "%s: index pointer is NULL", what);
  for (int64_t i = 0; i < n; ++i) {
    if (idx[i] < 0 || idx[i] >= nvox)
      return set_err(ctx, KWB_E_INVALID, "%s: index %lld out of range [0, %lld)", what,
                     (long long)idx[i], (long long)nvox);
    if (i > 0 && idx[i] <= idx[i - 1])
      return set_err(ctx, KWB_E_INVALID, "%s: indices must be sorted and unique", what);
  }
  return KWB_OK;
}

int validate_problem(kwb_ctx *ctx, const kwb_problem *P) {
  if (!P) return set_err(ctx, KWB_E_INVALID, "problem is NULL");
  if (P->ndim < 1 || P->ndim > 3) return set_err(ctx, KWB_E_INVALID, "ndim must be 1, 2 or 3");
  long long nvox = 1;
  for (int a = 0; a < 3; ++a) {
    const int64_t n = a < P->ndim ? P->N[a] : 1;
    if (n < 1) return set_err(ctx, KWB_E_INVALID, "grid size N[%d] = %lld must be >= 1", a, (long long)n);
    if (n > KWB_MAX_N)
      return set_err(ctx, KWB_E_UNSUPPORTED, "grid size N[%d] = %lld exceeds %d", a, (long long)n, KWB_MAX_N);
    FftPlan pl{};
    if (!plan_line((int)n, pl, 0))
      return set_err(ctx, KWB_E_UNSUPPORTED,
                     "grid size N[%d] = %lld has a prime factor above 7 and exceeds %d, the longest "
                     "line transformed by Bluestein's algorithm (radix 2, 3, 5, 7 lengths up to %d)",
                     a, (long long)n, KWB_BLUESTEIN_MAX_N, KWB_MAX_N);
    if (a < P->ndim && !(P->d[a] > 0)) return set_err(ctx, KWB_E_INVALID, "grid spacing d[%d] must be > 0", a);
    nvox *= n;
  }
  if (P->Nt == 0 || P->dt == 0)
    return set_err(ctx, KWB_E_INVALID, "Time array not set. Call make_time!(kgrid, sound_speed) before running.");
  if (P->Nt < 0 || !(P->dt > 0)) return set_err(ctx, KWB_E_INVALID, "Nt and dt must be positive");
  if (P->axisymmetric && P->ndim != 2)
    return set_err(ctx, KWB_E_INVALID, "the axisymmetric solver takes a 2D grid (x axial, y radial)");
  if (P->axisymmetric && P->tr.data)
    return set_err(ctx, KWB_E_INVALID, "time reversal is not part of the axisymmetric solver");
  for (int a = 0; a < P->ndim; ++a)
    if (P->pml_size[a] < 0) return set_err(ctx, KWB_E_INVALID, "pml_size must be >= 0");
  auto chk_field = [&](const kwb_field &f, const char *nm, bool optional) -> int {
    if (f.count == 0) return optional ? KWB_OK : set_err(ctx, KWB_E_INVALID, "%s is required", nm);
    if (!f.data) return set_err(ctx, KWB_E_INVALID, "%s: data is NULL", nm);
    if (f.count != 1 && f.count != nvox)
      return set_err(ctx, KWB_E_INVALID, "%s: %lld values for a grid of %lld points", nm,
                     (long long)f.count, nvox);
    return KWB_OK;
  };
  int rc;
  if (P->elastic) {
    if (P->ndim < 2) return set_err(ctx, KWB_E_INVALID, "the elastic solver takes a 2D or 3D grid");
    if (P->axisymmetric || P->tr.data)
      return set_err(ctx, KWB_E_INVALID, "time reversal and the axisymmetric form are not part of the elastic solver");
    if (P->BonA.count) return set_err(ctx, KWB_E_INVALID, "B/A is not part of the elastic solver");
    if (P->n_p_index > 0)
      return set_err(ctx, KWB_E_INVALID, "the elastic solver has stress sources, not pressure sources");
    if ((rc = chk_field(P->cs, "sound_speed_shear", false))) return rc;
    const bool speed_arr = (P->c0.count == nvox || P->cs.count == nvox) && nvox > 1;
    if (speed_arr && !(P->rho0.count == nvox && nvox > 1))
      return set_err(ctx, KWB_E_INVALID,
                     "a scalar density with array wave speeds is evaluated as a matrix power (cp^2) by the "
                     "reference (solver/elastic.jl:169); give the density as an array");
    if (P->has_alpha_shear && !(std::isfinite(P->alpha_coeff_shear) && std::isfinite(P->alpha_power)))
      return set_err(ctx, KWB_E_INVALID, "alpha_coeff_shear and alpha_power must be set for shear absorption");
    if ((rc = validate_index(ctx, P->s_index, P->n_s_index, nvox, "s_mask"))) return rc;
    for (int k = 0; k < 6; ++k) {
      if (!P->s_signal[k].data || P->n_s_index == 0) continue;
      if (P->s_signal[k].n_rows < P->n_s_index || P->s_signal[k].n_cols < 1)
        return set_err(ctx, KWB_E_INVALID, "BoundsError: stress source %d has %lld rows for %lld s_mask points",
                       k, (long long)P->s_signal[k].n_rows, (long long)P->n_s_index);
    }
  } else if (P->n_s_index > 0) {
    return set_err(ctx, KWB_E_INVALID, "stress sources belong to the elastic solver");
  }
  if ((rc = chk_field(P->c0, "sound_speed", false))) return rc;
  if ((rc = chk_field(P->rho0, "density", true))) return rc;
  if ((rc = chk_field(P->BonA, "BonA", true))) return rc;
  if (P->p0.count != 0 && (P->p0.count != nvox || !P->p0.data))
    return set_err(ctx, KWB_E_INVALID, "p0 must have one value per grid point");
  if (P->alpha_mode < 0 || P->alpha_mode > 2) return set_err(ctx, KWB_E_INVALID, "bad alpha_mode");
  if ((rc = validate_index(ctx, P->p_index, P->n_p_index, nvox, "p_mask"))) return rc;
  if ((rc = validate_index(ctx, P->u_index, P->n_u_index, nvox, "u_mask"))) return rc;
  if (P->n_p_index > 0) {
    if (!P->p_signal.data) return set_err(ctx, KWB_E_INVALID, "pressure source signal is NULL");
    if (P->p_signal.n_rows < P->n_p_index || P->p_signal.n_cols < 1)
      return set_err(ctx, KWB_E_INVALID,
                     "BoundsError: source.p has %lld rows for %lld p_mask points",
                     (long long)P->p_signal.n_rows, (long long)P->n_p_index);
  }
  for (int d = 0; d < 3; ++d) {
    if (!P->u_signal[d].data || P->n_u_index == 0) continue;
    if (P->u_signal[d].n_rows < P->n_u_index || P->u_signal[d].n_cols < 1)
      return set_err(ctx, KWB_E_INVALID, "BoundsError: velocity source %d has %lld rows for %lld u_mask points",
                     d, (long long)P->u_signal[d].n_rows, (long long)P->n_u_index);
  }
  if (P->n_groups < 0 || (P->n_groups > 0 && !P->groups))
    return set_err(ctx, KWB_E_INVALID, "sensor groups missing");
  for (int g = 0; g < P->n_groups; ++g) {
    const kwb_sensor_group &G = P->groups[g];
    if (G.record_mask >> KWB_REC_COUNT) return set_err(ctx, KWB_E_INVALID, "bad record mask");
    if (!G.dense && !G.cartesian && (rc = validate_index(ctx, G.index, G.n_index, nvox, "sensor mask")))
      return rc;
    if (G.dense && G.n_index != nvox && G.n_index != 0)
      return set_err(ctx, KWB_E_INVALID, "dense sensor group must cover the grid");
  }
  if (P->tr.data) {
    if (P->n_groups < 1) return set_err(ctx, KWB_E_INVALID, "time reversal needs a sensor mask");
    const kwb_sensor_group &G = P->groups[0];
    const long long npts = G.cartesian ? 0 : (G.dense ? nvox : G.n_index);
    if (P->tr.n_cols < 1) return set_err(ctx, KWB_E_INVALID, "time-reversal data has no columns");
    if (npts > 0 && P->tr.n_rows < npts)
      return set_err(ctx, KWB_E_INVALID, "BoundsError: time-reversal data has %lld rows for %lld mask points",
                     (long long)P->tr.n_rows, npts);
    const uint32_t series = (1u << KWB_REC_P) | (1u << KWB_REC_UX) | (1u << KWB_REC_UY) | (1u << KWB_REC_UZ);
    for (int g = 0; g < P->n_groups; ++g)
      if ((P->groups[g].record_mask & series) && !P->groups[g].cartesian && P->tr.n_cols > P->Nt)
        return set_err(ctx, KWB_E_INVALID,
                       "BoundsError: time-series outputs have %lld columns but time reversal runs %lld steps",
                       (long long)P->Nt, (long long)P->tr.n_cols);
  }
  if (P->alpha_mode != KWB_NO_ABSORPTION) {
    if (!std::isfinite(P->alpha_coeff) || !std::isfinite(P->alpha_power))
      return set_err(ctx, KWB_E_INVALID, "alpha_coeff and alpha_power must be set for an absorbing medium");
  }
  return KWB_OK;
}

void group_sizes(const kwb_problem *P, const kwb_sensor_group &G, long long nvox, kwb_group_sizes &s) {
  for (int f = 0; f < KWB_REC_COUNT; ++f) s.rows[f] = s.cols[f] = 0;
  const long long n = G.dense ? nvox : G.n_index;
  for (int f = 0; f < KWB_REC_COUNT; ++f) {
    if (!(G.record_mask & (1u << f))) continue;
    s.rows[f] = n;
    const bool series = f == KWB_REC_P || f == KWB_REC_UX || f == KWB_REC_UY || f == KWB_REC_UZ;
    s.cols[f] = series ? P->Nt : 1;
  }
}

// Point sources that fall on the lines of axis `a`: CSR over line ids.
void build_csr(const int64_t *idx, long long n, const int N[3], int a, std::vector<int> &ptr,
               std::vector<SrcEntry> &ent) {
  const long long Nx = N[0], Ny = N[1], Nz = N[2];
  const long long n_lines = a == 0 ? Ny * Nz : (a == 1 ? Nx * Nz : Nx * Ny);
  ptr.assign(n_lines + 1, 0);
  std::vector<SrcEntry> tmp(n);
  for (long long j = 0; j < n; ++j) {
    const long long v = idx[j];
    const long long x = v % Nx, y = (v / Nx) % Ny, z = v / (Nx * Ny);
    SrcEntry e;
    e.line = (int)(a == 0 ? y + Ny * z : (a == 1 ? x + Nx * z : x + Nx * y));
    e.pos = (int)(a == 0 ? x : (a == 1 ? y : z));
    e.j = (int)j;
    e.pad = 0;
    tmp[j] = e;
    ptr[e.line + 1]++;
  }
  for (long long l = 0; l < n_lines; ++l) ptr[l + 1] += ptr[l];
  ent.resize(n);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (long long j = 0; j < n; ++j) ent[fill[tmp[j].line]++] = tmp[j];
}

// Host -> device.  Large arrays go through the context's pinned buffer in halves: host threads
// copy chunk c into one half while the DMA of chunk c - 1 drains the other, instead of the
// driver's single-threaded staging of pageable memory.  Returns with both halves idle.
int upload(kwb_ctx *ctx, void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return KWB_OK;
  const size_t half = kPinFloats * sizeof(float);
  if (bytes < (size_t)8 << 20) {
    CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return KWB_OK;
  }
  if (!ctx->pin) {
    CU(cudaMallocHost(&ctx->pin, 2 * half));
    for (cudaEvent_t &e : ctx->pin_ev) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const size_t nch = (bytes + half - 1) / half;
  for (size_t c = 0; c < nch; ++c) {
    char *pin = reinterpret_cast<char *>(ctx->pin) + (c & 1) * half;
    if (c >= 2) CU(cudaEventSynchronize(ctx->pin_ev[c & 1]));  // this half's previous chunk is on the device
    const size_t lo = c * half, len = std::min(half, bytes - lo);
    const char *sp = static_cast<const char *>(src) + lo;
    parallel_range((long long)len, [pin, sp](long long a, long long b) { memcpy(pin + a, sp + a, (size_t)(b - a)); });
    CU(cudaMemcpyAsync(static_cast<char *>(dst) + lo, pin, len, cudaMemcpyHostToDevice, st));
    CU(cudaEventRecord(ctx->pin_ev[c & 1], st));
  }
  for (size_t c = nch > 2 ? nch - 2 : 0; c < nch; ++c) CU(cudaEventSynchronize(ctx->pin_ev[c & 1]));
  return KWB_OK;
}

int fill_f32(kwb_ctx *ctx, float *p, long long n, float v, cudaStream_t st) {
  if (n <= 0) return KWB_OK;
  kwb_k_fill_f32<<<(int)((n + 255) / 256), 256, 0, st>>>(p, n, v);
  CU(cudaGetLastError());
  return KWB_OK;
}
int fill_f64(kwb_ctx *ctx, double *p, long long n, double v, cudaStream_t st) {
  if (n <= 0) return KWB_OK;
  kwb_k_fill_f64<<<(int)((n + 255) / 256), 256, 0, st>>>(p, n, v);
  CU(cudaGetLastError());
  return KWB_OK;
}

// One elastic time step (kwb_elastic.cu).  run(name, algorithmic bytes, launcher) issues each
// launch, so the same sequence serves the captured step and the per-kernel profile.
template <class Run>
cudaError_t elastic_step(kwb_sim *S, long long s, Run &&run) {
  const SimDev &h = S->h;
  cudaStream_t st = S->stream;
  const int D = h.ndim;
  const double nv = (double)h.nvox;
  static const char *gname[2][3] = {{"el_grad_stress_x", "el_grad_stress_y", "el_grad_stress_z"},
                                    {"el_grad_velocity_x", "el_grad_velocity_y", "el_grad_velocity_z"}};
  cudaError_t e;
  // stress divergence: the pass along d adds d/dx_d sigma_dj to w_j
  for (int d = 0; d < D; ++d) {
    ElGrad g{};
    g.nf = D;
    for (int j = 0; j < D; ++j) {
      g.src[j] = h.el_s[kwb_stress_slot(d, j)];
      g.dst[j] = h.el_w[j];
    }
    g.acc = d > 0 ? 7 : 0;
    g.neg = 0;
    if ((e = run(gname[0][d], nv * 4.0 * D * (d > 0 ? 3 : 2), [&] { return el_grad(h, d, g, s, st); })) != cudaSuccess)
      return e;
  }
  if ((e = run("el_velocity", nv * 4.0 * (3 * D + (h.rho0 ? 2 : 0)), [&] { return el_velocity(h, s, st); })) != cudaSuccess)
    return e;
  if (h.n_u > 0 && (e = run("el_inject", 0.0, [&] { return el_inject(h, 0, s, st); })) != cudaSuccess) return e;
  // velocity gradients: dv_d/dx_d into w_d, dv_j/dx_d into the shear slot {d, j} (first writer
  // is the pass along the smaller axis, the other adds)
  for (int d = 0; d < D; ++d) {
    ElGrad g{};
    g.nf = D;
    int reads = D;
    for (int j = 0; j < D; ++j) {
      g.src[j] = h.u[j];
      g.dst[j] = h.el_w[kwb_stress_slot(d, j)];
      if (j < d) {
        g.acc |= 1 << j;
        ++reads;
      }
    }
    g.neg = 1;
    if ((e = run(gname[1][d], nv * 4.0 * (reads + D), [&] { return el_grad(h, d, g, s, st); })) != cudaSuccess)
      return e;
  }
  const int ns = D == 2 ? 3 : 6;
  if ((e = run("el_stress", nv * 4.0 * (3 * ns + 1 + (h.el_lam ? 2 : 0)), [&] { return el_stress(h, s, st); })) != cudaSuccess)
    return e;
  if (h.n_s > 0 && (e = run("el_inject", 0.0, [&] { return el_inject(h, 1, s, st); })) != cudaSuccess) return e;
  for (auto &g : S->groups) {
    if (g.spec.cartesian || g.n == 0) continue;
    if ((e = run("sensor_gather", 0.0, [&] { return launch_sensor_gather(S->d_sim, h, g.d_dev, g.n, s, st); })) != cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

// Enqueue one time step (eager).  step_s is relative to the device step base.
cudaError_t enqueue_step(kwb_sim *S, long long step_s) {
  const SimDev &h = S->h;
  cudaStream_t st = S->stream;
  cudaError_t e;
  if (h.elastic) return elastic_step(S, step_s, [](const char *, double, auto fn) { return fn(); });
  if (S->tr && (e = launch_tr_inject(S->d_sim, h, step_s, st)) != cudaSuccess) return e;
  // line passes: y, z, then x
  for (int a : {1, 2, 0}) {
    if (a >= h.ndim) continue;
    if ((e = launch_line_pass(S->d_sim, h, a, KWB_MODE_STEP, step_s, st)) != cudaSuccess) return e;
  }
  if (!h.fuse_xeos && (e = launch_eos_x_fwd(S->d_sim, h, step_s, st)) != cudaSuccess) return e;
  if (h.ndim == 2) {
    if ((e = launch_spec_pass(S->d_sim, h, 1, KWB_SPEC_FWD_MUL_INV, step_s, st)) != cudaSuccess) return e;
  } else if (h.ndim == 3 && h.plane) {
    if ((e = fast_plane(S->d_sim, h, step_s, st)) != cudaSuccess) return e;
  } else if (h.ndim == 3) {
    if ((e = launch_spec_pass(S->d_sim, h, 1, KWB_SPEC_FWD, step_s, st)) != cudaSuccess) return e;
    if ((e = launch_spec_pass(S->d_sim, h, 2, KWB_SPEC_FWD_MUL_INV, step_s, st)) != cudaSuccess) return e;
    if ((e = launch_spec_pass(S->d_sim, h, 1, KWB_SPEC_INV, step_s, st)) != cudaSuccess) return e;
  }
  if ((e = launch_eos_x_inv(S->d_sim, h, step_s, st)) != cudaSuccess) return e;
  for (auto &g : S->groups) {
    if (g.spec.cartesian || g.n == 0 || g.fused) continue;
    if ((e = launch_sensor_gather(S->d_sim, h, g.d_dev, g.n, step_s, st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int count_launches(const kwb_sim *S) {
  if (S->h.elastic) {
    int n = 2 * S->h.ndim + 2 + (S->h.n_u > 0 ? 1 : 0) + (S->h.n_s > 0 ? 1 : 0);
    for (auto &g : S->groups)
      if (!g.spec.cartesian && g.n > 0) ++n;
    return n;
  }
  int n = (S->tr ? 1 : 0) + S->h.ndim + (S->h.fuse_xeos ? 1 : 2) + (S->h.ndim == 2 ? 1 : (S->h.ndim == 3 ? (S->h.plane ? 1 : 3) : 0));
  for (auto &g : S->groups)
    if (!g.spec.cartesian && g.n > 0 && !g.fused) ++n;
  return n;
}

}  // namespace

// Device bytes a simulation of `P` holds (fields, spectra, medium, tables, sensor buffers and
// the FP64 upload staging), the figure admission control compares with free memory.
size_t estimate_device_bytes(const kwb_problem *P) {
  const int D = P->ndim;
  long long N[3] = {1, 1, 1};
  for (int a = 0; a < D; ++a) N[a] = P->N[a];
  const long long nvox = N[0] * N[1] * N[2];
  const long long nspec = (N[0] / 2 + 1) * N[1] * N[2];
  const bool c_arr = P->c0.count == nvox && nvox > 1;
  const bool r_arr = P->rho0.count == nvox && nvox > 1;
  const bool b_arr = P->BonA.count == nvox && nvox > 1;
  const bool nonlinear = P->BonA.count > 0;
  const bool dispersion = !c_arr && P->alpha_mode == KWB_STOKES && !P->elastic;
  size_t need;
  if (P->elastic) {
    // p, velocities, stresses and derivative scratch; rho0, lambda and mu per voxel with an array
    // density; FP64 staging of one array during set-up
    const int ns = D == 2 ? 3 : 6;
    need = (size_t)nvox * 4 * (1 + D + 2 * ns) + (size_t)nvox * 4 * (r_arr ? 3 : 0);
    if (r_arr || P->p0.count) need += (size_t)nvox * 8 * (1 + ((P->row_major && D > 1) ? 1 : 0));
    for (int k = 0; k < 6; ++k)
      if (P->s_signal[k].data) need += (size_t)P->s_signal[k].n_rows * P->s_signal[k].n_cols * 12;
    need += (size_t)P->n_s_index * 8 + (size_t)P->n_u_index * 8;
  } else {
    need = (size_t)nvox * 4 * (1 + 2 * D) + (size_t)nspec * 8;
    if (dispersion) need += (size_t)nvox * 4 + (size_t)nspec * 8;
    need += (size_t)nspec * 4 * (dispersion ? 2 : 1);
    need += (size_t)nvox * 4 * ((r_arr ? 1 : 0) + (c_arr ? 1 : 0) + ((nonlinear && (b_arr || r_arr)) ? 1 : 0));
    // FP64 staging during set-up (released once the simulation is created)
    if (c_arr || r_arr || b_arr || P->p0.count)
      need += (size_t)nvox * 8 * (((nonlinear && b_arr && r_arr) ? 2 : 1) + ((P->row_major && D > 1) ? 1 : 0));
  }
  for (int g = 0; g < P->n_groups; ++g) {
    const kwb_sensor_group &G = P->groups[g];
    if (G.cartesian) continue;
    const long long n = G.dense ? nvox : G.n_index;
    for (int f = 0; f < KWB_REC_COUNT; ++f)
      if (G.record_mask & (1u << f)) {
        const bool series = f == KWB_REC_P || f == KWB_REC_UX || f == KWB_REC_UY || f == KWB_REC_UZ;
        need += (size_t)n * (series ? (size_t)P->Nt * 4 : 8);
      }
  }
  if (P->n_p_index > 0) need += (size_t)P->p_signal.n_rows * P->p_signal.n_cols * 12;
  for (int d = 0; d < 3; ++d)
    if (P->u_signal[d].data) need += (size_t)P->u_signal[d].n_rows * P->u_signal[d].n_cols * 12;
  if (P->tr.data) need += (size_t)P->tr.n_rows * P->tr.n_cols * 12;
  return need + (size_t)16 * 1024 * 1024;  // per-axis tables, CSR lists, descriptor, slack
}

// =============================================================================================
// C ABI
// =============================================================================================

extern "C" {

int kwb_version(void) { return KWB_VERSION; }

int kwb_context_create(int device, kwb_ctx **out) {
  if (!out) return KWB_E_INVALID;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    g_create_err = std::string("no CUDA device available: ") + cudaGetErrorString(e);
    return KWB_E_DEVICE;
  }
  if (device < 0 || device >= n) {
    g_create_err = "device ordinal out of range";
    return KWB_E_INVALID;
  }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    g_create_err = cudaGetErrorString(e);
    return KWB_E_DEVICE;
  }
  if (prop.major != 10) {
    g_create_err = "libkwb is built for sm_100a (B200); device is sm_" + std::to_string(prop.major) +
                   std::to_string(prop.minor);
    return KWB_E_UNSUPPORTED;
  }
  kwb_ctx *ctx = new kwb_ctx();
  ctx->device = device;
  *out = ctx;
  return KWB_OK;
}

void kwb_context_destroy(kwb_ctx *ctx) {
  if (!ctx) return;
  kwb_server_shutdown(ctx);
  delete ctx;
}

const char *kwb_last_error(const kwb_ctx *ctx) {
  return ctx ? ctx->err.c_str() : g_create_err.c_str();
}

int kwb_query_outputs(kwb_ctx *ctx, const kwb_problem *P, kwb_group_sizes *sizes,
                      int64_t *p_final_full_len) {
  int rc = validate_problem(ctx, P);
  if (rc) return rc;
  long long nvox = 1;
  for (int a = 0; a < P->ndim; ++a) nvox *= P->N[a];
  for (int g = 0; g < P->n_groups; ++g) group_sizes(P, P->groups[g], nvox, sizes[g]);
  if (p_final_full_len) *p_final_full_len = P->tr.data ? nvox : 0;
  return KWB_OK;
}

// Capture KWB_CHUNK_STEPS steps (plus the device step-counter advance) as one CUDA graph that
// is replayed for every full chunk.
static int build_chunk_graph(kwb_sim *S) {
  kwb_ctx *ctx = S->ctx;
  const int K = KWB_CHUNK_STEPS;
  cudaGraph_t g;
  CU(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < K && e == cudaSuccess; ++s) e = enqueue_step(S, s);
  if (e == cudaSuccess) e = launch_advance_t0(S->d_t0, K, S->stream);
  cudaError_t e2 = cudaStreamEndCapture(S->stream, &g);
  if (e != cudaSuccess) return set_err(ctx, KWB_E_DEVICE, "graph capture: %s", cudaGetErrorString(e));
  CU(e2);
  e = cudaGraphInstantiate(&S->graph, g, 0);
  cudaGraphDestroy(g);
  CU(e);
  S->graph_K = K;
  return KWB_OK;
}

// ---- FFT schedule cache: key (device, library version, shape and the flags that select the
// kernels) -> Schedule text; in memory for the process and, unless KWB_TUNE_CACHE=none, in a text
// file (KWB_TUNE_CACHE, default $HOME/.cache/kwb/fft_schedules.txt), one "key<TAB>schedule" line each.
static std::mutex g_sched_mu;
static std::map<std::string, std::string> g_sched;
static bool g_sched_loaded = false;

static std::string sched_file() {
  const char *e = getenv("KWB_TUNE_CACHE");
  if (e && *e) return strcmp(e, "none") == 0 ? std::string() : std::string(e);
  const char *home = getenv("HOME");
  return home && *home ? std::string(home) + "/.cache/kwb/fft_schedules.txt" : std::string();
}

static void sched_load_locked() {
  if (g_sched_loaded) return;
  g_sched_loaded = true;
  const std::string path = sched_file();
  if (path.empty()) return;
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return;
  char line[1024];
  while (fgets(line, sizeof(line), f)) {
    char *tab = strchr(line, '\t');
    if (!tab) continue;
    *tab = 0;
    char *v = tab + 1;
    v[strcspn(v, "\r\n")] = 0;
    Schedule sc;
    if (schedule_parse(v, sc)) g_sched[line] = v;  // later lines win
  }
  fclose(f);
}

static void sched_store_locked(const std::string &key, const std::string &val) {
  g_sched[key] = val;
  const std::string path = sched_file();
  if (path.empty()) return;
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos && slash > 0) {  // create the directory chain
    for (size_t i = 1; i <= slash; ++i)
      if (path[i] == '/' || i == slash) mkdir(path.substr(0, i == slash ? slash : i).c_str(), 0755);
  }
  FILE *f = fopen(path.c_str(), "a");
  if (!f) return;  // an unwritable cache only costs a re-measurement in the next process
  fprintf(f, "%s\t%s\n", key.c_str(), val.c_str());
  fclose(f);
}

static std::string sched_key(int device, const SimDev &h) {
  cudaDeviceProp prop;
  char name[256] = "unknown";
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) snprintf(name, sizeof(name), "%s/%d", prop.name, prop.multiProcessorCount);
  char buf[512];
  const char *eo = getenv("KWB_TUNE_ORDER");
  snprintf(buf, sizeof(buf), "%.200s|v%d|nd%d|N%dx%dx%d|fast%d|plane%d|fuse%d|disp%d|fill%d|axi%d|rho%d|c%d|nl%d|ord%d",
           name, KWB_VERSION, h.ndim, h.N[0], h.N[1], h.N[2], h.fast, h.plane, h.fuse_xeos, h.dispersion,
           h.grid_fill, h.inv_r ? 1 : 0, h.rho0 ? 1 : 0, h.c0sq ? 1 : 0, (h.nonlinear && h.nlq) ? 2 : h.nonlinear,
           (eo && strcmp(eo, "1") == 0) ? 1 : 0);
  return buf;
}

// Pick the FFT schedule of a new simulation: KWB_TILE or KWB_TUNE=0 keep the size heuristic;
// otherwise a cached measurement of this shape, or a new one (FFTW.MEASURE's role,
// fft_utils.jl:59-60).  KWB_TUNE_PICK=i takes candidate i of every pass instead of measuring
// (tests).  Measuring runs the passes on the simulation's buffers, so its state fields are
// cleared afterwards.
static int choose_schedule(kwb_sim *S, SimDev &h, cudaStream_t st) {
  kwb_ctx *ctx = S->ctx;
  const char *tn = getenv("KWB_TUNE");
  const char *pk = getenv("KWB_TUNE_PICK");
  if (h.tile_override >= 0 || (tn && strcmp(tn, "0") == 0)) return KWB_OK;
  const int pick = pk && *pk ? atoi(pk) : -1;
  const std::string key = sched_key(ctx->device, h);
  Schedule sc;
  if (pick < 0) {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    sched_load_locked();
    auto it = g_sched.find(key);
    if (it != g_sched.end() && schedule_parse(it->second.c_str(), sc)) {
      schedule_apply(h, sc);
      S->schedule_src = "cache";
      return KWB_OK;
    }
  }
  TempBuf tmp(st, ctx->pool);
  SimDev *d_t;
  CU(tmp.alloc(&d_t, 1));
  std::string log;
  const char *eo = getenv("KWB_TUNE_ORDER");
  CU(tune_schedule(h, d_t, st, pick, eo && strcmp(eo, "1") == 0, &log));
  CU(cudaStreamSynchronize(st));
  // the measured passes wrote the state fields: back to the zero state
  const long long nvox = h.nvox;
  CU(cudaMemsetAsync(h.p, 0, nvox * 4, st));
  for (int a = 0; a < h.D; ++a) {
    CU(cudaMemsetAsync(h.u[a], 0, nvox * 4, st));
    CU(cudaMemsetAsync(h.rho[a], 0, nvox * 4, st));
  }
  if (h.spec) CU(cudaMemsetAsync(h.spec, 0, h.nspec * sizeof(float2), st));
  if (h.spec2) CU(cudaMemsetAsync(h.spec2, 0, h.nspec * sizeof(float2), st));
  if (h.rho_prev) CU(cudaMemsetAsync(h.rho_prev, 0, nvox * 4, st));
  schedule_of(h, sc);
  if (pick >= 0) {
    S->schedule_src = "pick " + std::to_string(pick);
    return KWB_OK;
  }
  S->schedule_src = "tuned";
  if (getenv("KWB_TUNE_LOG")) fprintf(stderr, "kwb tune %s: %s-> %s\n", key.c_str(), log.c_str(), schedule_str(sc).c_str());
  std::lock_guard<std::mutex> lk(g_sched_mu);
  sched_store_locked(key, schedule_str(sc));
  return KWB_OK;
}

// Set-up phase times (KWB_SETUP_LOG=1): the stream is synchronised at each mark, so the figures
// include the device work each phase queued; a diagnostic, printed to stderr.
struct SetupLog {
  bool on = false;
  cudaStream_t st = nullptr;
  std::chrono::steady_clock::time_point t0, last;
  std::string line;
  void start(cudaStream_t s) {
    const char *e = getenv("KWB_SETUP_LOG");
    on = e && strcmp(e, "1") == 0;
    st = s;
    t0 = last = std::chrono::steady_clock::now();
  }
  void mark(const char *what) {
    if (!on) return;
    cudaStreamSynchronize(st);
    const auto now = std::chrono::steady_clock::now();
    char b[96];
    snprintf(b, sizeof(b), "%s %.1f ", what, std::chrono::duration<double, std::milli>(now - last).count());
    line += b;
    last = now;
  }
  void done() {
    if (!on) return;
    mark("rest");
    fprintf(stderr, "kwb setup ms: %stotal %.1f\n", line.c_str(),
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  }
};

int kwb_sim_create(kwb_ctx *ctx, const kwb_problem *P, kwb_sim **out) {
  if (!ctx || !out) return KWB_E_INVALID;
  *out = nullptr;
  int rc = validate_problem(ctx, P);
  if (rc) return rc;
  CU(cudaSetDevice(ctx->device));
  std::unique_ptr<kwb_sim> S(new kwb_sim());
  S->ctx = ctx;
  if (!ctx->pool) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    CU(cudaMemPoolCreate(&ctx->pool, &props));
    uint64_t keep = UINT64_MAX;  // hold freed blocks for reuse until the context goes
    CU(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  CU(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
  S->mem.st = S->stream;
  S->mem.pool = ctx->pool;
  CU(cudaEventCreate(&S->ev0));
  CU(cudaEventCreate(&S->ev1));
  cudaStream_t st = S->stream;
  SimDev &h = S->h;
  DevBuf &M = S->mem;
  SetupLog slog;
  slog.start(st);

  const int D = P->ndim;
  h.ndim = D;
  h.D = D;
  for (int a = 0; a < 3; ++a) h.N[a] = a < D ? (int)P->N[a] : 1;
  h.n1 = h.N[0] / 2 + 1;
  h.nvox = (long long)h.N[0] * h.N[1] * h.N[2];
  h.nspec = (long long)h.n1 * h.N[1] * h.N[2];
  h.dt = (float)P->dt;
  const long long nvox = h.nvox;
  S->tr = P->tr.data != nullptr;
  S->Nt_grid = P->Nt;
  for (int a = 0; a < 3; ++a) S->d[a] = a < P->ndim ? P->d[a] : 1.0;
  S->dt = P->dt;
  S->Nt_loop = S->tr ? P->tr.n_cols : P->Nt;
  h.Nt = S->Nt_loop;
  h.elastic = P->elastic ? 1 : 0;

  // ---- medium scalars / flags
  const bool c_arr = P->c0.count == nvox && nvox > 1;
  const bool r_arr = P->rho0.count == nvox && nvox > 1;
  const bool b_arr = P->BonA.count == nvox && nvox > 1;
  const double c_s = P->c0.data[0];
  const double r_s = P->rho0.count ? P->rho0.data[0] : 1.0;
  // (in memory order: for row-major input the summation order differs from the reference's
  // column-major one, which changes c_ref only at FP64 round-off)
  const double c_ref = c_arr ? pairwise_sum(P->c0.data, nvox, 4) / (double)nvox : c_s;
  const bool absorbing = P->alpha_mode != KWB_NO_ABSORPTION;
  const bool nonlinear = P->BonA.count > 0;
  h.nonlinear = nonlinear;
  h.scalar_c = !c_arr;
  h.dispersion = (!c_arr && absorbing && P->alpha_mode == KWB_STOKES && !h.elastic) ? 1 : 0;
  h.dt_over_rho0_s = (float)(P->dt / r_s);
  h.dt_rho0_s = (float)(P->dt * r_s);
  h.c0sq_s = (float)(c_s * c_s);
  double tau = 0, eta = 0, y = 0;
  if (absorbing) {
    y = P->alpha_power;
    const double a_np = P->alpha_coeff * (1e-2 / (20.0 * std::log10(std::exp(1.0)))) *
                        std::pow(2.0 * kPi * 1e6, -y);
    tau = -2.0 * a_np * std::pow(c_ref, y - 1.0);
    eta = 2.0 * a_np * std::pow(c_ref, y - 1.0) * std::tan(kPi * y / 2.0);
  }

  // ---- FFT path: register-FFT kernels for power-of-two lines unless KWB_FFT_PATH=generic
  {
    const char *fp = getenv("KWB_FFT_PATH");
    h.fast = 3;  // bit 0: line passes, bit 1: equation-of-state passes
    if (fp && strcmp(fp, "generic") == 0) h.fast = 0;
    if (fp && strcmp(fp, "line") == 0) h.fast = 1;
    if (fp && strcmp(fp, "eos") == 0) h.fast = 2;
    const char *tv = getenv("KWB_TILE");
    h.tile_override = -1;
    memset(h.tile_var, -1, sizeof(h.tile_var));  // per-pass choices: the heuristic until tuned
    if (tv && strcmp(tv, "big") == 0) h.tile_override = 0;
    if (tv && strcmp(tv, "mid") == 0) h.tile_override = 1;
    if (tv && strcmp(tv, "small") == 0) h.tile_override = 2;
    if (h.elastic) h.fast &= 1;  // elastic: line passes only (no equation of state)
  }

  // ---- tile shapes and FFT plans
  CU(cudaDeviceGetAttribute(&h.num_sms, cudaDevAttrMultiProcessorCount, ctx->device));
  for (int a = 0; a < 3; ++a) plan_line(h.N[a], h.plan[a], 0);
  int FL[3];  // transform length per axis (the Bluestein inner length where there is one)
  for (int a = 0; a < 3; ++a) FL[a] = fft_len(h.plan[a]);
  h.L_line[0] = choose_L(FL[0], std::max(1, 2048 / h.N[0]), (h.N[1] + 1) / 2, 0, false);
  for (int a = 1; a < 3; ++a) h.L_line[a] = choose_L(FL[a], 8, (h.N[0] + 1) / 2, 0, false);
  h.L_eosx = choose_L(FL[0], std::max(1, 2048 / h.N[0]), (h.N[1] + 1) / 2, h.dispersion, true);
  for (int a = 1; a < 3; ++a) h.L_spec[a] = choose_L(FL[a], 8, h.n1, h.dispersion, true);
  h.L_spec[0] = 1;
  {
    // A simulation that runs alone gets narrower tiles and larger CTAs on small grids (latency:
    // 384^2 steps 2.2x faster); simulations of the batching scheduler keep full-width tiles, which
    // give more throughput when many share the GPU (64 mixed 2D sims: 29.7 vs 23.5 sims/s).
    const char *gf = getenv("KWB_GRID_FILL");
    h.grid_fill = !ctx->batched && !(gf && strcmp(gf, "0") == 0);
  }
  if (h.grid_fill) {
    // Small grids: fewer lines per tile until the shared-memory (Stockham) passes fill the GPU --
    // a 384^2 grid otherwise runs its x pass as 39 CTAs and its y spectrum pass as 25.  Strided
    // line passes stop at one wave and keep 4 complex lines (8 columns: one 32-byte sector per
    // row), since narrower tiles waste most of each sector they read.
    const long long NS = h.num_sms;
    auto shrink = [&](int &L, long long want, int floor_L, auto tiles) {
      while (L > floor_L && tiles(L) < want) L = std::max(floor_L, (L + 1) / 2);
    };
    const long long N0 = h.N[0], N1 = h.N[1], N2 = h.N[2];
    shrink(h.L_line[0], 4 * NS, 1, [&](int L) { return (N1 + 2 * L - 1) / (2 * L) * N2; });
    shrink(h.L_line[1], NS, 4, [&](int L) { return (N0 + 2 * L - 1) / (2 * L) * N2; });
    shrink(h.L_line[2], NS, 4, [&](int L) { return (N0 + 2 * L - 1) / (2 * L) * N1; });
    shrink(h.L_eosx, 4 * NS, 1, [&](int L) { return (N1 + 2 * L - 1) / (2 * L) * N2; });
    shrink(h.L_spec[1], 4 * NS, 1, [&](int L) { return (h.n1 + L - 1) / L * N2; });
    shrink(h.L_spec[2], 4 * NS, 1, [&](int L) { return (h.n1 + L - 1) / L * N1; });
  }

  // ---- admission by free device memory
  {
    const size_t need = estimate_device_bytes(P);
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b));
    uint64_t reserved = 0, used = 0;  // blocks held idle by this context's pool are free here
    CU(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    CU(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used));
    if (reserved > used) free_b += (size_t)(reserved - used);
    if (need + (size_t)64 * 1024 * 1024 > free_b)
      return set_err(ctx, KWB_E_NOMEM, "simulation needs %.1f MB of device memory, %.1f MB free",
                     need / 1e6, free_b / 1e6);
  }

  slog.mark("admission");
  // ---- fields
  CU(M.alloc(&h.err, 1));
  CU(cudaMemsetAsync(h.err, 0, sizeof(int), st));
  {
    const char *dc = getenv("KWB_TEST_DROP_TILE_COPY");
    h.test_drop_copy = dc && strcmp(dc, "1") == 0;
    // line-pass tiles by TMA copies (1) or 16-byte cp.async (0, the default): the tuner measures
    // both per pass unless KWB_TILE_TMA fixes the choice
    const char *tt = getenv("KWB_TILE_TMA");
    h.tile_tma = tt && strcmp(tt, "1") == 0;
    memset(h.tma_line, -1, sizeof(h.tma_line));
    const char *ep = getenv("KWB_EOS_PREFETCH");  // 0: no L2 prefetch of the EOS operands
    h.eos_prefetch = !(ep && strcmp(ep, "0") == 0);
  }
  CU(M.alloc(&h.p, nvox));
  CU(cudaMemsetAsync(h.p, 0, nvox * 4, st));
  for (int d = 0; d < D; ++d) {
    CU(M.alloc(&h.u[d], nvox));
    CU(cudaMemsetAsync(h.u[d], 0, nvox * 4, st));
    if (h.elastic) continue;
    CU(M.alloc(&h.rho[d], nvox));
    CU(cudaMemsetAsync(h.rho[d], 0, nvox * 4, st));
  }
  if (h.elastic) {
    for (int k = 0; k < 6; ++k) {
      if (D == 2 && (k == 2 || k > 3)) continue;  // 2-D: xx, yy, xy
      CU(M.alloc(&h.el_s[k], nvox));
      CU(M.alloc(&h.el_w[k], nvox));
      CU(cudaMemsetAsync(h.el_s[k], 0, nvox * 4, st));
    }
  } else {
    CU(M.alloc(&h.spec, h.nspec));
  }
  if (h.dispersion) {
    CU(M.alloc(&h.spec2, h.nspec));
    CU(M.alloc(&h.rho_prev, nvox));
    CU(cudaMemsetAsync(h.rho_prev, 0, nvox * 4, st));
  }
  CU(M.alloc(&S->d_t0, 1));
  CU(cudaMemsetAsync(S->d_t0, 0, 8, st));
  h.t0 = S->d_t0;

  slog.mark("fields");
  // ---- medium (FP64 upload, FP32 on device); the FP64 staging is set-up scratch only
  TempBuf tmp(st, ctx->pool);
  double *stage = nullptr, *stage2 = nullptr, *rm_in = nullptr;
  const bool need_stage = c_arr || r_arr || b_arr || P->p0.count;
  if (need_stage) CU(tmp.alloc(&stage, nvox));
  if (nonlinear && b_arr && r_arr) CU(tmp.alloc(&stage2, nvox));
  if (need_stage && P->row_major && D > 1) CU(tmp.alloc(&rm_in, nvox));
  // one grid-shaped FP64 array into column-major device staging
  auto upload_grid = [&](double *dst, const double *src) -> int {
    if (!rm_in) return upload(ctx, dst, src, nvox * 8, st);
    int r = upload(ctx, rm_in, src, nvox * 8, st);
    if (r) return r;
    CU(transpose_to_column_major(dst, rm_in, D, h.N, st));
    return KWB_OK;
  };
  if (h.elastic) {
    // lambda = rho0 (cp^2 - 2 cs^2), mu = rho0 cs^2 in FP64 (solver/elastic.jl:168-174, 419-423),
    // per voxel in the input's memory order when the density is an array (the speeds then may
    // be arrays or scalars), else scalars
    const bool cs_arr = P->cs.count == nvox && nvox > 1;
    const double cs_s = P->cs.data[0];
    if (r_arr) {
      std::vector<double> lam(nvox), mu(nvox);
      parallel_range(nvox, [&](long long lo, long long hi) {
        for (long long i = lo; i < hi; ++i) {
          const double cp = c_arr ? P->c0.data[i] : c_s, cs = cs_arr ? P->cs.data[i] : cs_s;
          const double rho = P->rho0.data[i];
          lam[i] = rho * (cp * cp - 2.0 * cs * cs);
          mu[i] = rho * (cs * cs);
        }
      });
      float *dl, *dm, *rho0;
      CU(M.alloc(&dl, nvox));
      CU(M.alloc(&dm, nvox));
      CU(M.alloc(&rho0, nvox));
      if ((rc = upload_grid(stage, lam.data()))) return rc;
      CU(convert_f64_to_f32(dl, stage, nvox, 0, st));
      if ((rc = upload_grid(stage, mu.data()))) return rc;
      CU(convert_f64_to_f32(dm, stage, nvox, 0, st));
      if ((rc = upload_grid(stage, P->rho0.data))) return rc;
      CU(convert_f64_to_f32(rho0, stage, nvox, 0, st));
      CU(cudaStreamSynchronize(st));  // the host arrays go out of scope
      h.el_lam = dl;
      h.el_mu = dm;
      h.rho0 = rho0;
    } else {
      h.el_lam_s = (float)(r_s * (c_s * c_s - 2.0 * cs_s * cs_s));
      h.el_mu_s = (float)(r_s * (cs_s * cs_s));
      // Kelvin-Voigt factors chi = 2 db2neper(alpha, y) c^(y-1), used by the 2-D homogeneous
      // branch only (elastic.jl:177-195, 282-295)
      auto chi = [&](double alpha, double c) {
        const double y = P->alpha_power;
        const double a_np = alpha * (1e-2 / (20.0 * std::log10(std::exp(1.0)))) * std::pow(2.0 * kPi * 1e6, -y);
        return 2.0 * a_np * std::pow(c, y - 1.0);
      };
      if (D == 2 && absorbing) h.el_chi_p = (float)chi(P->alpha_coeff, c_s);
      if (D == 2 && P->has_alpha_shear) h.el_chi_s = (float)chi(P->alpha_coeff_shear, cs_s);
    }
  } else {
    if (c_arr) {
      float *c0sq;
      CU(M.alloc(&c0sq, nvox));
      if ((rc = upload_grid(stage, P->c0.data))) return rc;
      CU(convert_f64_to_f32(c0sq, stage, nvox, 1, st));
      h.c0sq = c0sq;
    }
    // rho0 stays staged in FP64 for the nonlinearity term (stage2 when B/A is an array too)
    double *rho_stage = stage2 ? stage2 : stage;
    if (r_arr) {
      float *rho0;
      CU(M.alloc(&rho0, nvox));
      if ((rc = upload_grid(rho_stage, P->rho0.data))) return rc;
      CU(convert_f64_to_f32(rho0, rho_stage, nvox, 0, st));
      h.rho0 = rho0;
    }
    if (nonlinear) {
      const double b_s = P->BonA.data[0];
      if (b_arr || r_arr) {
        float *q;
        CU(M.alloc(&q, nvox));
        const double *bp = nullptr, *rp = nullptr;
        if (b_arr && r_arr) {
          if ((rc = upload_grid(stage, P->BonA.data))) return rc;
          bp = stage;
          rp = stage2;
        } else if (b_arr) {
          if ((rc = upload_grid(stage, P->BonA.data))) return rc;
          bp = stage;
        } else {
          rp = stage;
        }
        CU(build_nlq(q, bp, b_arr, b_s, rp, r_arr, r_s, nvox, st));
        h.nlq = q;
      } else {
        h.nlq_s = (float)((b_s / 2.0) / r_s);
      }
    }

  }

  slog.mark("medium");
  // ---- per-axis tables (FP64 on device)
  for (int a = 0; a < 3; ++a) {
    const int n = h.N[a];
    const int nt = fft_len(h.plan[a]);  // twiddles of the transform length
    float2 *tw, *gp, *gn;
    float *pd, *psd;
    CU(M.alloc(&tw, nt));
    CU(M.alloc(&gp, n));
    CU(M.alloc(&gn, n));
    CU(M.alloc(&pd, n));
    CU(M.alloc(&psd, n));
    CU(build_twiddles(tw, nt, st));
    if (h.plan[a].m > 0) {
      std::vector<float2> ch, chf;
      bluestein_tables(n, h.plan[a].m, ch, chf);
      float2 *dch, *dchf;
      CU(M.alloc(&dch, ch.size()));
      CU(M.alloc(&dchf, chf.size()));
      if ((rc = upload(ctx, dch, ch.data(), ch.size() * sizeof(float2), st))) return rc;
      if ((rc = upload(ctx, dchf, chf.data(), chf.size() * sizeof(float2), st))) return rc;
      h.plan[a].chirp = dch;
      h.plan[a].chirp_ft = dchf;
    }
    const double d = a < D ? P->d[a] : 1.0;
    CU(build_gradient(gp, gn, n, d, st));
    const int psz = a < D ? (int)P->pml_size[a] : 0;
    const double pal = a < D ? P->pml_alpha[a] : 0.0;
    CU(build_pml_deficit(pd, n, psz, pal, P->dt, 0, st));
    CU(build_pml_deficit(psd, n, psz, pal, P->dt, 1, st));
    h.tw[a] = tw;
    h.gpos[a] = gp;
    h.gneg[a] = gn;
    h.pml_def[a] = pd;
    h.pml_sg_def[a] = psd;
  }
  if (P->axisymmetric) {
    // 1/r on the radial axis: r = |y_vec|, y_vec = ((0:Ny-1) - (Ny-1)/2) dy, r = 0 -> dy/2
    // (grid.jl:137-139, axisymmetric.jl:100-103); FP64, rounded once
    std::vector<float> ir(h.N[1]);
    for (int j = 0; j < h.N[1]; ++j) {
      double r = std::fabs((j - (h.N[1] - 1) / 2.0) * P->d[1]);
      if (r == 0.0) r = P->d[1] / 2.0;
      ir[j] = (float)(1.0 / r);
    }
    float *dir;
    CU(M.alloc(&dir, h.N[1]));
    if ((rc = upload(ctx, dir, ir.data(), ir.size() * sizeof(float), st))) return rc;
    h.inv_r = dir;
  }
  {
    // 3-D y/z transforms in one cluster pass per kx plane (KWB_PLANE=0 keeps separate passes)
    const char *pv = getenv("KWB_PLANE");
    h.plane = (h.fast & 2) && D == 3 && !h.dispersion && fast_size(h.N[0]) && fast_plane_size(h.N[1], h.N[2]) &&
              !(pv && strcmp(pv, "0") == 0) && fast_plane_available();
    // the x line pass carries the EOS x R2C when both run on the register-FFT kernels
    // (KWB_FUSE_XEOS=0 keeps them separate)
    const char *fx = getenv("KWB_FUSE_XEOS");
    h.fuse_xeos = (h.fast & 3) == 3 && D >= 2 && !h.dispersion && fast_size(h.N[0]) && !(fx && strcmp(fx, "0") == 0);
  }
  // The EOS multiplier: allocated here, built once the FFT schedule is known, since the plane
  // pass's slot-major variants read it in their own layout (the tuner's timing launches only
  // need the buffer).
  int *slot_ky = nullptr, *slot_kz = nullptr;
  if (!h.elastic) {
    float *Mt, *M2 = nullptr;
    CU(M.alloc(&Mt, h.nspec));
    if (h.dispersion) CU(M.alloc(&M2, h.nspec));
    if (h.plane) {
      std::vector<int> ky(h.N[1]), kz(h.N[2]);
      fast_plane_slot_ky(h.N[1], ky.data());
      fast_plane_slot_kz(h.N[2], kz.data());
      CU(M.alloc(&slot_ky, h.N[1]));
      CU(M.alloc(&slot_kz, h.N[2]));
      if ((rc = upload(ctx, slot_ky, ky.data(), ky.size() * sizeof(int), st))) return rc;
      if ((rc = upload(ctx, slot_kz, kz.data(), kz.size() * sizeof(int), st))) return rc;
    }
    h.M = Mt;
    h.M2 = M2;
  }

  slog.mark("tables");
  // ---- sources
  auto c_at_points = [&](const int64_t *idx, long long n, double **dev_out) -> int {
    *dev_out = nullptr;
    if (!c_arr || n == 0) return KWB_OK;
    std::vector<double> c(n);
    const long long Nx = h.N[0], Ny = h.N[1], Nz = h.N[2];
    for (long long j = 0; j < n; ++j) {
      long long k = idx[j];  // column-major linear index
      if (P->row_major && D > 1) {
        const long long x = k % Nx, y = (k / Nx) % Ny, z = k / (Nx * Ny);
        k = D == 3 ? (x * Ny + y) * Nz + z : x * Ny + y;
      }
      c[j] = P->c0.data[k];
    }
    double *dc;
    CU(M.alloc(&dc, n));
    if (int r = upload(ctx, dc, c.data(), n * 8, st)) return r;
    CU(cudaStreamSynchronize(st));
    *dev_out = dc;
    return KWB_OK;
  };
  if (P->n_p_index > 0) {
    const long long n = P->n_p_index;
    h.n_p = (int)n;
    h.p_mode = P->p_mode;
    h.p_cols = (int)P->p_signal.n_cols;
    double *sig;
    CU(M.alloc(&sig, P->p_signal.n_rows * P->p_signal.n_cols));
    if ((rc = upload(ctx, sig, P->p_signal.data, P->p_signal.n_rows * P->p_signal.n_cols * 8, st))) return rc;
    double *cat;
    if ((rc = c_at_points(P->p_index, n, &cat))) return rc;
    float *tab;
    CU(M.alloc(&tab, n * h.p_cols));
    CU(build_source_table(tab, sig, P->p_signal.n_rows, n, h.p_cols, cat, c_s, c_arr, (double)D, 1, st));
    h.p_sig = tab;
    for (int a = 0; a < D; ++a) {
      std::vector<int> ptr;
      std::vector<SrcEntry> ent;
      build_csr(P->p_index, n, h.N, a, ptr, ent);
      int *dptr;
      SrcEntry *dent;
      CU(M.alloc(&dptr, ptr.size()));
      CU(M.alloc(&dent, ent.size()));
      if ((rc = upload(ctx, dptr, ptr.data(), ptr.size() * 4, st))) return rc;
      if ((rc = upload(ctx, dent, ent.data(), ent.size() * sizeof(SrcEntry), st))) return rc;
      CU(cudaStreamSynchronize(st));
      h.p_line_ptr[a] = dptr;
      h.p_entry[a] = dent;
    }
  }
  if (P->n_u_index > 0) {
    const long long n = P->n_u_index;
    h.n_u = (int)n;
    h.u_mode = P->u_mode;
    for (int a = 0; a < D; ++a) {
      const kwb_signal &sg = P->u_signal[a];
      if (!sg.data) continue;
      h.u_cols[a] = (int)sg.n_cols;
      double *sig;
      CU(M.alloc(&sig, sg.n_rows * sg.n_cols));
      if ((rc = upload(ctx, sig, sg.data, sg.n_rows * sg.n_cols * 8, st))) return rc;
      float *tab;
      CU(M.alloc(&tab, n * sg.n_cols));
      CU(build_source_table(tab, sig, sg.n_rows, n, sg.n_cols, nullptr, 1.0, 0, 1.0, 0, st));
      h.u_sig[a] = tab;
      if (h.elastic) continue;  // injected at point lists (below), not inside line passes
      std::vector<int> ptr;
      std::vector<SrcEntry> ent;
      build_csr(P->u_index, n, h.N, a, ptr, ent);
      int *dptr;
      SrcEntry *dent;
      CU(M.alloc(&dptr, ptr.size()));
      CU(M.alloc(&dent, ent.size()));
      if ((rc = upload(ctx, dptr, ptr.data(), ptr.size() * 4, st))) return rc;
      if ((rc = upload(ctx, dent, ent.data(), ent.size() * sizeof(SrcEntry), st))) return rc;
      CU(cudaStreamSynchronize(st));
      h.u_line_ptr[a] = dptr;
      h.u_entry[a] = dent;
    }
  }

  if (h.elastic && P->n_u_index > 0) {
    long long *di;
    CU(M.alloc(&di, P->n_u_index));
    if ((rc = upload(ctx, di, P->u_index, P->n_u_index * 8, st))) return rc;
    h.u_idx = di;
  }
  if (h.elastic && P->n_s_index > 0) {
    const long long n = P->n_s_index;
    h.n_s = (int)n;
    h.s_mode = P->s_mode;
    long long *di;
    CU(M.alloc(&di, n));
    if ((rc = upload(ctx, di, P->s_index, n * 8, st))) return rc;
    h.s_idx = di;
    for (int k = 0; k < 6; ++k) {
      const kwb_signal &sg = P->s_signal[k];
      if (!sg.data || !h.el_s[k]) continue;
      h.s_cols[k] = (int)sg.n_cols;
      double *sig;
      CU(M.alloc(&sig, sg.n_rows * sg.n_cols));
      if ((rc = upload(ctx, sig, sg.data, sg.n_rows * sg.n_cols * 8, st))) return rc;
      float *tab;
      CU(M.alloc(&tab, n * sg.n_cols));
      CU(build_source_table(tab, sig, sg.n_rows, n, sg.n_cols, nullptr, 1.0, 0, 1.0, 0, st));
      h.s_sig[k] = tab;
    }
    CU(cudaStreamSynchronize(st));
  }

  slog.mark("sources");
  // ---- sensor groups
  S->groups.resize(P->n_groups);
  // Pressure-only groups can be recorded by the fast x C2R pass as it writes p: one dense group
  // (every voxel) and one sparse group (through a per-x-line index of its points).
  const unsigned ponly = (1u << KWB_REC_P) | (1u << KWB_REC_P_MAX) | (1u << KWB_REC_P_MIN) |
                         (1u << KWB_REC_P_RMS) | (1u << KWB_REC_P_FINAL);
  const bool fast_inv = (h.fast & 2) && h.ndim >= 2 && !h.dispersion && fast_size(h.N[0]);
  bool sparse_taken = false;
  for (int g = 0; g < P->n_groups; ++g) {
    GroupHost &G = S->groups[g];
    G.spec = P->groups[g];
    G.spec.index = nullptr;
    G.spec.directivity_angle = nullptr;  // copied below: the caller's array may not outlive the call
    if (G.spec.cartesian) continue;
    const kwb_sensor_group &in = P->groups[g];
    G.n = in.dense ? nvox : in.n_index;
    if (!h.elastic && (in.record_mask & (1u << KWB_REC_P)) && G.n > 0 &&
        (in.directivity_angle || in.has_frequency_response)) {
      // one filter per distinct directivity angle (angle 0: no directivity for that point)
      std::map<double, int> ids;
      G.filt_of.resize(G.n);
      for (long long j = 0; j < G.n; ++j) {
        double th = 0.0;
        if (in.directivity_angle) th = in.directivity_angle[in.n_directivity_angle == 1 ? 0 : j];
        auto it = ids.find(th);
        if (it == ids.end()) {
          it = ids.emplace(th, (int)G.filt_sin.size()).first;
          G.filt_sin.push_back(th == 0.0 ? NAN : std::sin(th));
        }
        G.filt_of[j] = it->second;
      }
    }
    GroupDev &gd = G.dev;
    gd.n = G.n;
    gd.dense = in.dense;
    gd.mask = in.record_mask;
    gd.cnt_prms = std::max<int>(1, in.record_count[KWB_REC_P_RMS]);
    gd.cnt_urms = std::max<int>(1, in.record_count[KWB_REC_U_RMS]);
    gd.cnt_iavg = std::max<int>(1, in.record_count[KWB_REC_I_AVG]);
    gd.nt_alloc = P->Nt;
    if (G.n == 0) continue;
    if (!in.dense) {
      long long *di;
      CU(M.alloc(&di, G.n));
      if ((rc = upload(ctx, di, in.index, G.n * 8, st))) return rc;
      CU(cudaStreamSynchronize(st));
      gd.idx = di;
    }
    const unsigned m = in.record_mask;
    if (m & (1u << KWB_REC_P)) {
      CU(M.alloc(&gd.ser_p, G.n * P->Nt));
      CU(cudaMemsetAsync(gd.ser_p, 0, G.n * P->Nt * 4, st));
    }
    for (int d = 0; d < 3; ++d)
      if (m & (1u << (KWB_REC_UX + d))) {
        CU(M.alloc(&gd.ser_u[d], G.n * P->Nt));
        CU(cudaMemsetAsync(gd.ser_u[d], 0, G.n * P->Nt * 4, st));
      }
    if (m & (1u << KWB_REC_P_MAX)) { CU(M.alloc(&gd.pmax, G.n)); if ((rc = fill_f32(ctx, gd.pmax, G.n, -INFINITY, st))) return rc; }
    if (m & (1u << KWB_REC_P_MIN)) { CU(M.alloc(&gd.pmin, G.n)); if ((rc = fill_f32(ctx, gd.pmin, G.n, INFINITY, st))) return rc; }
    if (m & (1u << KWB_REC_P_FINAL)) { CU(M.alloc(&gd.pfinal, G.n)); if ((rc = fill_f32(ctx, gd.pfinal, G.n, 0.f, st))) return rc; }
    if (m & (1u << KWB_REC_P_RMS)) { CU(M.alloc(&gd.prms, G.n)); if ((rc = fill_f64(ctx, gd.prms, G.n, 0.0, st))) return rc; }
    if (m & (1u << KWB_REC_U_MAX)) { CU(M.alloc(&gd.umax, G.n)); if ((rc = fill_f64(ctx, gd.umax, G.n, -INFINITY, st))) return rc; }
    if (m & (1u << KWB_REC_U_RMS)) { CU(M.alloc(&gd.urms, G.n)); if ((rc = fill_f64(ctx, gd.urms, G.n, 0.0, st))) return rc; }
    if (m & (1u << KWB_REC_U_FINAL)) { CU(M.alloc(&gd.ufinal, G.n)); if ((rc = fill_f64(ctx, gd.ufinal, G.n, 0.0, st))) return rc; }
    if (m & (1u << KWB_REC_I_AVG)) { CU(M.alloc(&gd.iavg, G.n)); if ((rc = fill_f64(ctx, gd.iavg, G.n, 0.0, st))) return rc; }
    if (m & (1u << KWB_REC_I_MAX)) { CU(M.alloc(&gd.imax, G.n)); if ((rc = fill_f64(ctx, gd.imax, G.n, -INFINITY, st))) return rc; }
    if (fast_inv && !S->tr && !in.dense && !sparse_taken && !(m & ~ponly)) {
      // per-x-line index of the points: the sorted column-major indices are sorted by line, then x
      const long long Nx = h.N[0], nlines = (long long)h.N[1] * h.N[2];
      std::vector<int> ptr(nlines + 1, 0);
      std::vector<int2> ent(G.n);
      for (long long j = 0; j < G.n; ++j) {
        const long long v = in.index[j];
        ptr[v / Nx + 1]++;
        ent[j] = make_int2((int)(v % Nx), (int)j);
      }
      for (long long k = 0; k < nlines; ++k) ptr[k + 1] += ptr[k];
      int *dptr;
      int2 *dent;
      CU(M.alloc(&dptr, ptr.size()));
      CU(M.alloc(&dent, ent.size()));
      if ((rc = upload(ctx, dptr, ptr.data(), ptr.size() * sizeof(int), st))) return rc;
      if ((rc = upload(ctx, dent, ent.data(), ent.size() * sizeof(int2), st))) return rc;
      gd.line_ptr = dptr;
      gd.line_ent = dent;
      G.fused = true;
      sparse_taken = true;
    }
    CU(M.alloc(&G.d_dev, 1));
    if ((rc = upload(ctx, G.d_dev, &gd, sizeof(GroupDev), st))) return rc;
    CU(cudaStreamSynchronize(st));
    if (G.fused) h.sparse_p = G.d_dev;
  }

  slog.mark("sensors");
  // ---- time reversal data: p / (D c^2) at group 0's points
  if (S->tr) {
    const kwb_sensor_group &G0 = P->groups[0];
    const long long n = G0.cartesian ? 0 : (G0.dense ? nvox : G0.n_index);
    h.n_tr = (int)n;
    if (n > 0) {
      std::vector<int64_t> idx;
      const int64_t *ip = G0.index;
      if (G0.dense) {
        idx.resize(n);
        for (long long j = 0; j < n; ++j) idx[j] = j;
        ip = idx.data();
      }
      long long *di;
      CU(M.alloc(&di, n));
      if ((rc = upload(ctx, di, ip, n * 8, st))) return rc;
      double *sig;
      CU(M.alloc(&sig, P->tr.n_rows * P->tr.n_cols));
      if ((rc = upload(ctx, sig, P->tr.data, P->tr.n_rows * P->tr.n_cols * 8, st))) return rc;
      double *cat;
      if ((rc = c_at_points(ip, n, &cat))) return rc;
      float *tab;
      CU(M.alloc(&tab, n * P->tr.n_cols));
      CU(build_source_table(tab, sig, P->tr.n_rows, n, P->tr.n_cols, cat, c_s, c_arr, (double)D, 1, st));
      h.tr_idx = di;
      h.tr_sig = tab;
      CU(cudaStreamSynchronize(st));
    }
  }

  // ---- a dense pressure-only sensor group is updated inside the fast x C2R pass
  {
    for (auto &G : S->groups) {
      if (!fast_inv || G.spec.cartesian || !G.dev.dense || G.n == 0 || (G.dev.mask & ~ponly)) continue;
      h.dense_p = G.d_dev;
      G.fused = true;
      break;
    }
  }
  CU(h.elastic ? el_prime(h) : prime_attributes(h));

  slog.mark("tr+dense");
  // ---- FFT schedule: measured on first use of this shape (simulations of the batching
  // scheduler share the GPU with others, so they keep the heuristic)
  if (!h.elastic && !ctx->batched && S->Nt_loop > 0) {
    if ((rc = choose_schedule(S.get(), h, st))) return rc;
    CU(prime_attributes(h));
  }
  if (!h.elastic) {
    // [kz][ky][kx]; with the plane pass [kx][kz][slot], or [kx][slot][k_z in register order]
    // for its slot-major variants
    const double d3[3] = {P->d[0], D > 1 ? P->d[1] : 1.0, D > 2 ? P->d[2] : 1.0};
    CU(build_eos_multiplier(const_cast<float *>(h.M), const_cast<float *>(h.M2), h.N, d3, c_ref, P->dt,
                            c_arr ? 1.0 : c_s * c_s, absorbing, tau, eta, y, h.plane ? slot_ky : nullptr,
                            fast_plane_slot_major(h) ? slot_kz : nullptr, st));
  }

  slog.mark("schedule");
  // ---- device descriptor
  CU(M.alloc(&S->d_sim, 1));
  if ((rc = upload(ctx, S->d_sim, &h, sizeof(SimDev), st))) return rc;

  slog.mark("descriptor");
  // ---- p0 initialisation (first_order_steps.jl:58-191); skipped in time-reversal mode
  if (P->p0.count && !S->tr) {
    if ((rc = upload_grid(stage, P->p0.data))) return rc;
    CU(convert_f64_to_f32(h.p, stage, nvox, 0, st));
    if (h.elastic) {
      CU(el_init(h, st));  // every normal stress = -p0 (elastic.jl:211-215, 441-446)
    } else {
      for (int a = 0; a < D; ++a) CU(launch_line_pass(S->d_sim, h, a, KWB_MODE_INIT, 0, st));
    }
  }
  CU(cudaStreamSynchronize(st));

  S->progress = P->progress;
  S->progress_user = P->progress_user;
  if (S->progress) CU(cudaMallocHost(&S->p_host, nvox * 4));
  S->launches_per_step = count_launches(S.get());
  slog.done();
  *out = S.release();
  return KWB_OK;
}

static int sim_enqueue(kwb_sim *S, long long steps) {
  kwb_ctx *ctx = S->ctx;
  CU(cudaSetDevice(ctx->device));
  const long long remaining = S->Nt_loop - S->steps_done;
  if (steps > remaining) steps = remaining;
  if (steps <= 0) return KWB_OK;
  if (S->progress) {
    for (long long i = 0; i < steps; ++i) {
      const long long t = S->steps_done;
      CU(enqueue_step(S, t - S->t0_host));
      CU(cudaMemcpyAsync(S->p_host, S->h.p, S->h.nvox * 4, cudaMemcpyDeviceToHost, S->stream));
      CU(cudaStreamSynchronize(S->stream));
      S->steps_done++;
      S->progress(t + 1, S->Nt_loop, S->p_host, S->progress_user);
    }
    return KWB_OK;
  }
  if (steps >= KWB_CHUNK_STEPS && !S->graph) {
    const int rc = build_chunk_graph(S);
    if (rc) return rc;
  }
  // steps launched one by one index from the device counter t0 (step_s = steps_done - t0_host);
  // a graph chunk indexes from t0 itself, so t0 first catches up with them
  if (S->graph && steps >= S->graph_K && S->t0_host != S->steps_done) {
    CU(launch_advance_t0(S->d_t0, S->steps_done - S->t0_host, S->stream));
    S->t0_host = S->steps_done;
  }
  while (S->graph && steps >= S->graph_K) {
    CU(cudaGraphLaunch(S->graph, S->stream));
    S->t0_host += S->graph_K;
    S->steps_done += S->graph_K;
    steps -= S->graph_K;
  }
  for (long long i = 0; i < steps; ++i) {
    CU(enqueue_step(S, S->steps_done - S->t0_host));
    S->steps_done++;
  }
  return KWB_OK;
}

int kwb_sim_advance(kwb_sim *S, int64_t steps) {
  if (!S) return KWB_E_INVALID;
  return sim_enqueue(S, steps);
}

// The device error word: set by a kernel whose bounded wait gave up (a tile copy into shared
// memory that did not complete in its time budget).  Read after the stream is synchronised.
static int check_device_err(kwb_sim *S) {
  if (!S->h.err) return KWB_OK;
  kwb_ctx *ctx = S->ctx;
  int e = 0;
  CU(cudaMemcpy(&e, S->h.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e)
    return set_err(ctx, KWB_E_DEVICE,
                   "a device-side wait gave up: a tile copy into shared memory did not complete within "
                   "its time budget (error word %d)", e);
  return KWB_OK;
}

int kwb_sim_advance_timed(kwb_sim *S, int64_t steps, double *device_ms) {
  if (!S) return KWB_E_INVALID;
  kwb_ctx *ctx = S->ctx;
  CU(cudaSetDevice(ctx->device));
  // capture the replayed chunk first, so that the timed interval holds device work only
  if (!S->progress && !S->graph && steps >= KWB_CHUNK_STEPS && S->Nt_loop - S->steps_done >= KWB_CHUNK_STEPS) {
    const int rc = build_chunk_graph(S);
    if (rc) return rc;
  }
  CU(cudaEventRecord(S->ev0, S->stream));
  int rc = sim_enqueue(S, steps);
  if (rc) return rc;
  CU(cudaEventRecord(S->ev1, S->stream));
  CU(cudaEventSynchronize(S->ev1));
  float ms = 0;
  CU(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
  if (device_ms) *device_ms = ms;
  return check_device_err(S);
}

int64_t kwb_sim_steps_done(const kwb_sim *S) { return S ? S->steps_done : -1; }

int kwb_sim_sync(kwb_sim *S) {
  if (!S) return KWB_E_INVALID;
  kwb_ctx *ctx = S->ctx;
  CU(cudaStreamSynchronize(S->stream));
  return check_device_err(S);
}

int kwb_sim_read_pressure(kwb_sim *S, float *p_host) {
  if (!S || !p_host) return KWB_E_INVALID;
  kwb_ctx *ctx = S->ctx;
  CU(cudaSetDevice(ctx->device));
  CU(cudaMemcpyAsync(p_host, S->h.p, S->h.nvox * 4, cudaMemcpyDeviceToHost, S->stream));
  CU(cudaStreamSynchronize(S->stream));
  return KWB_OK;
}

// The reference's post-loop filters (first_order_steps.jl:836-910) on the device series of
// group G, in place, before it is read back.  Applied once: the filters are cleared after.
static int apply_post_filters(kwb_sim *S, GroupHost &G) {
  kwb_ctx *ctx = S->ctx;
  cudaStream_t st = S->stream;
  const int Nt = (int)G.dev.nt_alloc;
  const int nf = (int)G.filt_sin.size();
  const long long n = G.n;
  const SimDev &h = S->h;
  double dmin = h.ndim == 1 ? S->d[0] : std::min(S->d[0], S->d[1]);
  if (h.ndim == 3) dmin = std::min(dmin, S->d[2]);
  TempBuf tmp(st, ctx->pool);
  float *hk, *out;
  double *H, *cosT, *sinv;
  int *fid;
  CU(tmp.alloc(&hk, (size_t)nf * Nt));
  CU(tmp.alloc(&H, (size_t)nf * Nt));
  CU(tmp.alloc(&cosT, Nt));
  CU(tmp.alloc(&sinv, nf));
  CU(tmp.alloc(&fid, n));
  CU(tmp.alloc(&out, (size_t)n * Nt));
  CU(cudaMemcpyAsync(sinv, G.filt_sin.data(), nf * sizeof(double), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(fid, G.filt_of.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
  CU(filter_build_kernels(hk, H, cosT, Nt, nf, sinv, G.spec.directivity_size, dmin, S->dt, G.spec.has_frequency_response,
                          G.spec.frequency_center, G.spec.frequency_bandwidth, st));
  CU(filter_apply(out, G.dev.ser_p, hk, fid, Nt, n, st));
  CU(cudaMemcpyAsync(G.dev.ser_p, out, (size_t)n * Nt * sizeof(float), cudaMemcpyDeviceToDevice, st));
  CU(cudaStreamSynchronize(st));  // the host vectors above are read by the copies
  G.filt_sin.clear();
  G.filt_of.clear();
  return KWB_OK;
}

}  // extern "C"

// Read a simulation's outputs into the caller's arrays; the first row0 time rows of every time
// series are already there (kwb_solve streams them while later steps run).
static int read_outputs_from(kwb_sim *S, kwb_outputs *out, long long row0) {
  if (!S || !out) return KWB_E_INVALID;
  kwb_ctx *ctx = S->ctx;
  CU(cudaSetDevice(ctx->device));
  CU(cudaStreamSynchronize(S->stream));
  if (const int erc = check_device_err(S)) return erc;
  const double Ntd = (double)S->Nt_loop;
  for (size_t g = 0; g < S->groups.size(); ++g) {
    if (!out->groups) break;
    const GroupHost &G = S->groups[g];
    kwb_group_outputs &o = out->groups[g];
    const unsigned m = G.spec.record_mask;
    const long long n = G.spec.cartesian ? G.spec.n_index : G.n;
    auto want = [&](int f) { return (m & (1u << f)) && o.field[f]; };
    if (G.spec.cartesian || n == 0) {
      // never filled: initial values (first_order.jl:417-421, sensor.jl:109-133)
      for (int f = 0; f < KWB_REC_COUNT; ++f) {
        if (!want(f)) continue;
        const bool series = f == KWB_REC_P || f == KWB_REC_UX || f == KWB_REC_UY || f == KWB_REC_UZ;
        const long long cnt = series ? n * S->Nt_grid : n;
        double v = 0.0;
        if (f == KWB_REC_P_MAX || f == KWB_REC_U_MAX || f == KWB_REC_I_MAX) v = -INFINITY;
        if (f == KWB_REC_P_MIN) v = INFINITY;
        for (long long i = 0; i < cnt; ++i) o.field[f][i] = v;
      }
      continue;
    }
    const GroupDev &gd = G.dev;
    auto get32 = [&](const float *src, long long cnt, double *dst) -> int {
      return read_f32_as_f64(ctx, S->stream, src, cnt, dst);
    };
    auto get64 = [&](const double *src, long long cnt, double *dst) -> int {
      CU(cudaMemcpyAsync(dst, src, cnt * 8, cudaMemcpyDeviceToHost, S->stream));
      CU(cudaStreamSynchronize(S->stream));
      return KWB_OK;
    };
    auto rms = [&](double *a) {  // sqrt(sum / Nt), the reference's p_rms / u_rms
      parallel_range(n, [a, Ntd](long long lo, long long hi) {
        for (long long i = lo; i < hi; ++i) a[i] = std::sqrt(a[i] / Ntd);
      });
    };
    int rc;
    if (want(KWB_REC_P) && !G.filt_sin.empty() && (rc = apply_post_filters(S, S->groups[g]))) return rc;
    const long long r0 = std::min(row0, gd.nt_alloc), rows = gd.nt_alloc - r0;
    if (want(KWB_REC_P) && (rc = get32(gd.ser_p + r0 * n, n * rows, o.field[KWB_REC_P] + r0 * n))) return rc;
    for (int d = 0; d < 3; ++d)
      if (want(KWB_REC_UX + d) && (rc = get32(gd.ser_u[d] + r0 * n, n * rows, o.field[KWB_REC_UX + d] + r0 * n)))
        return rc;
    if (want(KWB_REC_P_MAX) && (rc = get32(gd.pmax, n, o.field[KWB_REC_P_MAX]))) return rc;
    if (want(KWB_REC_P_MIN) && (rc = get32(gd.pmin, n, o.field[KWB_REC_P_MIN]))) return rc;
    if (want(KWB_REC_P_FINAL) && (rc = get32(gd.pfinal, n, o.field[KWB_REC_P_FINAL]))) return rc;
    if (want(KWB_REC_P_RMS)) {
      if ((rc = get64(gd.prms, n, o.field[KWB_REC_P_RMS]))) return rc;
      rms(o.field[KWB_REC_P_RMS]);
    }
    if (want(KWB_REC_U_MAX) && (rc = get64(gd.umax, n, o.field[KWB_REC_U_MAX]))) return rc;
    if (want(KWB_REC_U_RMS)) {
      if ((rc = get64(gd.urms, n, o.field[KWB_REC_U_RMS]))) return rc;
      rms(o.field[KWB_REC_U_RMS]);
    }
    if (want(KWB_REC_U_FINAL) && (rc = get64(gd.ufinal, n, o.field[KWB_REC_U_FINAL]))) return rc;
    if (want(KWB_REC_I_AVG) && (rc = get64(gd.iavg, n, o.field[KWB_REC_I_AVG]))) return rc;
    if (want(KWB_REC_I_MAX) && (rc = get64(gd.imax, n, o.field[KWB_REC_I_MAX]))) return rc;
  }
  if (S->tr && out->p_final_full) {
    const int rc = read_f32_as_f64(ctx, S->stream, S->h.p, S->h.nvox, out->p_final_full);
    if (rc) return rc;
  }
  return KWB_OK;
}

// Time-series rows [r0, r1) of every recorded series into the caller's arrays, on stream cs
// (ordered after the steps that wrote them by the caller).  Series rows are written once, by the
// step of the same index, and post-loop filters are not pending (streamable).
static int copy_series_rows(kwb_sim *S, kwb_outputs *out, long long r0, long long r1, cudaStream_t cs) {
  for (size_t g = 0; g < S->groups.size(); ++g) {
    const GroupHost &G = S->groups[g];
    kwb_group_outputs &o = out->groups[g];
    const long long n = G.n;
    if (G.spec.cartesian || n == 0) continue;
    const GroupDev &gd = G.dev;
    const long long a = std::min(r0, gd.nt_alloc), b = std::min(r1, gd.nt_alloc);
    if (b <= a) continue;
    const float *src[4] = {gd.ser_p, gd.ser_u[0], gd.ser_u[1], gd.ser_u[2]};
    const int fld[4] = {KWB_REC_P, KWB_REC_UX, KWB_REC_UY, KWB_REC_UZ};
    for (int k = 0; k < 4; ++k) {
      if (!(G.spec.record_mask & (1u << fld[k])) || !o.field[fld[k]] || !src[k]) continue;
      const int rc = read_f32_as_f64(S->ctx, cs, src[k] + a * n, (b - a) * n, o.field[fld[k]] + a * n);
      if (rc) return rc;
    }
  }
  return KWB_OK;
}

// kwb_solve streams the time series back while the loop runs: no progress callback, no time
// reversal, no elastic solver and no post-loop filters (which rewrite the series at the end).
static bool series_streamable(const kwb_sim *S, const kwb_outputs *out) {
  if (!out || !out->groups || S->progress || S->tr || S->h.elastic) return false;
  for (const GroupHost &G : S->groups)
    if (!G.filt_sin.empty()) return false;
  return true;
}

extern "C" {

int kwb_sim_read_outputs(kwb_sim *S, kwb_outputs *out) { return read_outputs_from(S, out, 0); }

void kwb_sim_destroy(kwb_sim *S) {
  if (!S) return;
  cudaSetDevice(S->ctx->device);
  if (S->stream) cudaStreamSynchronize(S->stream);
  delete S;
}

}  // extern "C"

extern "C" int kwb_sim_schedule(const kwb_sim *S, char *buf, int64_t len) {
  if (!S || !buf || len <= 0) return KWB_E_INVALID;
  Schedule sc;
  schedule_of(S->h, sc);
  snprintf(buf, (size_t)len, "%s: %s", S->schedule_src.c_str(), schedule_str(sc).c_str());
  return KWB_OK;
}

// accessors for the serving scheduler (kwb_serve.cu)
cudaStream_t kwb_sim_stream_of(kwb_sim *S) { return S->stream; }
long long kwb_sim_nt_of(const kwb_sim *S) { return S->Nt_loop; }
void kwb_ctx_set_err(kwb_ctx *ctx, const char *msg) { ctx->err = msg ? msg : ""; }
void kwb_ctx_set_batched(kwb_ctx *ctx) { ctx->batched = true; }
int kwb_ctx_device(const kwb_ctx *ctx) { return ctx->device; }
KwbServer *&kwb_ctx_server_slot(kwb_ctx *ctx) { return ctx->server; }

extern "C" {

int kwb_estimate_device_bytes(kwb_ctx *ctx, const kwb_problem *P, int64_t *bytes) {
  int rc = validate_problem(ctx, P);
  if (rc) return rc;
  if (bytes) *bytes = (int64_t)estimate_device_bytes(P);
  return KWB_OK;
}

int kwb_sim_info(const kwb_sim *S, int64_t *device_bytes, int32_t *launches_per_step) {
  if (!S) return KWB_E_INVALID;
  if (device_bytes) *device_bytes = (int64_t)S->mem.bytes;
  if (launches_per_step) *launches_per_step = S->launches_per_step;
  return KWB_OK;
}

// The rest of the time loop in blocks of kSolveBlock steps: while block i runs, the time-series
// rows of block i - 1 (at first, of the steps already done) are copied to the caller on a second
// stream, so only the last block's rows and the aggregates are read after the loop.
constexpr long long kSolveBlock = 8 * KWB_CHUNK_STEPS;

int kwb_sim_finish(kwb_sim *S, kwb_outputs *out) {
  if (!S || !out) return KWB_E_INVALID;
  kwb_ctx *ctx = S->ctx;
  CU(cudaSetDevice(ctx->device));
  if (!series_streamable(S, out)) {
    const int rc = kwb_sim_advance(S, S->Nt_loop - S->steps_done);
    return rc ? rc : read_outputs_from(S, out, 0);
  }
  cudaStream_t cs = nullptr;
  cudaEvent_t done[2] = {nullptr, nullptr};
  int rc = KWB_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(done[0], S->stream);  // the steps already done
  if (e != cudaSuccess) rc = set_err(ctx, KWB_E_DEVICE, "CUDA error %s at solve streams", cudaGetErrorString(e));
  long long rows = 0;
  for (int i = 0; !rc && S->steps_done < S->Nt_loop; ++i) {
    const long long s = S->steps_done;
    if ((rc = kwb_sim_advance(S, std::min(kSolveBlock, S->Nt_loop - s)))) break;
    if ((e = cudaEventRecord(done[(i + 1) & 1], S->stream)) != cudaSuccess) {
      rc = set_err(ctx, KWB_E_DEVICE, "CUDA error %s at solve event", cudaGetErrorString(e));
      break;
    }
    if (s > rows) {  // rows [rows, s) are final once the previous block has completed
      if ((e = cudaStreamWaitEvent(cs, done[i & 1], 0)) != cudaSuccess) {
        rc = set_err(ctx, KWB_E_DEVICE, "CUDA error %s at solve wait", cudaGetErrorString(e));
        break;
      }
      if ((rc = copy_series_rows(S, out, rows, s, cs))) break;
      rows = s;
    }
  }
  if (!rc) rc = read_outputs_from(S, out, rows);
  if (cs) {
    cudaStreamSynchronize(cs);
    cudaStreamDestroy(cs);
  }
  for (cudaEvent_t ev : done)
    if (ev) cudaEventDestroy(ev);
  return rc;
}

int kwb_solve(kwb_ctx *ctx, const kwb_problem *P, kwb_outputs *out) {
  kwb_sim *S = nullptr;
  int rc = kwb_sim_create(ctx, P, &S);
  if (rc) return rc;
  rc = kwb_sim_finish(S, out);
  kwb_sim_destroy(S);
  return rc;
}

int kwb_sim_profile(kwb_sim *S, int64_t steps, kwb_kernel_times *out) {
  if (!S || !out) return KWB_E_INVALID;
  kwb_ctx *ctx = S->ctx;
  CU(cudaSetDevice(ctx->device));
  memset(out, 0, sizeof(*out));
  const SimDev &h = S->h;
  cudaStream_t st = S->stream;
  const double nv = (double)h.nvox, ns = (double)h.nspec;
  const int hr = h.rho0 ? 1 : 0;
  auto slot = [&](const char *name, double bytes) -> int {
    for (int i = 0; i < out->n; ++i)
      if (!strcmp(out->name[i], name)) return i;
    const int i = out->n++;
    snprintf(out->name[i], sizeof(out->name[i]), "%s", name);
    out->bytes_per_launch[i] = bytes;
    return i;
  };
  const long long remaining = S->Nt_loop - S->steps_done;
  if (steps > remaining) steps = remaining;
  std::vector<cudaEvent_t> evs;
  struct Rec { int slot; size_t e0; };
  std::vector<Rec> recs;
  auto ev = [&]() -> cudaEvent_t {
    cudaEvent_t e;
    cudaEventCreate(&e);
    evs.push_back(e);
    return e;
  };
  cudaError_t err = cudaSuccess;
  auto timed = [&](int sl, auto fn) {
    if (err != cudaSuccess) return;
    cudaEvent_t a = ev(), b = ev();
    cudaEventRecord(a, st);
    err = fn();
    cudaEventRecord(b, st);
    recs.push_back({sl, evs.size() - 2});
  };
  for (long long i = 0; i < steps && err == cudaSuccess; ++i) {
    const long long s = S->steps_done - S->t0_host;
    if (h.elastic) {
      elastic_step(S, s, [&](const char *nm, double bytes, auto fn) {
        timed(slot(nm, bytes), fn);
        return err;
      });
      S->steps_done++;
      continue;
    }
    if (S->tr) timed(slot("tr_inject", h.n_tr * 8.0), [&] { return launch_tr_inject(S->d_sim, h, s, st); });
    const double eos_rd = nv * 4.0 * (h.D + (h.c0sq ? 1 : 0) + (h.nonlinear && h.nlq ? 1 : 0) + (h.dispersion ? 2 : 0));
    for (int a : {1, 2, 0}) {
      if (a >= h.ndim) continue;
      static const char *nm[3] = {"line_pass_x", "line_pass_y", "line_pass_z"};
      // fused x pass: its own traffic plus the EOS forward's, less the rho_x it no longer re-reads
      const double fused = (a == 0 && h.fuse_xeos) ? eos_rd - nv * 4.0 + ns * 8.0 : 0.0;
      timed(slot(a == 0 && h.fuse_xeos ? "line_pass_x_eos_fwd" : nm[a], nv * 4.0 * (5 + hr) + fused),
            [&] { return launch_line_pass(S->d_sim, h, a, KWB_MODE_STEP, s, st); });
    }
    if (!h.fuse_xeos)
      timed(slot("eos_x_fwd", eos_rd + ns * 8.0 * (h.dispersion ? 2 : 1)), [&] { return launch_eos_x_fwd(S->d_sim, h, s, st); });
    if (h.ndim == 2) {
      timed(slot("spec_y_mul", ns * 8.0 * (h.dispersion ? 3 : 2) + ns * 4.0 * (h.dispersion ? 2 : 1)),
            [&] { return launch_spec_pass(S->d_sim, h, 1, KWB_SPEC_FWD_MUL_INV, s, st); });
    } else if (h.ndim == 3 && h.plane) {
      timed(slot("spec_yz_plane", ns * 16.0 + ns * 4.0), [&] { return fast_plane(S->d_sim, h, s, st); });
    } else if (h.ndim == 3) {
      timed(slot("spec_y_fwd", ns * 16.0 * (h.dispersion ? 2 : 1)), [&] { return launch_spec_pass(S->d_sim, h, 1, KWB_SPEC_FWD, s, st); });
      timed(slot("spec_z_mul", ns * 8.0 * (h.dispersion ? 3 : 2) + ns * 4.0 * (h.dispersion ? 2 : 1)),
            [&] { return launch_spec_pass(S->d_sim, h, 2, KWB_SPEC_FWD_MUL_INV, s, st); });
      timed(slot("spec_y_inv", ns * 16.0), [&] { return launch_spec_pass(S->d_sim, h, 1, KWB_SPEC_INV, s, st); });
    }
    timed(slot("eos_x_inv", ns * 8.0 + nv * 4.0 + (h.ndim == 1 ? ns * 4.0 : 0.0)), [&] { return launch_eos_x_inv(S->d_sim, h, s, st); });
    for (auto &g : S->groups) {
      if (g.spec.cartesian || g.n == 0 || g.fused) continue;
      timed(slot("sensor_gather", 0.0), [&] { return launch_sensor_gather(S->d_sim, h, g.d_dev, g.n, s, st); });
    }
    S->steps_done++;
  }
  cudaError_t e2 = cudaStreamSynchronize(st);
  for (auto &r : recs) {
    float ms = 0;
    cudaEventElapsedTime(&ms, evs[r.e0], evs[r.e0 + 1]);
    out->total_ms[r.slot] += ms;
    out->launches[r.slot] += 1;
  }
  for (auto e : evs) cudaEventDestroy(e);
  CU(err);
  CU(e2);
  return KWB_OK;
}

}  // extern "C"
