// kwb_eos_pressure_noalloc: the equation-of-state step without any device allocation.
//
// Some callers cannot call cudaMalloc: hosts that own all device memory through their own pool
// and forbid hidden allocations (simulation frameworks embedding this library as a plugin),
// real-time loops that must not allocate after start-up, and code that runs while another
// thread may be capturing a CUDA graph.  For them this entry point computes the pressure from
// the split density with the same kernels as kwb_solve's time step, but its scratch -- the
// kernel descriptor, the twiddle tables, the EOS multiplier and the complex half spectrum --
// lives in one file-scope device array of fixed size instead of cudaMalloc'd buffers.
//
// Costs and limits:
//   * the array (KWB_NOALLOC_SCRATCH_BYTES = 32 MiB) is part of the module image: every GPU that
//     loads libkwb holds it until the process exits, used or not;
//   * the half spectrum must fit: (Nx/2 + 1) * Ny * Nz <= KWB_NOALLOC_MAX_SPECTRUM (2,621,440,
//     e.g. 2048 x 2048, or 160^3); larger grids are rejected with KWB_E_UNSUPPORTED;
//   * the dispersion branch (scalar c0 with :stokes absorption) needs a second spectrum and the
//     previous density and is not offered here;
//   * every call shares the array, so calls whose GPU work overlaps (different streams, threads
//     or processes sharing a device context) race on it and must be serialised by the caller.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/kwb.h"
#include "kwb_internal.h"

#define KWB_NOALLOC_SCRATCH_BYTES (32u << 20)
#define KWB_NOALLOC_MAX_DEVICES 64

// Scratch of kwb_eos_pressure_noalloc.  In host code this name is only a stand-in for the
// symbol: the device address comes from cudaGetSymbolAddress (noalloc_base below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[KWB_NOALLOC_SCRATCH_BYTES];

namespace {

// layout inside g_noalloc_scratch (byte offsets, each region 256-byte aligned)
constexpr size_t kOffSim = 0;                             // SimDev descriptor
constexpr size_t kOffT0 = 4096;                           // device step base (zeroed every call)
constexpr size_t kOffTw = 4352;                           // 3 x KWB_MAX_N twiddles (float2)
constexpr size_t kOffM = kOffTw + 3 * KWB_MAX_N * 8;      // EOS multiplier, nspec floats
static_assert(sizeof(SimDev) <= kOffT0 - kOffSim, "descriptor does not fit its region");
static_assert(kOffM % 256 == 0, "alignment");

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

std::mutex g_mu;
void *g_base[KWB_NOALLOC_MAX_DEVICES];
// Last error of this host thread: concurrent callers (one per device, say) never share it.
thread_local std::string g_err;

int fail(int code, const char *msg) {
  g_err = msg;
  return code;
}

// Writes the kernel descriptor into the scratch array and zeroes the device step base.  The
// descriptor travels as a kernel parameter (copied when the launch is issued), so no host
// buffer has to outlive the call.
__global__ void k_noalloc_setup(const __grid_constant__ SimDev h, SimDev *dst, long long *t0) {
  *dst = h;
  *t0 = 0;
}

// Device address of the scratch array on `device`; looked up once per device with that device
// current (the caller's current device is restored by the entry point).
int noalloc_base(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (device < 0 || device >= KWB_NOALLOC_MAX_DEVICES) return fail(KWB_E_INVALID, "device ordinal out of range");
  if (!g_base[device]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      g_err = std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") + cudaGetErrorString(e);
      return KWB_E_DEVICE;
    }
    g_base[device] = ptr;
  }
  *out = static_cast<unsigned char *>(g_base[device]);
  return KWB_OK;
}

}  // namespace

extern "C" const char *kwb_noalloc_last_error(void) { return g_err.c_str(); }

extern "C" int kwb_eos_pressure_noalloc(int device, int32_t ndim, const int64_t N_in[3],
                                        const double d_in[3], double dt, double c_ref,
                                        int32_t alpha_mode, double alpha_coeff, double alpha_power,
                                        const float *const rho[3], const float *c0sq,
                                        float c0sq_scalar, const float *nlq, float nlq_scalar,
                                        int32_t nonlinear, float *p, void *stream) {
  using namespace kwb;
  if (ndim < 1 || ndim > 3 || !N_in || !d_in || !rho || !p) return fail(KWB_E_INVALID, "bad arguments");
  if (alpha_mode == KWB_STOKES && !c0sq)
    return fail(KWB_E_UNSUPPORTED, "the dispersion branch (scalar c0 with :stokes) is not offered without allocation");
  if (!(dt > 0) || !(c_ref > 0) || !std::isfinite(dt) || !std::isfinite(c_ref))
    return fail(KWB_E_INVALID, "dt and c_ref must be finite and positive");
  if (alpha_mode != KWB_NO_ABSORPTION && alpha_mode != KWB_NO_DISPERSION && alpha_mode != KWB_STOKES)
    return fail(KWB_E_INVALID, "alpha_mode must be KWB_NO_ABSORPTION, KWB_NO_DISPERSION or KWB_STOKES");
  if (alpha_mode != KWB_NO_ABSORPTION && (!std::isfinite(alpha_coeff) || !std::isfinite(alpha_power)))
    return fail(KWB_E_INVALID, "alpha_coeff and alpha_power must be finite");
  if (!c0sq && !(std::isfinite(c0sq_scalar) && c0sq_scalar > 0))
    return fail(KWB_E_INVALID, "c0sq_scalar must be finite and positive when c0sq is NULL");
  if (nonlinear && !nlq && !std::isfinite(nlq_scalar))
    return fail(KWB_E_INVALID, "nlq_scalar must be finite when nlq is NULL");
  SimDev h{};
  h.tile_override = -1;
  memset(h.tile_var, -1, sizeof(h.tile_var));
  h.ndim = h.D = ndim;
  for (int a = 0; a < 3; ++a) {
    const int64_t n = a < ndim ? N_in[a] : 1;
    if (n < 1 || n > KWB_MAX_N) return fail(KWB_E_UNSUPPORTED, "grid side outside 1..4096");
    if (!make_plan((int)n, h.plan[a]))
      return fail(KWB_E_UNSUPPORTED, "grid side has a prime factor above 7 (no Bluestein transform without allocation)");
    h.N[a] = (int)n;
    if (a < ndim && !rho[a]) return fail(KWB_E_INVALID, "rho component pointer is NULL");
  }
  h.n1 = h.N[0] / 2 + 1;
  h.nvox = (long long)h.N[0] * h.N[1] * h.N[2];
  h.nspec = (long long)h.n1 * h.N[1] * h.N[2];
  if (h.nspec > KWB_NOALLOC_MAX_SPECTRUM) {
    char msg[200];
    snprintf(msg, sizeof(msg), "half spectrum of %lld elements exceeds the no-alloc limit of %d "
             "((Nx/2+1)*Ny*Nz); use kwb_solve / kwb_sim_create", h.nspec, KWB_NOALLOC_MAX_SPECTRUM);
    return fail(KWB_E_UNSUPPORTED, msg);
  }
  const size_t off_spec = align256(kOffM + (size_t)h.nspec * 4);
  if (off_spec + (size_t)h.nspec * 8 > KWB_NOALLOC_SCRATCH_BYTES)
    return fail(KWB_E_UNSUPPORTED, "scratch layout overflow");

  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return fail(KWB_E_DEVICE, "cudaSetDevice failed");
  unsigned char *base = nullptr;
  int rc = noalloc_base(device, &base);
  if (rc) {
    cudaSetDevice(prev);
    return rc;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  h.dt = (float)dt;
  for (int a = 0; a < ndim; ++a) h.rho[a] = const_cast<float *>(rho[a]);
  h.p = p;
  h.c0sq = c0sq;
  h.c0sq_s = c0sq_scalar;
  h.scalar_c = c0sq ? 0 : 1;
  h.nonlinear = nonlinear ? 1 : 0;
  h.nlq = nlq;
  h.nlq_s = nlq_scalar;
  h.M = reinterpret_cast<float *>(base + kOffM);
  h.spec = reinterpret_cast<float2 *>(base + off_spec);
  for (int a = 0; a < 3; ++a) h.tw[a] = reinterpret_cast<float2 *>(base + kOffTw + (size_t)a * KWB_MAX_N * 8);
  h.L_line[0] = 1;
  h.L_line[1] = h.L_line[2] = 1;
  h.L_eosx = choose_L(h.N[0], 2048 / h.N[0], (h.N[1] + 1) / 2, 0, true);
  for (int a = 1; a < 3; ++a) h.L_spec[a] = choose_L(h.N[a], 8, h.n1, 0, true);
  h.Nt = 1;
  h.t0 = reinterpret_cast<long long *>(base + kOffT0);

  double tau = 0.0, y = 0.0;
  const int absorbing = alpha_mode != KWB_NO_ABSORPTION;
  if (absorbing) {
    y = alpha_power;
    const double a_np = alpha_coeff * (1e-2 / (20.0 * std::log10(std::exp(1.0)))) *
                        std::pow(2.0 * 3.141592653589793238462643 * 1e6, -y);
    tau = -2.0 * a_np * std::pow(c_ref, y - 1.0);
  }
  const double d3[3] = {d_in[0], ndim > 1 ? d_in[1] : 1.0, ndim > 2 ? d_in[2] : 1.0};
  const double csq_fold = c0sq ? 1.0 : (double)c0sq_scalar;

  cudaError_t e = prime_attributes(h);
  // The step base must start at zero; every other region is fully rewritten below.
  if (e == cudaSuccess) {
    k_noalloc_setup<<<1, 1, 0, st>>>(h, reinterpret_cast<SimDev *>(base + kOffSim),
                                     reinterpret_cast<long long *>(base + kOffT0));
    e = cudaGetLastError();
  }
  for (int a = 0; a < ndim && e == cudaSuccess; ++a) e = build_twiddles(const_cast<float2 *>(h.tw[a]), h.N[a], st);
  if (e == cudaSuccess)
    e = build_eos_multiplier(const_cast<float *>(h.M), nullptr, h.N, d3, c_ref, dt, csq_fold, absorbing, tau, 0.0, y, nullptr, nullptr, st);
  const SimDev *d_sim = reinterpret_cast<const SimDev *>(base + kOffSim);
  if (e == cudaSuccess) e = launch_eos_x_fwd(d_sim, h, 0, st);
  if (e == cudaSuccess && ndim == 2) e = launch_spec_pass(d_sim, h, 1, KWB_SPEC_FWD_MUL_INV, 0, st);
  if (e == cudaSuccess && ndim == 3) {
    e = launch_spec_pass(d_sim, h, 1, KWB_SPEC_FWD, 0, st);
    if (e == cudaSuccess) e = launch_spec_pass(d_sim, h, 2, KWB_SPEC_FWD_MUL_INV, 0, st);
    if (e == cudaSuccess) e = launch_spec_pass(d_sim, h, 1, KWB_SPEC_INV, 0, st);
  }
  if (e == cudaSuccess) e = launch_eos_x_inv(d_sim, h, 0, st);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    g_err = std::string("CUDA error in kwb_eos_pressure_noalloc: ") + cudaGetErrorString(e);
    return KWB_E_DEVICE;
  }
  return KWB_OK;
}
