// FFT schedule autotuner: the choices of a simulation's time-step passes measured on the device.
//
// The reference plans its FFTs with FFTW's measured planning (plan_rfft(...; flags=FFTW.MEASURE),
// KWave.jl/src/fft_utils.jl:59-60).  Here every pass of the time step has a few valid schedules
// and the fastest is measured on first use of a grid shape:
//   * register-FFT passes: the tile variant -- full-width tiles, 128-thread tiles or one-warp
//     tiles --, for the line passes whether the tiles are staged by TMA copies or by 16-byte
//     cp.async, and, for the 3-D cluster plane pass, 8 CTAs of 512 threads or 16 of 256 per plane
//     with row-major or slot-major rows;
//   * Stockham passes (other lengths): the radix order of each axis's plan, the complex lines per
//     tile, and the threads per CTA of the line passes.
// Each candidate runs on the simulation's own buffers before its initial conditions are set
// (sensors, sources and time reversal are switched off in the timing descriptor): one warm-up
// time step, then three timed with CUDA events, so that a candidate is judged by the step it
// gives; the passes are tuned one at a time, each with the others at their current choice.  Every candidate computes the same transform: the tile shape
// and thread count leave the arithmetic of each line unchanged, so results are bit-identical
// whatever is picked -- a simulation gives the same fields alone, tuned, and in a batch, which
// keeps the heuristic.  A different radix order only reorders FP32 rounding; it is explored
// only on request (KWB_TUNE_ORDER=1), since it gives up that bit-for-bit agreement.
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "kwb_internal.h"

namespace kwb {

void schedule_of(const SimDev &h, Schedule &s) {
  memset(&s, 0, sizeof(s));
  memcpy(s.tile_var, h.tile_var, sizeof(s.tile_var));
  memcpy(s.tma_line, h.tma_line, sizeof(s.tma_line));
  for (int a = 0; a < 3; ++a) {
    s.thr_line[a] = h.thr_line[a];
    s.L_line[a] = h.L_line[a];
    s.L_spec[a] = h.L_spec[a];
    s.plan_order[a] = h.plan_order[a];
  }
  s.L_eosx = h.L_eosx;
}

void schedule_apply(SimDev &h, const Schedule &s) {
  memcpy(h.tile_var, s.tile_var, sizeof(h.tile_var));
  memcpy(h.tma_line, s.tma_line, sizeof(h.tma_line));
  for (int a = 0; a < 3; ++a) {
    h.thr_line[a] = s.thr_line[a];
    h.L_line[a] = s.L_line[a];
    h.L_spec[a] = s.L_spec[a];
    h.plan_order[a] = s.plan_order[a];
    plan_line(h.N[a], h.plan[a], h.plan_order[a]);
  }
  h.L_eosx = s.L_eosx;
}

std::string schedule_str(const Schedule &s) {
  char buf[256];
  snprintf(buf, sizeof(buf),
           "tile=%d,%d,%d,%d,%d,%d,%d,%d tma=%d,%d,%d threads=%d,%d,%d L=%d,%d,%d,%d,%d,%d order=%d,%d,%d",
           s.tile_var[0], s.tile_var[1], s.tile_var[2], s.tile_var[3], s.tile_var[4], s.tile_var[5],
           s.tile_var[6], s.tile_var[7], s.tma_line[0], s.tma_line[1], s.tma_line[2], s.thr_line[0], s.thr_line[1],
           s.thr_line[2], s.L_line[0], s.L_line[1], s.L_line[2], s.L_eosx, s.L_spec[1], s.L_spec[2],
           s.plan_order[0], s.plan_order[1], s.plan_order[2]);
  return buf;
}

bool schedule_parse(const char *txt, Schedule &s) {
  int tv[8], tm[3], th[3], L[6], po[3];
  if (sscanf(txt, "tile=%d,%d,%d,%d,%d,%d,%d,%d tma=%d,%d,%d threads=%d,%d,%d L=%d,%d,%d,%d,%d,%d order=%d,%d,%d",
             &tv[0], &tv[1], &tv[2], &tv[3], &tv[4], &tv[5], &tv[6], &tv[7], &tm[0], &tm[1], &tm[2], &th[0], &th[1],
             &th[2], &L[0], &L[1], &L[2], &L[3], &L[4], &L[5], &po[0], &po[1], &po[2]) != 23)
    return false;
  memset(&s, 0, sizeof(s));
  for (int a = 0; a < 3; ++a) {
    if (tm[a] < -1 || tm[a] > 1) return false;
    s.tma_line[a] = (signed char)tm[a];
  }
  for (int i = 0; i < 8; ++i) {
    if (tv[i] < -1 || tv[i] >= KWB_PLANE_VARIANTS) return false;
    s.tile_var[i] = (signed char)tv[i];
  }
  for (int a = 0; a < 3; ++a) {
    if (th[a] < 0 || th[a] > KWB_PASS_THREADS_MAX || th[a] % 32) return false;
    if (po[a] < 0 || po[a] > 2) return false;
    s.thr_line[a] = (short)th[a];
    s.plan_order[a] = (signed char)po[a];
    s.L_line[a] = L[a];
  }
  s.L_eosx = L[3];
  s.L_spec[0] = 1;
  s.L_spec[1] = L[4];
  s.L_spec[2] = L[5];
  for (int i = 0; i < 6; ++i)
    if (L[i] < 1 || L[i] > 4096) return false;
  return true;
}

namespace {

bool line_is_fast(const SimDev &h, int a) { return (h.fast & 1) && fast_size(h.N[a]) && (a == 0 || h.N[0] % 4 == 0); }
bool eos_is_fast(const SimDev &h) { return (h.fast & 2) && h.ndim >= 2 && !h.dispersion && fast_size(h.N[0]); }
bool spec_is_fast(const SimDev &h, int a) { return (h.fast & 2) && !h.dispersion && fast_size(h.N[a]); }

struct Tuner {
  SimDev t;  // timing descriptor
  SimDev *d_t;
  cudaStream_t st;
  int pick;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::string *log;

  // Average device time of one launch of `go` with the descriptor t (FLT_MAX if it failed).
  template <class F>
  float time(F go) {
    cudaError_t e = cudaMemcpyAsync(d_t, &t, sizeof(SimDev), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = prime_attributes(t);
    if (e == cudaSuccess) e = go();
    if (e == cudaSuccess) e = cudaEventRecord(e0, st);
    for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = go();
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return FLT_MAX;
    }
    return ms / 3.f;
  }

  // Try `n` candidates set by set(i) (i < n), keep the fastest (or candidate `pick`).
  template <class Set, class F>
  void choose(const char *what, int n, Set set, F go) {
    if (n <= 0) return;
    int best = 0;
    if (pick >= 0) {
      best = pick < n ? pick : n - 1;
    } else {
      float tb = FLT_MAX;
      for (int i = 0; i < n; ++i) {
        set(i);
        const float ms = time(go);
        if (log) {
          char b[96];
          snprintf(b, sizeof(b), "%s[%d]=%.4fms ", what, i, ms);
          *log += b;
        }
        if (ms < tb) {
          tb = ms;
          best = i;
        }
      }
    }
    set(best);
  }
};

// Lines-per-tile candidates around the heuristic choice L0, clamped as the heuristic is.
std::vector<int> l_candidates(int N, int L0, int cap, int disp, bool spec) {
  std::vector<int> out;
  for (int want : {L0, 2 * L0, L0 / 2, L0 / 4}) {
    if (want < 1) continue;
    const int L = choose_L(N, want, cap, disp, spec);
    bool seen = false;
    for (int v : out) seen |= v == L;
    if (!seen) out.push_back(L);
  }
  return out;
}

}  // namespace

cudaError_t tune_schedule(SimDev &h, SimDev *d_scratch, cudaStream_t st, int pick, bool explore_order,
                          std::string *log) {
  Tuner T;
  T.t = h;
  SimDev &t = T.t;
  // timing descriptor: no sensors, sources or time reversal (their buffers stay untouched)
  t.dense_p = nullptr;
  t.sparse_p = nullptr;
  t.n_p = 0;
  t.n_u = 0;
  t.n_tr = 0;
  for (int a = 0; a < 3; ++a) {
    t.p_line_ptr[a] = nullptr;
    t.p_entry[a] = nullptr;
    t.u_sig[a] = nullptr;
    t.u_line_ptr[a] = nullptr;
    t.u_entry[a] = nullptr;
  }
  T.d_t = d_scratch;
  T.st = st;
  T.pick = pick;
  T.log = log;
  cudaError_t e = cudaEventCreate(&T.e0);
  if (e == cudaSuccess) e = cudaEventCreate(&T.e1);
  if (e != cudaSuccess) return e;
  const int D = h.ndim;
  const SimDev *d = d_scratch;
  // Every candidate is timed on whole time steps (the step's passes launched as the simulation
  // launches them, each waiting on its predecessor by programmatic dependent launch), not on its
  // own pass alone: a pass's tile shape also changes how its launch overlaps its neighbours'.
  auto step = [&]() -> cudaError_t {
    cudaError_t e;
    for (int a : {1, 2, 0})
      if (a < D && (e = launch_line_pass(d, t, a, KWB_MODE_STEP, 0, st)) != cudaSuccess) return e;
    if (!t.fuse_xeos && (e = launch_eos_x_fwd(d, t, 0, st)) != cudaSuccess) return e;
    if (D == 2) {
      if ((e = launch_spec_pass(d, t, 1, KWB_SPEC_FWD_MUL_INV, 0, st)) != cudaSuccess) return e;
    } else if (D == 3 && t.plane) {
      if ((e = fast_plane(d, t, 0, st)) != cudaSuccess) return e;
    } else if (D == 3) {
      if ((e = launch_spec_pass(d, t, 1, KWB_SPEC_FWD, 0, st)) != cudaSuccess) return e;
      if ((e = launch_spec_pass(d, t, 2, KWB_SPEC_FWD_MUL_INV, 0, st)) != cudaSuccess) return e;
      if ((e = launch_spec_pass(d, t, 1, KWB_SPEC_INV, 0, st)) != cudaSuccess) return e;
    }
    return launch_eos_x_inv(d, t, 0, st);
  };

  // line passes (the x pass carries the EOS x R2C when fused)
  for (int a = 0; a < D; ++a) {
    auto go = step;
    if (line_is_fast(t, a)) {
      T.choose("line_tile", 3, [&, a](int i) { t.tile_var[KWB_SLOT_LINE0 + a] = (signed char)i; }, go);
      // tiles staged by TMA copies or by 16-byte cp.async (unless KWB_TILE_TMA fixes it)
      if (!getenv("KWB_TILE_TMA"))
        T.choose("line_tma", 2, [&, a](int i) { t.tma_line[a] = (signed char)(i == 0 ? 0 : 1); }, go);
      continue;
    }
    // Stockham: radix order (distinct plans only; with explore_order), then lines per tile,
    // then threads per CTA
    std::vector<int> orders;
    std::vector<FftPlan> plans;
    for (int o = 0; o < (explore_order ? 3 : 1); ++o) {
      FftPlan pl = t.plan[a];
      if (!plan_line(t.N[a], pl, o)) continue;
      bool dup = false;
      for (const FftPlan &q : plans) dup |= q.nstages == pl.nstages && !memcmp(q.radix, pl.radix, pl.nstages * sizeof(int));
      if (dup) continue;
      plans.push_back(pl);
      orders.push_back(o);
    }
    T.choose("line_order", (int)orders.size(), [&, a](int i) {
      t.plan_order[a] = (signed char)orders[i];
      t.plan[a] = plans[i];
    }, go);
    const int cap = a == 0 ? (t.N[1] + 1) / 2 : (t.N[0] + 1) / 2;
    const std::vector<int> Ls = l_candidates(fft_len(t.plan[a]), t.L_line[a], cap, 0, false);
    T.choose("line_L", (int)Ls.size(), [&, a](int i) { t.L_line[a] = Ls[i]; }, go);
    const int thr[4] = {0, 256, 512, 1024};
    T.choose("line_threads", 4, [&, a](int i) { t.thr_line[a] = (short)thr[i]; }, go);
  }

  // equation of state, x direction
  if (D >= 1) {
    if (eos_is_fast(t)) {
      if (!t.fuse_xeos)
        T.choose("eos_fwd_tile", 3, [&](int i) { t.tile_var[KWB_SLOT_EOS_FWD] = (signed char)i; },
                 step);
      T.choose("eos_inv_tile", 3, [&](int i) { t.tile_var[KWB_SLOT_EOS_INV] = (signed char)i; },
               step);
    } else {
      const std::vector<int> Ls = l_candidates(fft_len(t.plan[0]), t.L_eosx, (t.N[1] + 1) / 2, t.dispersion, true);
      T.choose("eos_L", (int)Ls.size(), [&](int i) { t.L_eosx = Ls[i]; }, step);
    }
  }

  // the 3-D cluster plane pass: 8 CTAs of 512 threads or 16 of 256 per kx plane, rows kept
  // row-major (block-wide z transforms) or slot-major (one warp per z line).  The slot-major
  // kernels read the multiplier in another layout; timing them on the row-major table reads the
  // same bytes from the same buffer.
  if (t.plane) {
    int ids[KWB_PLANE_VARIANTS];
    const int nv = fast_plane_variants(ids);
    T.choose("plane", nv > 1 ? nv : 0, [&](int i) { t.tile_var[KWB_SLOT_PLANE] = (signed char)ids[i]; },
             step);
  }
  // spectrum passes along y and z
  if (!t.plane) {
    for (int a = 1; a < D; ++a) {
      auto go = step;
      if (spec_is_fast(t, a)) {
        T.choose("spec_tile", 3, [&, a](int i) { t.tile_var[KWB_SLOT_SPEC1 + a - 1] = (signed char)i; }, go);
      } else {
        const std::vector<int> Ls = l_candidates(fft_len(t.plan[a]), t.L_spec[a], t.n1, t.dispersion, true);
        T.choose("spec_L", (int)Ls.size(), [&, a](int i) { t.L_spec[a] = Ls[i]; }, go);
      }
    }
  }
  cudaEventDestroy(T.e0);
  cudaEventDestroy(T.e1);
  Schedule s;
  schedule_of(t, s);
  schedule_apply(h, s);
  return cudaGetLastError();
}

}  // namespace kwb
