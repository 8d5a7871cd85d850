// Continuous batching of independent simulations on one GPU (kwb_submit / kwb_poll / kwb_wait /
// kwb_cancel / kwb_solve_batch).
//
// A scheduler thread per context keeps a FIFO of submitted requests and a set of admitted
// simulations.  A request is admitted -- its simulation created, its medium and tables made
// resident -- as soon as a slot and device memory allow (modelled bytes against free memory and
// an optional cap).  Every admitted simulation advances in CUDA-graph chunks of `chunk` time
// steps on its own stream, so work from different requests overlaps on the device; a request
// that finishes is read back into the caller's buffers and its memory is released, which
// admits the next ones.  Failures stay per request: an invalid or oversized problem completes
// with its status while the others run on; cancelling a request drops it at its next chunk
// boundary.  Every wait here is on host state with a caller-given timeout; nothing spins on the
// device.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/kwb.h"
#include "kwb_internal.h"

struct kwb_ctx;  // kwb_api.cu
size_t estimate_device_bytes(const kwb_problem *P);
cudaStream_t kwb_sim_stream_of(kwb_sim *S);
long long kwb_sim_nt_of(const kwb_sim *S);
void kwb_ctx_set_err(kwb_ctx *ctx, const char *msg);
int kwb_ctx_device(const kwb_ctx *ctx);
void kwb_ctx_set_batched(kwb_ctx *ctx);

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  uint64_t ticket = 0;
  const kwb_problem *P = nullptr;
  kwb_outputs *out = nullptr;
  int state = 0;  // 0 queued, 1 running, 2 done
  int status = KWB_E_BUSY;
  bool cancel = false;
  kwb_sim *sim = nullptr;
  cudaEvent_t ev = nullptr;
  bool inflight = false;
  size_t bytes = 0;
  long long voxels = 0;
  int64_t t_submit = 0, t_start = 0, t_end = 0;
  std::string err;
};

}  // namespace

struct KwbServer {
  kwb_ctx *owner = nullptr;
  kwb_ctx *inner = nullptr;  // private context for the scheduler thread's simulation calls
  std::thread th;
  std::mutex mu;
  std::condition_variable cv_done, cv_work;
  std::deque<Request *> queued;
  std::vector<Request *> running;
  std::unordered_map<uint64_t, Request *> all;
  uint64_t next_ticket = 1;
  bool stop = false;
  int max_running = 64;
  // Admission by size: a request starts while the running simulations hold at most this many
  // voxels (or when nothing runs).  Small grids cannot fill the GPU alone, so many run together;
  // large ones run a few at a time, since more would only split the L2 between their working
  // sets and lengthen every request's latency.
  long long voxel_budget = 4LL << 20;
  long long running_voxels = 0;
  int chunk = 32;
  size_t mem_cap = 0;  // 0: free device memory only
  size_t running_bytes = 0;
  kwb_serving_stats stats{};

  void finish(Request *r, int status, const char *err) {
    r->status = status;
    if (err) r->err = err;
    r->t_end = now_ns();
    r->state = 2;
    if (status == KWB_OK) stats.completed++;
    else if (status == KWB_E_CANCELLED) stats.cancelled++;
    else stats.failed++;
  }

  void release_sim(Request *r) {
    if (r->ev) cudaEventDestroy(r->ev);
    r->ev = nullptr;
    if (r->sim) kwb_sim_destroy(r->sim);
    r->sim = nullptr;
    running_bytes -= std::min(running_bytes, r->bytes);
    running_voxels -= std::min(running_voxels, r->voxels);
  }

  // Admit queued requests while slots and memory allow.  Called with `mu` held; drops it around
  // the (blocking) simulation set-up.
  bool admit(std::unique_lock<std::mutex> &lk) {
    bool changed = false;
    while (!queued.empty() && (int)running.size() < max_running) {
      Request *r = queued.front();
      if (r->cancel) {
        queued.pop_front();
        finish(r, KWB_E_CANCELLED, "cancelled before admission");
        changed = true;
        continue;
      }
      long long vox = 1;
      for (int a = 0; a < r->P->ndim; ++a) vox *= r->P->N[a];
      if (!running.empty() && voxel_budget > 0 && running_voxels + vox > voxel_budget) break;
      const size_t need = estimate_device_bytes(r->P);
      if (mem_cap && running_bytes + need > mem_cap) {
        if (running.empty()) {  // can never fit under the cap
          queued.pop_front();
          finish(r, KWB_E_NOMEM, "request exceeds the serving memory cap");
          changed = true;
          continue;
        }
        break;
      }
      queued.pop_front();
      lk.unlock();
      kwb_sim *sim = nullptr;
      int rc = kwb_sim_create(inner, r->P, &sim);
      std::string msg = rc ? kwb_last_error(inner) : "";
      cudaEvent_t ev = nullptr;
      if (!rc && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        kwb_sim_destroy(sim);
        sim = nullptr;
        rc = KWB_E_DEVICE;
        msg = "cudaEventCreate failed";
      }
      lk.lock();
      changed = true;
      if (rc == KWB_E_NOMEM && !running.empty()) {  // wait for running simulations to free memory
        queued.push_front(r);
        break;
      }
      if (rc) {
        finish(r, rc, msg.c_str());
        cv_done.notify_all();
        continue;
      }
      r->sim = sim;
      r->ev = ev;
      r->bytes = need;
      running_bytes += need;
      r->voxels = vox;
      running_voxels += vox;
      r->state = 1;
      r->t_start = now_ns();
      running.push_back(r);
      stats.admitted++;
      stats.peak_running = std::max<int64_t>(stats.peak_running, (int64_t)running.size());
    }
    return changed;
  }

  // One pass over the running simulations: retire finished ones, queue the next chunk of the
  // others.  Called without `mu` held (touches only scheduler-owned state, then locks to retire).
  bool progress() {
    bool changed = false;
    std::vector<Request *> snapshot;
    {
      std::lock_guard<std::mutex> lk(mu);
      snapshot = running;
    }
    for (Request *r : snapshot) {
      if (r->inflight) {
        const cudaError_t q = cudaEventQuery(r->ev);
        if (q == cudaErrorNotReady) continue;
        r->inflight = false;
        if (q != cudaSuccess) {
          std::lock_guard<std::mutex> lk(mu);
          finish(r, KWB_E_DEVICE, cudaGetErrorString(q));
          retire(r);
          changed = true;
          continue;
        }
      }
      bool cancel;
      {
        std::lock_guard<std::mutex> lk(mu);
        cancel = r->cancel;
      }
      const long long done = kwb_sim_steps_done(r->sim), Nt = kwb_sim_nt_of(r->sim);
      if (cancel) {
        std::lock_guard<std::mutex> lk(mu);
        finish(r, KWB_E_CANCELLED, "cancelled");
        retire(r);
        changed = true;
        continue;
      }
      if (done >= Nt) {
        const int rc = kwb_sim_read_outputs(r->sim, r->out);
        std::string msg = rc ? kwb_last_error(inner) : "";
        std::lock_guard<std::mutex> lk(mu);
        finish(r, rc, rc ? msg.c_str() : nullptr);
        retire(r);
        changed = true;
        continue;
      }
      int rc = kwb_sim_advance(r->sim, chunk);
      if (!rc && cudaEventRecord(r->ev, kwb_sim_stream_of(r->sim)) != cudaSuccess) rc = KWB_E_DEVICE;
      if (rc) {
        std::string msg = kwb_last_error(inner);
        std::lock_guard<std::mutex> lk(mu);
        finish(r, rc, msg.c_str());
        retire(r);
        changed = true;
        continue;
      }
      r->inflight = true;
      stats.chunks++;
      changed = true;
    }
    return changed;
  }

  // with mu held
  void retire(Request *r) {
    running.erase(std::remove(running.begin(), running.end(), r), running.end());
    release_sim(r);
    cv_done.notify_all();
  }

  void loop() {
    cudaSetDevice(kwb_ctx_device(inner));
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
      bool changed = admit(lk);
      const bool any_running = !running.empty();
      lk.unlock();
      if (any_running) changed |= progress();
      lk.lock();
      if (stop) break;
      if (!changed) {
        if (running.empty() && queued.empty()) cv_work.wait(lk);
        else cv_work.wait_for(lk, std::chrono::microseconds(50));
      }
    }
    // shutdown: cancel everything still pending or running
    for (Request *r : queued) finish(r, KWB_E_CANCELLED, "context destroyed");
    queued.clear();
    lk.unlock();
    for (Request *r : running) {
      if (r->sim) kwb_sim_sync(r->sim);
      finish(r, KWB_E_CANCELLED, "context destroyed");
      release_sim(r);
    }
    lk.lock();
    running.clear();
    cv_done.notify_all();
  }
};

static KwbServer *server_of(kwb_ctx *ctx, KwbServer *&slot) {
  if (!slot) {
    KwbServer *s = new KwbServer();
    s->owner = ctx;
    kwb_context_create(kwb_ctx_device(ctx), &s->inner);
    if (s->inner) kwb_ctx_set_batched(s->inner);
    s->th = std::thread([s] { s->loop(); });
    slot = s;
  }
  return slot;
}

// kwb_api.cu keeps the server pointer in the context
KwbServer *&kwb_ctx_server_slot(kwb_ctx *ctx);

void kwb_server_shutdown(kwb_ctx *ctx) {
  KwbServer *&slot = kwb_ctx_server_slot(ctx);
  if (!slot) return;
  {
    std::lock_guard<std::mutex> lk(slot->mu);
    slot->stop = true;
  }
  slot->cv_work.notify_all();
  slot->th.join();
  for (auto &kv : slot->all) delete kv.second;
  kwb_context_destroy(slot->inner);
  delete slot;
  slot = nullptr;
}

extern "C" {

int kwb_serving_voxel_budget(kwb_ctx *ctx, int64_t voxels) {
  if (!ctx || voxels < 0) return KWB_E_INVALID;
  KwbServer *s = server_of(ctx, kwb_ctx_server_slot(ctx));
  std::lock_guard<std::mutex> lk(s->mu);
  s->voxel_budget = voxels;
  s->cv_work.notify_all();
  return KWB_OK;
}

int kwb_serving_config(kwb_ctx *ctx, int32_t max_running, int32_t chunk_steps, int64_t mem_cap_bytes) {
  if (!ctx || max_running < 1 || chunk_steps < 1 || mem_cap_bytes < 0) return KWB_E_INVALID;
  KwbServer *s = server_of(ctx, kwb_ctx_server_slot(ctx));
  std::lock_guard<std::mutex> lk(s->mu);
  s->max_running = max_running;
  s->chunk = chunk_steps;
  s->mem_cap = (size_t)mem_cap_bytes;
  s->cv_work.notify_all();
  return KWB_OK;
}

int kwb_submit(kwb_ctx *ctx, const kwb_problem *problem, kwb_outputs *outputs, uint64_t *ticket) {
  if (!ctx || !problem || !outputs || !ticket) return KWB_E_INVALID;
  KwbServer *s = server_of(ctx, kwb_ctx_server_slot(ctx));
  Request *r = new Request();
  r->P = problem;
  r->out = outputs;
  r->t_submit = now_ns();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->ticket = s->next_ticket++;
    s->all[r->ticket] = r;
    s->queued.push_back(r);
    s->stats.submitted++;
  }
  s->cv_work.notify_all();
  *ticket = r->ticket;
  return KWB_OK;
}

int kwb_poll(kwb_ctx *ctx, uint64_t ticket, int32_t *done) {
  if (!ctx || !done) return KWB_E_INVALID;
  KwbServer *s = kwb_ctx_server_slot(ctx);
  if (!s) return KWB_E_NOTFOUND;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return KWB_E_NOTFOUND;
  *done = it->second->state == 2;
  return KWB_OK;
}

int kwb_wait(kwb_ctx *ctx, uint64_t ticket, int64_t timeout_ns, kwb_request_info *info) {
  if (!ctx) return KWB_E_INVALID;
  KwbServer *s = kwb_ctx_server_slot(ctx);
  if (!s) return KWB_E_NOTFOUND;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return KWB_E_NOTFOUND;
  Request *r = it->second;
  auto pred = [&] { return r->state == 2; };
  if (timeout_ns < 0) s->cv_done.wait(lk, pred);
  else if (!s->cv_done.wait_for(lk, std::chrono::nanoseconds(timeout_ns), pred)) return KWB_E_TIMEOUT;
  if (info) {
    info->status = r->status;
    info->submit_ns = r->t_submit;
    info->start_ns = r->t_start;
    info->end_ns = r->t_end;
    snprintf(info->error, sizeof(info->error), "%s", r->err.c_str());
  }
  const int st = r->status;
  if (st != KWB_OK) kwb_ctx_set_err(ctx, r->err.c_str());
  s->all.erase(it);
  delete r;
  return st;
}

int kwb_cancel(kwb_ctx *ctx, uint64_t ticket) {
  if (!ctx) return KWB_E_INVALID;
  KwbServer *s = kwb_ctx_server_slot(ctx);
  if (!s) return KWB_E_NOTFOUND;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return KWB_E_NOTFOUND;
    it->second->cancel = true;
  }
  s->cv_work.notify_all();
  return KWB_OK;
}

int kwb_serving_stats_get(kwb_ctx *ctx, kwb_serving_stats *out) {
  if (!ctx || !out) return KWB_E_INVALID;
  KwbServer *s = kwb_ctx_server_slot(ctx);
  if (!s) {
    memset(out, 0, sizeof(*out));
    return KWB_OK;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->queued = (int64_t)s->queued.size();
  out->running = (int64_t)s->running.size();
  out->running_bytes = (int64_t)s->running_bytes;
  return KWB_OK;
}

int kwb_solve_batch(kwb_ctx *ctx, int32_t n, const kwb_problem *const *problems,
                    kwb_outputs *const *outputs, int32_t *status) {
  if (!ctx || n < 0 || (n > 0 && (!problems || !outputs || !status))) return KWB_E_INVALID;
  std::vector<uint64_t> t(n);
  for (int i = 0; i < n; ++i) {
    int rc = kwb_submit(ctx, problems[i], outputs[i], &t[i]);
    if (rc) return rc;
  }
  int first = KWB_OK;
  for (int i = 0; i < n; ++i) {
    status[i] = kwb_wait(ctx, t[i], -1, nullptr);
    if (status[i] && !first) first = status[i];
  }
  return first;
}

}  // extern "C"
