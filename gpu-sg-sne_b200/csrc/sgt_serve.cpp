// sgt_serve.cpp -- continuous batching of embedding requests on one device.
//
// Two native threads share the device with the caller:
//   admission  takes waiting requests in FIFO order as soon as the request's
//              footprint fits the HBM budget and a slot is free, builds its
//              job (P upload, autotune, Y0) on a stream of its own and queues
//              the first round;
//   scheduler  keeps every running job `rounds_ahead` rounds of
//              `iters_per_round` iterations ahead of the GPU (one graph
//              launch per round, an event per round), and when a job's last
//              round has run copies its coordinates to the caller's buffer,
//              frees its memory (stream-ordered, no device synchronisation)
//              and returns its footprint to the budget.
// Jobs therefore overlap on the GPU whatever their size or arrival time; the
// hardware interleaves the kernels of all streams.  Streams carry priorities
// that rise as n falls, so the short iterations of small embeddings are not
// queued behind the thousands of blocks of a large one.
//
// Only the public C ABI of the engine is used (sgt_job_*), plus the CUDA
// runtime for streams and events.
#include "../../include/sgtsne_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace {

// requests of fewer points run without the locality order of job creation
constexpr int SGT_SERVE_ORDER_MIN_N = 1000000;

struct Request {
  long long id = 0;
  sgt_params p{};
  int n = 0;
  long nnz = 0;
  const int *rowptr = nullptr;
  const int *col = nullptr;
  const float *val = nullptr;
  const float *y0 = nullptr;
  float *y_out = nullptr;
  size_t footprint = 0;
  int state = SGT_REQ_WAITING;
  sgt_status status = SGT_OK;
  double t_submit = 0, t_admit = 0, t_done = 0;
  // while running (scheduler thread only, after admission)
  struct Slot *slot = nullptr;
  sgt_job *job = nullptr;
  int iters_total = 0, iters_queued = 0;
  std::deque<cudaEvent_t> inflight;  // one event per queued round
};

struct Slot {
  sgt_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  int prio = 0;
};

}  // namespace

struct sgt_server {
  int device = 0;
  sgt_server_config cfg{};
  std::chrono::steady_clock::time_point t0;
  int prio_least = 0, prio_greatest = 0;

  std::mutex mu;
  std::condition_variable cv_admit;  // admission: a request, budget or slot appeared
  std::condition_variable cv_sched;  // scheduler: an admitted job is ready
  std::condition_variable cv_done;   // poll: a request finished
  std::deque<std::unique_ptr<Request>> reqs;  // by id
  std::deque<Request *> waiting;
  std::vector<Request *> ready;     // admitted, not yet taken by the scheduler
  std::deque<long long> finished;   // ids for poll
  std::vector<Slot *> free_slots;   // idle contexts with their streams
  std::vector<std::unique_ptr<Slot>> slots;
  size_t used = 0;
  int active = 0;  // admitted, not yet retired
  bool stop = false;

  std::thread admit_thr, sched_thr;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  int prio_for(int n) const {
    // greatest (numerically lowest) priority for the smallest embeddings
    const int levels = prio_least - prio_greatest + 1;
    int lv = (int)std::floor((std::log2((double)std::max(n, 2)) - 10.0) / 1.5);
    lv = std::max(0, std::min(levels - 1, lv));
    return prio_greatest + lv;
  }
};

namespace {

// under srv->mu
Slot *take_slot(sgt_server *srv, int prio) {
  for (size_t k = 0; k < srv->free_slots.size(); k++) {
    if (srv->free_slots[k]->prio == prio) {
      Slot *s = srv->free_slots[k];
      srv->free_slots.erase(srv->free_slots.begin() + k);
      return s;
    }
  }
  return nullptr;
}

Slot *new_slot(sgt_server *srv, int prio, sgt_status *st) {
  std::unique_ptr<Slot> s(new Slot());
  s->prio = prio;
  *st = sgt_create(srv->device, &s->ctx);
  if (*st != SGT_OK) return nullptr;
  if (cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, prio) != cudaSuccess) {
    sgt_destroy(s->ctx);
    *st = SGT_ERR_CUDA;
    return nullptr;
  }
  *st = sgt_set_stream(s->ctx, s->stream);
  if (*st != SGT_OK) {
    sgt_destroy(s->ctx);
    cudaStreamDestroy(s->stream);
    return nullptr;
  }
  Slot *raw = s.get();
  std::lock_guard<std::mutex> lk(srv->mu);
  srv->slots.push_back(std::move(s));
  return raw;
}

// under srv->mu: a request leaves the running set
void finish_locked(sgt_server *srv, Request *r, int state, sgt_status status) {
  r->state = state;
  r->status = status;
  r->t_done = srv->now();
  srv->used -= r->footprint;
  srv->active--;
  if (r->slot) srv->free_slots.push_back(r->slot);
  r->slot = nullptr;
  srv->finished.push_back(r->id);
  srv->cv_done.notify_all();
  srv->cv_admit.notify_all();
}

sgt_status queue_round(Request *r, int iters_per_round, std::vector<cudaEvent_t> &pool) {
  const int k = std::min(iters_per_round, r->iters_total - r->iters_queued);
  sgt_status st = sgt_job_run(r->job, k);
  if (st != SGT_OK) return st;
  cudaEvent_t ev = nullptr;
  if (!pool.empty()) {
    ev = pool.back();
    pool.pop_back();
  } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    return SGT_ERR_CUDA;
  }
  if (cudaEventRecord(ev, r->slot->stream) != cudaSuccess) {
    pool.push_back(ev);
    return SGT_ERR_CUDA;
  }
  r->inflight.push_back(ev);
  r->iters_queued += k;
  return SGT_OK;
}

void admission_loop(sgt_server *srv) {
  cudaSetDevice(srv->device);
  std::vector<cudaEvent_t> pool;  // events created here move to the scheduler
  std::unique_lock<std::mutex> lk(srv->mu);
  for (;;) {
    srv->cv_admit.wait(lk, [&] {
      if (srv->stop) return true;
      if (srv->waiting.empty() || srv->active >= srv->cfg.max_active) return false;
      return srv->used + srv->waiting.front()->footprint <= srv->cfg.hbm_budget;
    });
    if (srv->stop) {
      // requests never admitted fail; running ones finish in the scheduler
      while (!srv->waiting.empty()) {
        Request *r = srv->waiting.front();
        srv->waiting.pop_front();
        r->state = SGT_REQ_FAILED;
        r->status = SGT_ERR_INVALID_ARG;
        r->t_done = srv->now();
        srv->finished.push_back(r->id);
      }
      srv->cv_done.notify_all();
      break;
    }
    Request *r = srv->waiting.front();
    srv->waiting.pop_front();
    srv->used += r->footprint;
    srv->active++;
    const int prio = srv->prio_for(r->n);
    Slot *slot = take_slot(srv, prio);
    lk.unlock();
    sgt_status st = SGT_OK;
    if (!slot) slot = new_slot(srv, prio, &st);
    sgt_job *job = nullptr;
    if (slot) {
      r->slot = slot;
      st = sgt_job_create(slot->ctx, &r->p, r->n, r->rowptr, r->col, r->val, 0, &job);
      if (st == SGT_OK) st = sgt_job_set_y(job, r->y0, SGT_LAYOUT_POINT_MAJOR, 0);
      if (st == SGT_OK) {
        r->job = job;
        st = queue_round(r, srv->cfg.iters_per_round, pool);
      }
      if (st != SGT_OK && job) {
        cudaStreamSynchronize(slot->stream);
        sgt_job_destroy(job);
        r->job = nullptr;
        for (cudaEvent_t e : r->inflight) cudaEventDestroy(e);
        r->inflight.clear();
      }
    }
    lk.lock();
    if (st != SGT_OK) {
      finish_locked(srv, r, SGT_REQ_FAILED, st);
      continue;
    }
    r->state = SGT_REQ_RUNNING;
    r->t_admit = srv->now();
    srv->ready.push_back(r);
    srv->cv_sched.notify_all();
  }
  lk.unlock();
  for (cudaEvent_t e : pool) cudaEventDestroy(e);
}

void scheduler_loop(sgt_server *srv) {
  cudaSetDevice(srv->device);
  std::vector<Request *> running;
  std::vector<cudaEvent_t> pool;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(srv->mu);
      if (running.empty())
        srv->cv_sched.wait(lk, [&] {
          return !srv->ready.empty() || (srv->stop && srv->active == 0);
        });
      running.insert(running.end(), srv->ready.begin(), srv->ready.end());
      srv->ready.clear();
      if (running.empty() && srv->stop && srv->active == 0) break;
    }
    bool progress = false;
    for (size_t k = 0; k < running.size();) {
      Request *r = running[k];
      while (!r->inflight.empty() && cudaEventQuery(r->inflight.front()) == cudaSuccess) {
        pool.push_back(r->inflight.front());
        r->inflight.pop_front();
        progress = true;
      }
      sgt_status st = SGT_OK;
      if (r->iters_queued < r->iters_total &&
          (int)r->inflight.size() < srv->cfg.rounds_ahead) {
        st = queue_round(r, srv->cfg.iters_per_round, pool);
        progress = true;
      }
      const bool done = st == SGT_OK && r->iters_queued == r->iters_total && r->inflight.empty();
      if (st != SGT_OK || done) {
        if (done) st = sgt_job_get_y(r->job, r->y_out, SGT_LAYOUT_POINT_MAJOR, 0, 1);
        cudaStreamSynchronize(r->slot->stream);
        for (cudaEvent_t e : r->inflight) pool.push_back(e);
        r->inflight.clear();
        sgt_job_destroy(r->job);
        r->job = nullptr;
        {
          std::lock_guard<std::mutex> lk(srv->mu);
          finish_locked(srv, r, st == SGT_OK ? SGT_REQ_DONE : SGT_REQ_FAILED, st);
        }
        running.erase(running.begin() + k);
        progress = true;
        continue;
      }
      k++;
    }
    if (!progress) {
      // nothing finished and every job is `rounds_ahead` rounds ahead:
      // wait a little, or until a new job is admitted
      std::unique_lock<std::mutex> lk(srv->mu);
      srv->cv_sched.wait_for(lk, std::chrono::microseconds(50),
                             [&] { return !srv->ready.empty(); });
    }
  }
  for (cudaEvent_t e : pool) cudaEventDestroy(e);
}

}  // namespace

extern "C" {

void sgt_server_config_default(sgt_server_config *cfg) {
  if (!cfg) return;
  cfg->hbm_budget = (size_t)150 << 30;
  cfg->max_active = 128;
  cfg->iters_per_round = 16;
  cfg->rounds_ahead = 2;
}

sgt_status sgt_server_create(int device, const sgt_server_config *cfg, sgt_server **out) {
  if (!out) return SGT_ERR_INVALID_ARG;
  *out = nullptr;
  sgt_server_config c;
  sgt_server_config_default(&c);
  if (cfg) c = *cfg;
  if (c.hbm_budget == 0 || c.max_active < 1 || c.max_active > 1024 || c.iters_per_round < 1 ||
      c.iters_per_round > 256 || c.rounds_ahead < 1)
    return SGT_ERR_INVALID_ARG;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return SGT_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return SGT_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return SGT_ERR_CUDA;
  sgt_server *srv = new sgt_server();
  srv->device = device;
  srv->cfg = c;
  srv->t0 = std::chrono::steady_clock::now();
  if (cudaDeviceGetStreamPriorityRange(&srv->prio_least, &srv->prio_greatest) != cudaSuccess) {
    srv->prio_least = srv->prio_greatest = 0;
  }
  srv->admit_thr = std::thread(admission_loop, srv);
  srv->sched_thr = std::thread(scheduler_loop, srv);
  *out = srv;
  return SGT_OK;
}

void sgt_server_destroy(sgt_server *srv) {
  if (!srv) return;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
    srv->cv_admit.notify_all();
    srv->cv_sched.notify_all();
  }
  srv->admit_thr.join();
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->cv_sched.notify_all();
  }
  srv->sched_thr.join();
  cudaSetDevice(srv->device);
  for (auto &s : srv->slots) {
    sgt_destroy(s->ctx);
    cudaStreamDestroy(s->stream);
  }
  delete srv;
}

sgt_status sgt_server_submit(sgt_server *srv, const sgt_params *params, int n, const int *rowptr,
                             const int *col, const float *val, const float *y0, float *y_out,
                             long long *id) {
  if (!srv || !params || !rowptr || !col || !val || !y0 || !y_out || !id || n < 2)
    return SGT_ERR_INVALID_ARG;
  if (params->d < 1 || params->d > 3 || params->max_iter < 0) return SGT_ERR_UNSUPPORTED;
  if (params->relayout_every > 0 || params->kl_every > 0) return SGT_ERR_UNSUPPORTED;
  std::unique_ptr<Request> r(new Request());
  r->p = *params;
  // the locality order's creation cost (diffusion steps, relabelling) runs in
  // the admission thread, under the load of the running jobs, and delays
  // every admission behind it more than its faster SpMV gains over one
  // request; it pays off for a single very large embedding only
  if (n < SGT_SERVE_ORDER_MIN_N) r->p.locality_order = 0;
  r->n = n;
  r->nnz = rowptr[n];
  r->rowptr = rowptr;
  r->col = col;
  r->val = val;
  r->y0 = y0;
  r->y_out = y_out;
  r->iters_total = params->max_iter;
  r->footprint = sgt_job_footprint(&r->p, n, r->nnz);
  if (r->footprint == 0 || r->footprint > srv->cfg.hbm_budget) return SGT_ERR_NO_MEMORY;
  std::lock_guard<std::mutex> lk(srv->mu);
  if (srv->stop) return SGT_ERR_INVALID_ARG;
  r->id = (long long)srv->reqs.size();
  r->t_submit = srv->now();
  *id = r->id;
  srv->waiting.push_back(r.get());
  srv->reqs.push_back(std::move(r));
  srv->cv_admit.notify_all();
  return SGT_OK;
}

sgt_status sgt_server_poll(sgt_server *srv, double wait_ms, long long *ids, int cap, int *count) {
  if (!srv || !count || cap < 0 || (cap > 0 && !ids)) return SGT_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(srv->mu);
  if (srv->finished.empty() && wait_ms > 0)
    srv->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(wait_ms),
                          [&] { return !srv->finished.empty(); });
  int c = 0;
  while (c < cap && !srv->finished.empty()) {
    ids[c++] = srv->finished.front();
    srv->finished.pop_front();
  }
  *count = c;
  return SGT_OK;
}

sgt_status sgt_server_request_info(sgt_server *srv, long long id, sgt_request_info *info) {
  if (!srv || !info) return SGT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(srv->mu);
  if (id < 0 || id >= (long long)srv->reqs.size()) return SGT_ERR_INVALID_ARG;
  const Request *r = srv->reqs[(size_t)id].get();
  info->state = r->state;
  info->status = r->status;
  info->n = r->n;
  info->d = r->p.d;
  info->iters = r->iters_total;
  info->footprint = r->footprint;
  info->t_submit = r->t_submit;
  info->t_admit = r->t_admit;
  info->t_done = r->t_done;
  return SGT_OK;
}

double sgt_server_now(const sgt_server *srv) { return srv ? srv->now() : 0.0; }

}  // extern "C"
