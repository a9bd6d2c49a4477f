// rte_server.cpp -- continuous-batching request server for forward solves on one GPU.
//
// Requests of any grid size, SH order, medium and sources arrive at any time (rte_server_submit).
// A scheduler admits them as execution slots and HBM free up: a request takes an idle context of
// its shape (grid, order, precision) when one exists, otherwise a new context is made if its HBM
// footprint fits the budget (idle contexts of other shapes are evicted, least recently used
// first, to make room).  Every context owns a CUDA stream, so admitted requests run concurrently
// on the device; each context replays one CUDA graph per shape for the Neumann series
// (rte_forward_graph) and keeps its medium, pair kernel and partial sums resident.  A request
// that does not fit now waits while later ones that do fit go ahead.  Latency is measured from
// submit to completion.  Nothing here calls exit(); waits are bounded by the caller's timeout.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rte_b200.h"
#include "rte_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  long long id = 0;
  rte_request rq;
  std::vector<double> mua, mus;
  std::vector<rte_cplx> trans, ref;
  Clock::time_point t_submit, t_start, t_done;
  int status = RTE_OK;
  std::string msg;  // why the request failed, handed to the waiting thread's rte_last_error(NULL)
  bool started = false, done = false, cancelled = false;
  double device_ms = 0.0;
};

struct ShapeKey {
  int n, L, prec;
  double dx, g, nidx;
  bool operator==(const ShapeKey& o) const {
    return n == o.n && L == o.L && prec == o.prec && dx == o.dx && g == o.g && nidx == o.nidx;
  }
};

struct Slot {
  rte_ctx* ctx = nullptr;  // made by the first worker that uses the slot
  ShapeKey key;
  size_t bytes = 0;
  bool busy = false;
  Clock::time_point last;
};

ShapeKey key_of(const rte_request& r) { return ShapeKey{r.n, r.nL, r.precision, r.dx, r.g, r.n_index}; }

// HBM of a context of this shape: distributions, split-K partials, batch buffers and, for the
// mixed precision path, the stored FP32 pair kernel (N x N).
size_t estimate_bytes(const ShapeKey& k, int nsrc) {
  const size_t N = (size_t)k.n * k.n * k.n, C = (size_t)(k.L + 1) * (k.L + 1);
  const size_t nb = nsrc == 1 ? 1 : (nsrc <= 2 ? 2 : 4);
  size_t b = 8 * N * C * (24 + 14 * nb) + (64ull << 20);
  if (k.prec == RTE_PREC_MIXED) {
    b += 4 * ((N + 127) / 128 * 128) * ((N + 31) / 32 * 32);  // stored pair kernel (128-destination blocks)
    b += 8 * N * C * nb * ((N + 1023) / 1024 + 8);            // partial sums of 1024-source chunks
  }
  return b;
}

}  // namespace

struct rte_server {
  int device = 0;
  size_t budget = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> pending;
  std::map<long long, std::unique_ptr<Req>> reqs;
  std::vector<std::unique_ptr<Slot>> slots;
  size_t used = 0;
  long long next_id = 1;
  bool stopping = false;
  std::vector<std::thread> workers;
  long long n_submitted = 0, n_completed = 0, n_failed = 0, n_cancelled = 0;
  std::vector<double> latencies;  // completed requests, ms
  Clock::time_point t_first, t_last;
  bool have_first = false;
  int inflight = 0;
  std::string err;
};

// Slot for r, or nullptr (wait) / (Slot*)1 (never fits).  Caller holds s->mu.
static Slot* admit(rte_server* s, Req* r) {
  const ShapeKey k = key_of(r->rq);
  for (auto& sl : s->slots)
    if (!sl->busy && sl->key == k) return sl.get();
  const size_t need = estimate_bytes(k, r->rq.nsrc);
  if (need > s->budget) return (Slot*)1;
  while (s->used + need > s->budget) {  // evict idle contexts, least recently used first
    int lru = -1;
    for (size_t q = 0; q < s->slots.size(); q++)
      if (!s->slots[q]->busy && (lru < 0 || s->slots[q]->last < s->slots[lru]->last)) lru = (int)q;
    if (lru < 0) return nullptr;
    if (s->slots[lru]->ctx) rte_destroy(s->slots[lru]->ctx);
    s->used -= s->slots[lru]->bytes;
    s->slots.erase(s->slots.begin() + lru);
  }
  std::unique_ptr<Slot> sl(new Slot);
  sl->key = k;
  sl->bytes = need;
  s->used += need;
  s->slots.push_back(std::move(sl));
  return s->slots.back().get();
}

static rte_ctx* make_ctx(const rte_server* s, const ShapeKey& key, int* rc) {
  rte_config cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.nx = cfg.ny = cfg.nz = key.n;
  cfg.x_min = -key.n * key.dx / 2;
  cfg.x_max = key.n * key.dx / 2;
  cfg.y_min = -key.n * key.dx / 2;
  cfg.y_max = key.n * key.dx / 2;
  cfg.z_min = 0;
  cfg.z_max = key.n * key.dx;
  cfg.nL = key.L;
  cfg.prop_thresh = 4.0 * key.n * key.dx;  // every pair couples
  cfg.self_sub_vox = 1;
  cfg.g = key.g;
  cfg.n = key.nidx;
  cfg.c = 1.0;
  cfg.model = RTE_MODEL_EXACT;
  cfg.precision = key.prec;
  cfg.kernel_mode = RTE_KERNEL_AUTO;  // stored pair kernel when it fits; uniform media by FFT
  cfg.device = s->device;
  rte_ctx* ctx = nullptr;
  *rc = rte_create(&cfg, &ctx);
  return *rc == RTE_OK ? ctx : nullptr;
}

static void worker_main(rte_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    Req* r = nullptr;
    Slot* sl = nullptr;
    s->cv_work.wait(lk, [&] {
      if (s->stopping) return true;
      for (auto it = s->pending.begin(); it != s->pending.end();) {
        Slot* q = admit(s, *it);
        if (q == (Slot*)1) {  // larger than the whole budget: it can never run
          char m[160];
          snprintf(m, sizeof m, "request needs %.2f GB of HBM, the server's budget is %.2f GB",
                   estimate_bytes(key_of((*it)->rq), (*it)->rq.nsrc) / 1e9, s->budget / 1e9);
          (*it)->msg = m;
          (*it)->status = RTE_ERR_NOMEM;
          (*it)->done = true;
          (*it)->t_done = Clock::now();
          s->n_failed++;
          it = s->pending.erase(it);
          s->cv_done.notify_all();
          continue;
        }
        if (q) {
          r = *it;
          sl = q;
          s->pending.erase(it);
          return true;
        }
        ++it;
      }
      return false;
    });
    if (!r) return;  // stopping
    sl->busy = true;
    r->started = true;
    r->t_start = Clock::now();
    s->inflight++;
    lk.unlock();
    int rc = RTE_OK;
    if (!sl->ctx) sl->ctx = make_ctx(s, sl->key, &rc);
    if (rc != RTE_OK) r->msg = rte_last_error(nullptr);  // rte_create's message (this thread's)
    if (rc == RTE_OK) rc = rte_set_medium_voxel(sl->ctx, r->mua.data(), r->mus.data());
    if (rc == RTE_OK) {
      rte_report rep;
      r->trans.assign((size_t)r->rq.nsrc * r->rq.n * r->rq.n, rte_cplx{0, 0});
      r->ref.assign(r->trans.size(), rte_cplx{0, 0});
      (void)cudaGetLastError();  // a handled failure of an earlier request on this thread is not this one's
      rc = rte_forward_graph(sl->ctx, r->rq.nsrc, r->rq.src, r->rq.terms, r->trans.data(), r->ref.data(), &rep);
      r->device_ms = rep.ms_device;
    }
    lk.lock();
    if (rc != RTE_OK && sl->ctx) {  // a failed context is not reused
      s->err = rte_last_error(sl->ctx);
      r->msg = s->err;
      rte_destroy(sl->ctx);
      sl->ctx = nullptr;
    }
    r->status = rc;
    sl->busy = false;
    sl->last = Clock::now();
    s->inflight--;
    r->t_done = Clock::now();
    r->done = true;
    if (rc == RTE_OK) {
      s->n_completed++;
      s->latencies.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
      s->t_last = r->t_done;
    } else {
      s->n_failed++;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

extern "C" {

int rte_server_create(int device, double hbm_budget_gb, int nworkers, rte_server** out) {
  if (!out || nworkers < 1 || nworkers > 64) {
    rte_set_global_error("rte_server_create: null output or nworkers outside 1..64");
    return RTE_ERR_ARG;
  }
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  size_t fr = 0, tot = 0;
  if (e == cudaSuccess) e = cudaMemGetInfo(&fr, &tot);
  if (e != cudaSuccess) {
    rte_set_global_error(cudaGetErrorString(e));
    return RTE_ERR_DEVICE;
  }
  rte_server* s = new rte_server;
  s->device = device;
  s->budget = hbm_budget_gb > 0 ? (size_t)(hbm_budget_gb * 1e9) : (size_t)(0.85 * (double)fr);
  for (int q = 0; q < nworkers; q++) s->workers.emplace_back(worker_main, s);
  *out = s;
  return RTE_OK;
}

int rte_server_submit(rte_server* s, const rte_request* rq, long long* ticket) {
  if (!s || !rq || !ticket || !rq->mua || !rq->mus) {
    rte_set_global_error("rte_server_submit: null argument");
    return RTE_ERR_ARG;
  }
  if (rq->n < 2 || rq->n > 256 || rq->nL < 0 || rq->nL > 7 || rq->nsrc < 1 || rq->nsrc > 4 || rq->terms < 0 ||
      !(rq->dx > 0)) {
    rte_set_global_error("rte_server_submit: n outside 2..256, nL outside 0..7, nsrc outside 1..4, terms < 0 or dx <= 0");
    return RTE_ERR_ARG;
  }
  std::unique_ptr<Req> r(new Req);
  r->rq = *rq;
  const size_t N = (size_t)rq->n * rq->n * rq->n;
  r->mua.assign(rq->mua, rq->mua + N);
  r->mus.assign(rq->mus, rq->mus + N);
  r->rq.mua = r->rq.mus = nullptr;
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->have_first) {
    s->t_first = r->t_submit;
    s->have_first = true;
  }
  r->id = s->next_id++;
  *ticket = r->id;
  s->pending.push_back(r.get());
  s->reqs[r->id] = std::move(r);
  s->n_submitted++;
  s->cv_work.notify_one();
  return RTE_OK;
}

int rte_server_wait(rte_server* s, long long ticket, double timeout_s, rte_cplx* trans, rte_cplx* ref,
                    rte_result_info* info) {
  if (!s) return RTE_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return RTE_ERR_ARG;
  Req* r = it->second.get();
  // negative or NaN: poll; +inf or beyond 1e8 s (about three years): 1e8 s, which keeps the
  // deadline inside the clock's range
  const double wait_s = std::isfinite(timeout_s) ? std::min(std::max(timeout_s, 0.0), 1e8) : (timeout_s > 0 ? 1e8 : 0.0);
  const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(wait_s));
  if (!s->cv_done.wait_until(lk, deadline, [&] { return r->done; })) return RTE_ERR_TIMEOUT;
  if (info) {
    info->status = r->status;
    info->latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    info->queue_ms = r->started ? std::chrono::duration<double, std::milli>(r->t_start - r->t_submit).count()
                                : info->latency_ms;
    info->service_ms = r->started ? std::chrono::duration<double, std::milli>(r->t_done - r->t_start).count() : 0.0;
    info->device_ms = r->device_ms;
  }
  if (r->status != RTE_OK) rte_set_global_error(r->msg.empty() ? "request cancelled" : r->msg.c_str());
  if (r->status == RTE_OK) {
    if (trans) memcpy(trans, r->trans.data(), r->trans.size() * sizeof(rte_cplx));
    if (ref) memcpy(ref, r->ref.data(), r->ref.size() * sizeof(rte_cplx));
  }
  const int st = r->status;
  s->reqs.erase(it);
  return st;
}

int rte_server_cancel(rte_server* s, long long ticket) {
  if (!s) return RTE_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return RTE_ERR_ARG;
  Req* r = it->second.get();
  if (r->started || r->done) return RTE_ERR_STATE;  // running work is not interrupted
  for (auto p = s->pending.begin(); p != s->pending.end(); ++p)
    if (*p == r) {
      s->pending.erase(p);
      break;
    }
  r->status = RTE_ERR_CANCELLED;
  r->cancelled = true;
  r->done = true;
  r->t_done = Clock::now();
  s->n_cancelled++;
  s->cv_done.notify_all();
  return RTE_OK;
}

int rte_server_stats(rte_server* s, rte_server_info* o) {
  if (!s || !o) return RTE_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(o, 0, sizeof *o);
  o->submitted = s->n_submitted;
  o->completed = s->n_completed;
  o->failed = s->n_failed;
  o->cancelled = s->n_cancelled;
  o->inflight = s->inflight;
  o->pending = (long long)s->pending.size();
  o->contexts = (int)s->slots.size();
  o->hbm_reserved = s->used;
  std::vector<double> l = s->latencies;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
    o->p50_ms = pct(0.50);
    o->p99_ms = pct(0.99);
    double m = 0;
    for (double x : l) m += x;
    o->mean_ms = m / l.size();
  }
  if (s->have_first && s->n_completed > 0) o->wall_s = std::chrono::duration<double>(s->t_last - s->t_first).count();
  return RTE_OK;
}

void rte_server_destroy(rte_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto& sl : s->slots)
    if (sl->ctx) rte_destroy(sl->ctx);
  delete s;
}

}  // extern "C"
