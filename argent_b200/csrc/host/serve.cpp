// serve.cpp — continuous batching of render requests over one context.
//
// argent's serve renders final stills one job at a time: render_pass in
// chunks sized for about 1.5 s, seed 7, sample indices continuing across
// chunks, a cancel check between chunks (crates/argent/src/serve/queue.rs:
// 599-617); the live preview runs progressive passes of its own
// (serve/live.rs:747,767).  Here every request in flight advances together:
// each step is one argent_render_batch in which the active requests, most
// urgent first, take chunks of samples up to the step's path-sample budget.
// A request's film receives exactly the sample indices a single
// render_pass of `spp` samples would, in chunks (render.rs:70,86).
//
// Order: a request's urgency is its priority minus its waiting time over
// the aging period (so a final that has waited long outranks a fresh
// preview), ties by ticket.  Admission: queued requests enter the active set
// in that order while the active set is below max_active and their films
// fit in the film budget; films come from a pool keyed by (width, height,
// flags).
//
// Chunks: the step's budget of path-samples grows with the work pending
// (a quarter of it, between step_path_samples and step_path_samples_max), so a
// deep queue runs in larger, more efficient batches.  Requests whose
// remaining work is under a sixteenth of the budget finish in this step (up
// to half the budget); the rest goes to the other active requests strictly
// in urgency order, so large requests render one or two at a time at the
// device's full rate, near first come first served, instead of all sharing
// it.  Aging keeps any request from waiting for ever.
//
// Bound: with max_pending set, a submit that finds that many requests
// queued or active is refused with ARGENT_E_BUSY (argent's queue refuses a
// job when 24 are waiting, serve/queue.rs:28,364-366); with
// max_pending_path_samples, one that would take the work still to render
// past that bound is refused too (unless nothing of its priority is
// pending), which bounds every admitted request's wait when requests arrive
// faster than the device renders them.
//
// Threads: submit, poll and cancel lock the queue and may be called from
// any thread.  step and read drive the context and belong to the thread
// that owns it (a context is single-stream and not thread-safe).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../../../include/argent_gpu.h"
#include "overlap.h"

namespace {

struct Request {
  uint64_t ticket;
  ArgentServeRequest req;
  int32_t state;
  uint32_t samples;    // finished
  uint32_t scheduled;  // issued: finished or in a batch in flight
  uint32_t in_flight;  // batches in flight that hold a chunk of it
  bool cancel;
  ArgentFilm* film;
  uint64_t film_bytes;
  double t_submit, t_start, t_done;
};

uint64_t film_bytes(uint32_t w, uint32_t h, uint32_t flags) {
  if (flags == 0) flags = ARGENT_FILM_KAHAN;
  uint64_t per = 12 + ((flags & ARGENT_FILM_KAHAN) ? 4 : 0) + ((flags & ARGENT_FILM_FP64) ? 8 : 0);
  return 3ull * w * h * per;
}

}  // namespace

struct ArgentServe {
  ArgentCtx* ctx;
  ArgentServeConfig cfg;
  std::mutex mu;
  uint64_t next_ticket = 1;
  std::map<uint64_t, Request> reqs;  // ticket order = submission order
  uint64_t film_in_use = 0;
  std::map<std::tuple<uint32_t, uint32_t, uint32_t>, std::vector<ArgentFilm*>> pool;
  uint64_t pool_bytes = 0;
  std::chrono::steady_clock::time_point t0;
  uint64_t steps = 0, path_samples = 0, rejected = 0;
  // Batches in flight, oldest first: completion event and (ticket, samples).
  struct Batch {
    cudaEvent_t done;
    std::vector<std::pair<uint64_t, uint32_t>> parts;
  };
  std::deque<Batch> flight;
  std::vector<cudaEvent_t> idle_events;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

// A pooled film, cleared; nullptr and an error code if allocation fails.
int take_film(ArgentServe* s, const ArgentServeRequest& r, ArgentFilm** out) {
  auto key = std::make_tuple(r.width, r.height, r.film_flags);
  auto it = s->pool.find(key);
  if (it != s->pool.end() && !it->second.empty()) {
    ArgentFilm* f = it->second.back();
    it->second.pop_back();
    s->pool_bytes -= film_bytes(r.width, r.height, r.film_flags);
    int rc = argent_film_clear(f);
    if (rc != ARGENT_OK) {
      argent_film_destroy(f);
      return rc;
    }
    *out = f;
    return ARGENT_OK;
  }
  return argent_film_create(s->ctx, r.width, r.height, r.film_flags, out);
}

// Films in use and pooled films together stay within the film budget; a
// released film goes back to the pool (its bytes move from in-use to pooled).
void give_film(ArgentServe* s, Request& q) {
  if (!q.film) return;
  s->pool[std::make_tuple(q.req.width, q.req.height, q.req.film_flags)].push_back(q.film);
  s->pool_bytes += q.film_bytes;
  s->film_in_use -= q.film_bytes;
  q.film = nullptr;
}

void drain_pool(ArgentServe* s) {
  for (auto& kv : s->pool)
    for (ArgentFilm* f : kv.second) argent_film_destroy(f);
  s->pool.clear();
  s->pool_bytes = 0;
}

bool pooled(ArgentServe* s, const ArgentServeRequest& r) {
  auto it = s->pool.find(std::make_tuple(r.width, r.height, r.film_flags));
  return it != s->pool.end() && !it->second.empty();
}

double urgency(const Request* q, double now, double aging_s) {
  return (double)q->req.priority - (now - q->t_submit) / aging_s;
}

void sort_urgent_first(std::vector<Request*>& v, double now, double aging_s) {
  std::sort(v.begin(), v.end(), [&](const Request* a, const Request* b) {
    double ua = urgency(a, now, aging_s), ub = urgency(b, now, aging_s);
    if (ua != ub) return ua < ub;
    return a->ticket < b->ticket;
  });
}

// Path-samples not yet issued.
uint64_t remaining(const Request* q) {
  return (uint64_t)(q->req.spp - q->scheduled) * q->req.width * q->req.height;
}

// Applies finished batches in order: waits for the oldest when `wait`,
// otherwise takes only those already done.  Returns the first failure.
int retire(ArgentServe* s, bool wait) {
  int rc = ARGENT_OK;
  while (!s->flight.empty()) {
    ArgentServe::Batch& b = s->flight.front();
    cudaError_t e = wait ? cudaEventSynchronize(b.done) : cudaEventQuery(b.done);
    if (e == cudaErrorNotReady) break;
    wait = false;
    int st = e == cudaSuccess ? ARGENT_OK : ARGENT_E_CUDA;
    if (st == ARGENT_OK) st = ctx_check_status(s->ctx);
    if (st != ARGENT_OK && rc == ARGENT_OK) rc = st;
    std::lock_guard<std::mutex> g(s->mu);
    double t = s->now();
    for (auto& part : b.parts) {
      auto it = s->reqs.find(part.first);
      if (it == s->reqs.end()) continue;
      Request& q = it->second;
      --q.in_flight;
      if (st != ARGENT_OK) {
        if (q.state == ARGENT_REQ_ACTIVE) {
          q.state = ARGENT_REQ_FAILED;
          q.t_done = t;
        }
      } else {
        q.samples += part.second;
        s->path_samples += (uint64_t)part.second * q.req.width * q.req.height;
        if (q.state == ARGENT_REQ_ACTIVE && q.samples >= q.req.spp) {
          q.state = ARGENT_REQ_DONE;
          q.t_done = t;
        }
      }
      if (q.in_flight == 0 && q.state == ARGENT_REQ_FAILED) give_film(s, q);
    }
    s->idle_events.push_back(b.done);
    s->flight.pop_front();
  }
  return rc;
}

}  // namespace

extern "C" {

int argent_serve_create(ArgentCtx* ctx, const ArgentServeConfig* cfg, ArgentServe** out) {
  if (!ctx || !out) return ARGENT_E_INVALID;
  *out = nullptr;
  ArgentServe* s = new (std::nothrow) ArgentServe();
  if (!s) return ARGENT_E_OOM;
  s->ctx = ctx;
  std::memset(&s->cfg, 0, sizeof(s->cfg));
  if (cfg) s->cfg = *cfg;
  if (s->cfg.film_budget == 0) s->cfg.film_budget = 8ull << 30;
  if (s->cfg.max_active == 0) s->cfg.max_active = 64;
  if (s->cfg.step_path_samples == 0) s->cfg.step_path_samples = 1ull << 26;
  if (s->cfg.aging_ms == 0) s->cfg.aging_ms = 250;
  if (s->cfg.step_path_samples_max == 0) s->cfg.step_path_samples_max = 2 * s->cfg.step_path_samples;
  s->cfg.step_path_samples_max = std::max(s->cfg.step_path_samples_max, s->cfg.step_path_samples);
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return ARGENT_OK;
}

void argent_serve_destroy(ArgentServe* s) {
  if (!s) return;
  argent_ctx_sync(s->ctx);
  for (auto& b : s->flight) cudaEventDestroy(b.done);
  for (cudaEvent_t e : s->idle_events) cudaEventDestroy(e);
  for (auto& kv : s->reqs)
    if (kv.second.film) argent_film_destroy(kv.second.film);
  drain_pool(s);
  delete s;
}

double argent_serve_now(ArgentServe* s) { return s ? s->now() : 0.0; }

int argent_serve_submit(ArgentServe* s, const ArgentServeRequest* req, uint64_t* ticket) {
  if (!s || !req || !ticket) return ARGENT_E_INVALID;
  if (!req->scene || req->width == 0 || req->height == 0 || req->spp == 0 ||
      (uint64_t)req->width * req->height > (1ull << 31) || !scene_belongs(req->scene, s->ctx) ||
      req->settings.max_depth > 64)
    return ARGENT_E_INVALID;
  uint64_t fb = film_bytes(req->width, req->height, req->film_flags);
  if (fb > s->cfg.film_budget) return ARGENT_E_BUSY;
  std::lock_guard<std::mutex> g(s->mu);
  if (s->cfg.max_pending || s->cfg.max_pending_path_samples) {
    // A bounded queue, as argent's (queue.rs:364-366): refuse rather than
    // let the wait of every admitted request grow without bound.  The bound
    // counts requests, or the work they still need, or both.
    uint32_t n = 0, same = 0;
    uint64_t work = 0;
    for (auto& kv : s->reqs)
      if (kv.second.state == ARGENT_REQ_QUEUED || kv.second.state == ARGENT_REQ_ACTIVE) {
        ++n;
        work += remaining(&kv.second);
        if (kv.second.req.priority == req->priority) ++same;
      }
    uint64_t mine = (uint64_t)req->spp * req->width * req->height;
    // The work bound spares a request whose priority level has nothing
    // pending, so the largest requests are never all refused while the
    // small ones keep the pending work near the bound.
    bool busy = (s->cfg.max_pending && n >= s->cfg.max_pending) ||
                (s->cfg.max_pending_path_samples && same > 0 &&
                 work + mine > s->cfg.max_pending_path_samples);
    if (busy) {
      ++s->rejected;
      return ARGENT_E_BUSY;
    }
  }
  Request q;
  std::memset(&q, 0, sizeof(q));
  q.ticket = s->next_ticket++;
  q.req = *req;
  q.state = ARGENT_REQ_QUEUED;
  q.film_bytes = fb;
  q.t_submit = s->now();
  q.t_start = q.t_done = -1.0;
  s->reqs.emplace(q.ticket, q);
  *ticket = q.ticket;
  return ARGENT_OK;
}

int argent_serve_poll(ArgentServe* s, uint64_t ticket, ArgentServeStatus* st) {
  if (!s || !st) return ARGENT_E_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return ARGENT_E_INVALID;
  const Request& q = it->second;
  st->state = q.state;
  st->samples = q.samples;
  st->spp = q.req.spp;
  st->t_submit = q.t_submit;
  st->t_start = q.t_start;
  st->t_done = q.t_done;
  return ARGENT_OK;
}

int argent_serve_cancel(ArgentServe* s, uint64_t ticket) {
  if (!s) return ARGENT_E_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return ARGENT_E_INVALID;
  if (it->second.state == ARGENT_REQ_QUEUED || it->second.state == ARGENT_REQ_ACTIVE) it->second.cancel = true;
  return ARGENT_OK;
}

int argent_serve_step(ArgentServe* s, uint32_t* pending) {
  if (!s) return ARGENT_E_INVALID;
  int rc = retire(s, false);
  std::vector<ArgentBatchItem> items;
  std::vector<Request*> in_batch;
  std::vector<uint32_t> chunk;
  {
    std::lock_guard<std::mutex> g(s->mu);
    // Cancellations take effect between batches, as in queue.rs:605-608,
    // once none of the request's batches is in flight.
    for (auto& kv : s->reqs) {
      Request& q = kv.second;
      if (q.cancel && q.in_flight == 0 && (q.state == ARGENT_REQ_QUEUED || q.state == ARGENT_REQ_ACTIVE)) {
        give_film(s, q);
        q.state = ARGENT_REQ_CANCELLED;
        q.t_done = s->now();
      }
    }
    std::vector<Request*> active, queued;
    for (auto& kv : s->reqs) {
      if (kv.second.state == ARGENT_REQ_ACTIVE) active.push_back(&kv.second);
      if (kv.second.state == ARGENT_REQ_QUEUED) queued.push_back(&kv.second);
    }
    const double now = s->now(), aging_s = s->cfg.aging_ms * 1e-3;
    sort_urgent_first(queued, now, aging_s);
    for (Request* q : queued) {
      if (active.size() >= s->cfg.max_active) break;
      if (!pooled(s, q->req) && s->film_in_use + s->pool_bytes + q->film_bytes > s->cfg.film_budget) {
        // Free the pooled films of other sizes before refusing admission.
        drain_pool(s);
        if (s->film_in_use + q->film_bytes > s->cfg.film_budget) break;
      }
      int frc = take_film(s, q->req, &q->film);
      if (frc != ARGENT_OK) {
        q->state = ARGENT_REQ_FAILED;
        q->t_done = s->now();
        continue;
      }
      s->film_in_use += q->film_bytes;
      q->state = ARGENT_REQ_ACTIVE;
      q->t_start = s->now();
      active.push_back(q);
    }
    sort_urgent_first(active, now, aging_s);
    uint64_t pending_work = 0;
    for (auto& kv : s->reqs)
      if (kv.second.state == ARGENT_REQ_QUEUED || kv.second.state == ARGENT_REQ_ACTIVE)
        pending_work += remaining(&kv.second);
    const uint64_t budget =
        std::min(s->cfg.step_path_samples_max, std::max(s->cfg.step_path_samples, pending_work / 4));
    // Small requests (at most a sixteenth of the budget left) finish in
    // this step, in urgency order, up to half the budget; the rest of the
    // budget goes to the other requests strictly in urgency order, so the
    // most urgent large request renders at the device's full rate instead
    // of sharing it with every other one (which would make each large
    // request wait for all of them).  A request reached with no budget left
    // waits for a later step; its urgency grows while it waits.
    std::vector<std::pair<Request*, uint32_t>> take;
    uint64_t left = budget;
    const uint64_t small_cap = budget / 2;
    uint64_t small_used = 0;
    for (Request* q : active) {
      if (q->cancel || q->scheduled >= q->req.spp) continue;
      uint64_t r = remaining(q);
      if (r <= budget / 16 && small_used + r <= small_cap) {
        take.emplace_back(q, q->req.spp - q->scheduled);
        small_used += r;
      }
    }
    left -= small_used;
    for (Request* q : active) {
      if (q->cancel || q->scheduled >= q->req.spp) continue;
      bool taken = false;
      for (auto& t : take) taken = taken || t.first == q;
      if (taken) continue;
      uint64_t px = (uint64_t)q->req.width * q->req.height;
      uint64_t want = q->req.spp - q->scheduled;
      uint64_t n = std::min<uint64_t>(want, left / px);
      // A request larger than the whole budget still advances when it is
      // the first one this step reaches.
      if (n == 0 && take.empty()) n = 1;
      if (n == 0) continue;
      take.emplace_back(q, (uint32_t)n);
      left = n * px >= left ? 0 : left - n * px;
    }
    for (auto& t : take) {
      Request* q = t.first;
      uint64_t n = t.second;
      ArgentBatchItem it;
      std::memset(&it, 0, sizeof(it));
      it.scene = q->req.scene;
      it.camera = q->req.camera;
      it.film = q->film;
      it.settings = q->req.settings;
      it.count = (uint32_t)n;
      it.seed = q->req.seed;
      items.push_back(it);
      in_batch.push_back(q);
      chunk.push_back((uint32_t)n);
    }
  }
  if (!items.empty()) {
    cudaEvent_t done = nullptr;
    if (!s->idle_events.empty()) {
      done = s->idle_events.back();
      s->idle_events.pop_back();
    } else if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) != cudaSuccess) {
      done = nullptr;
    }
    int brc = done ? render_batch_overlapped(s->ctx, items.data(), (uint32_t)items.size(), done) : ARGENT_E_CUDA;
    std::lock_guard<std::mutex> g(s->mu);
    if (brc == ARGENT_OK) {
      ArgentServe::Batch b;
      b.done = done;
      for (size_t i = 0; i < in_batch.size(); ++i) {
        in_batch[i]->scheduled += chunk[i];
        ++in_batch[i]->in_flight;
        b.parts.emplace_back(in_batch[i]->ticket, chunk[i]);
      }
      s->flight.push_back(std::move(b));
      ++s->steps;
    } else {
      if (done) s->idle_events.push_back(done);
      double t = s->now();
      for (Request* q : in_batch) {
        q->state = ARGENT_REQ_FAILED;
        q->t_done = t;
      }
      if (rc == ARGENT_OK) rc = brc;
    }
  }
  if (rc != ARGENT_OK) {
    // After a failure nothing stays in flight: wait for every batch.
    argent_ctx_sync(s->ctx);
    int r2 = retire(s, false);
    (void)r2;
  } else {
    // Without overlap wait for this step's batch; with it, for the older
    // of two in flight (or for the one in flight when nothing was issued).
    size_t depth = s->cfg.overlap ? 2 : 1;
    if (s->flight.size() >= depth || (items.empty() && !s->flight.empty())) rc = retire(s, true);
  }
  std::lock_guard<std::mutex> g(s->mu);
  for (auto& kv : s->reqs)
    if (kv.second.state == ARGENT_REQ_FAILED && kv.second.in_flight == 0) give_film(s, kv.second);
  if (pending) {
    uint32_t n = 0;
    for (auto& kv : s->reqs)
      if (kv.second.state == ARGENT_REQ_QUEUED || kv.second.state == ARGENT_REQ_ACTIVE) ++n;
    *pending = n;
  }
  return rc;
}

int argent_serve_read(ArgentServe* s, uint64_t ticket, float* color, float* albedo, float* normal) {
  if (!s) return ARGENT_E_INVALID;
  ArgentFilm* f = nullptr;
  {
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || it->second.state != ARGENT_REQ_DONE || !it->second.film) return ARGENT_E_INVALID;
    f = it->second.film;
  }
  int rc = argent_film_read(f, color, albedo, normal);
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  give_film(s, it->second);
  s->reqs.erase(it);
  return rc;
}

int argent_serve_release(ArgentServe* s, uint64_t ticket) {
  if (!s) return ARGENT_E_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return ARGENT_E_INVALID;
  Request& q = it->second;
  if (q.state == ARGENT_REQ_QUEUED || q.state == ARGENT_REQ_ACTIVE) return ARGENT_E_INVALID;
  if (q.in_flight > 0) return ARGENT_E_BUSY;  // a failed request's batch still runs
  give_film(s, q);
  s->reqs.erase(it);
  return ARGENT_OK;
}

int argent_serve_stats(ArgentServe* s, uint64_t* steps, uint64_t* path_samples, uint64_t* film_bytes_in_use) {
  if (!s) return ARGENT_E_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  if (steps) *steps = s->steps;
  if (path_samples) *path_samples = s->path_samples;
  if (film_bytes_in_use) *film_bytes_in_use = s->film_in_use;
  return ARGENT_OK;
}

}  // extern "C"
