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
// Admission: queued requests enter the active set in (priority, ticket)
// order while the active set is below max_active and their films fit in the
// film budget; films come from a pool keyed by (width, height, flags).
//
// Threads: submit, poll and cancel lock the queue and may be called from
// any thread.  step and read drive the context and belong to the thread
// that owns it (a context is single-stream and not thread-safe).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../../../include/argent_gpu.h"

namespace {

struct Request {
  uint64_t ticket;
  ArgentServeRequest req;
  int32_t state;
  uint32_t samples;
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
  uint64_t steps = 0, path_samples = 0;

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

bool urgent_first(const Request* a, const Request* b) {
  if (a->req.priority != b->req.priority) return a->req.priority < b->req.priority;
  return a->ticket < b->ticket;
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
  if (s->cfg.step_path_samples == 0) s->cfg.step_path_samples = 1ull << 25;
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return ARGENT_OK;
}

void argent_serve_destroy(ArgentServe* s) {
  if (!s) return;
  for (auto& kv : s->reqs)
    if (kv.second.film) argent_film_destroy(kv.second.film);
  drain_pool(s);
  delete s;
}

double argent_serve_now(ArgentServe* s) { return s ? s->now() : 0.0; }

int argent_serve_submit(ArgentServe* s, const ArgentServeRequest* req, uint64_t* ticket) {
  if (!s || !req || !ticket) return ARGENT_E_INVALID;
  if (!req->scene || req->width == 0 || req->height == 0 || req->spp == 0 ||
      (uint64_t)req->width * req->height > (1ull << 31))
    return ARGENT_E_INVALID;
  uint64_t fb = film_bytes(req->width, req->height, req->film_flags);
  if (fb > s->cfg.film_budget) return ARGENT_E_BUSY;
  std::lock_guard<std::mutex> g(s->mu);
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
  std::vector<ArgentBatchItem> items;
  std::vector<Request*> in_batch;
  std::vector<uint32_t> chunk;
  {
    std::lock_guard<std::mutex> g(s->mu);
    // Cancellations take effect between batches, as in queue.rs:605-608.
    for (auto& kv : s->reqs) {
      Request& q = kv.second;
      if (q.cancel && (q.state == ARGENT_REQ_QUEUED || q.state == ARGENT_REQ_ACTIVE)) {
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
    std::sort(queued.begin(), queued.end(), urgent_first);
    for (Request* q : queued) {
      if (active.size() >= s->cfg.max_active) break;
      if (!pooled(s, q->req) && s->film_in_use + s->pool_bytes + q->film_bytes > s->cfg.film_budget) {
        // Free the pooled films of other sizes before refusing admission.
        drain_pool(s);
        if (s->film_in_use + q->film_bytes > s->cfg.film_budget) break;
      }
      int rc = take_film(s, q->req, &q->film);
      if (rc != ARGENT_OK) {
        q->state = ARGENT_REQ_FAILED;
        q->t_done = s->now();
        continue;
      }
      s->film_in_use += q->film_bytes;
      q->state = ARGENT_REQ_ACTIVE;
      q->t_start = s->now();
      active.push_back(q);
    }
    std::sort(active.begin(), active.end(), urgent_first);
    // Chunks: the most urgent requests first, each as many whole samples of
    // its frame as the step's budget leaves (at least one for the first).
    uint64_t left = s->cfg.step_path_samples;
    for (Request* q : active) {
      uint64_t px = (uint64_t)q->req.width * q->req.height;
      uint64_t want = q->req.spp - q->samples;
      uint64_t n = std::min<uint64_t>(want, left / px);
      if (n == 0) {
        if (!items.empty()) break;
        n = 1;
      }
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
      left = n * px >= left ? 0 : left - n * px;
      if (left == 0) break;
    }
  }
  int rc = ARGENT_OK;
  if (!items.empty()) {
    rc = argent_render_batch(s->ctx, items.data(), (uint32_t)items.size());
    if (rc == ARGENT_OK) rc = argent_ctx_sync(s->ctx);
  }
  std::lock_guard<std::mutex> g(s->mu);
  double t = s->now();
  for (size_t i = 0; i < in_batch.size(); ++i) {
    Request* q = in_batch[i];
    if (rc != ARGENT_OK) {
      q->state = ARGENT_REQ_FAILED;
      q->t_done = t;
      give_film(s, *q);
      continue;
    }
    q->samples += chunk[i];
    s->path_samples += (uint64_t)chunk[i] * q->req.width * q->req.height;
    if (q->samples >= q->req.spp) {
      q->state = ARGENT_REQ_DONE;
      q->t_done = t;
    }
  }
  if (!items.empty()) ++s->steps;
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
