// Many independent instances on one GPU: a batch run to completion together
// and a request loop with admission against a device-memory budget. Neither
// has a counterpart in the reference (its driver runs one problem per
// process); both are written on the library's own C-ABI.
//
// Every instance is an eg_ctx with its own CUDA stream. Host worker threads
// advance instances through eg_stepper_*, so the kernels of different
// instances overlap on the GPU while each instance keeps its own kernels,
// reductions and control flow: a result is bitwise the one the instance gives
// alone.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/euler2d_cuda.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

eg_run_opts schedule(int steps, int newton_steps, double cfl, int form, int precond) {
  eg_run_opts ro{};
  ro.integrator = 0;
  ro.steps = steps;
  ro.newton_steps = newton_steps;
  ro.max_newton = 30;
  ro.dt = 1e-3;
  ro.cfl = cfl;
  ro.end = 0.2;
  ro.tol = 1e-12;
  ro.timing_only = 1;
  ro.save_solution = 0;
  ro.prefix = "run";
  ro.form_name = form == EG_FORM_DG ? "dg" : "hdg";
  ro.assembly_name = "partial";
  ro.solver_name = "gmres";
  ro.precond_name = precond == EG_PC_BLOCK_ILU0 ? "block-ilu0" : "block-jacobi";
  ro.ilu_ordering_name = "none";
  ro.check_update = 0;
  return ro;
}

// Runs one instance through its schedule; fills res (updates, timings,
// errors, drift). Returns the first failing status.
int run_schedule(eg_ctx *ctx, const eg_run_opts &ro, eg_run_result &res) {
  res = eg_run_result{};
  eg_stepper *st = nullptr;
  int rc = eg_stepper_create(ctx, &ro, &st);
  if (rc != EG_OK) return rc;
  eg_update_stats us{};
  int updates = 0;
  double newton_s = 0., device_ms = 0.;
  while ((rc = eg_stepper_next(st, &us)) == EG_OK) {
    ++updates;
    newton_s += us.iteration_s;
    device_ms += us.device_ms;
  }
  if (rc == -1) rc = eg_stepper_finish(st, &res);
  res.updates = updates;
  res.newton_seconds = newton_s;
  res.newton_device_ms = device_ms;
  res.mean_newton_s = updates ? newton_s / updates : 0.;
  eg_stepper_destroy(st);
  return rc;
}

}  // namespace

// ------------------------------------------------------------------ batch
struct eg_batch {
  int device = 0;
  std::vector<eg_ctx *> ctx;
  std::vector<eg_run_result> res;
  std::vector<int> status;
};

extern "C" {

int eg_batch_create(int count, const eg_desc *descs, const eg_opts *opts, int device, eg_batch **out) {
  if (count <= 0 || !descs || !opts || !out) return EG_ERR_INVALID;
  *out = nullptr;
  int rc = eg_set_device(device);
  if (rc != EG_OK) return rc;
  auto *b = new eg_batch();
  b->device = device;
  for (int i = 0; i < count; ++i) {
    eg_ctx *c = nullptr;
    rc = eg_create(&descs[i], &opts[i], &c);
    if (rc != EG_OK) {
      eg_batch_destroy(b);
      return rc;
    }
    b->ctx.push_back(c);
  }
  b->res.assign(count, eg_run_result{});
  b->status.assign(count, -1);
  *out = b;
  return EG_OK;
}

int eg_batch_run(eg_batch *b, const eg_run_opts *ro, int threads, eg_batch_stats *st) {
  if (!b || !ro) return EG_ERR_INVALID;
  const int count = (int)b->ctx.size();
  threads = std::max(1, std::min(threads, count));
  std::atomic<int> next{0};
  const double t0 = now_s();
  auto worker = [&] {
    eg_set_device(b->device);  // the device is current per host thread
    for (int i = next++; i < count; i = next++) b->status[i] = run_schedule(b->ctx[i], *ro, b->res[i]);
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
  if (st) {
    *st = eg_batch_stats{};
    st->seconds = now_s() - t0;
    for (int i = 0; i < count; ++i) {
      st->updates += b->res[i].updates;
      if (b->status[i] != EG_OK) ++st->failed;
    }
  }
  for (int i = 0; i < count; ++i)
    if (b->status[i] != EG_OK) return b->status[i];
  return EG_OK;
}

int eg_batch_result(const eg_batch *b, int i, int *status, eg_run_result *res) {
  if (!b || i < 0 || i >= (int)b->ctx.size()) return EG_ERR_INVALID;
  if (status) *status = b->status[i];
  if (res) *res = b->res[i];
  return EG_OK;
}

eg_ctx *eg_batch_context(eg_batch *b, int i) {
  if (!b || i < 0 || i >= (int)b->ctx.size()) return nullptr;
  return b->ctx[i];
}

void eg_batch_destroy(eg_batch *b) {
  if (!b) return;
  eg_set_device(b->device);
  for (eg_ctx *c : b->ctx) eg_destroy(c);
  delete b;
}

}  // extern "C"

// ----------------------------------------------------------------- server
namespace {

using ShapeKey = std::tuple<int, int, int, int, int, int>;  // nx, ny, k, form, precond, precision
ShapeKey shape_of(const eg_request &r) { return {r.nx, r.ny, r.k, r.form, r.precond, r.precision}; }

// Device bytes of a context of this shape after one schedule (the buffers
// eg_create, the first solve and the time loop allocate), for admission
// before the first context of the shape exists.
long long estimate_bytes(const eg_request &r) {
  const long long q = r.k + 1, p = q * q, m = 4 * p, t = 4 * q, n = (long long)r.nx * r.ny, nf = 2 * n;
  const long long nu = n * m, nl = nf * t, N = std::max(nu, nl), R = 20;
  long long d = 14 * nu + 5 * nf * q + N * (R + 1) + 6 * N + 2 * nl;
  if (r.form == EG_FORM_HDG) {
    d += n * m * (4 * t + 1) + n * 4 * q * 17 + n * 4 * t + n * (q >= 5 ? 16 : 4) * t * t + 4 * nl + nf * t * t +
         nf * t / 2;
    if (r.precision == EG_PRECISION_MIXED) d += (n * m * 4 * t + nf * t * t + nl * (R + 9) + n * 4 * t) / 2;
    if (r.precond == EG_PC_BLOCK_ILU0) d += 8 * nf * t * t + n * 16 * t * t;
  } else {
    d += n * m * m + n * m / 2;
    if (r.precond == EG_PC_BLOCK_ILU0) d += 6 * n * m * m;
  }
  return d * 8 + d * 8 / 50;  // 2% for small tables and workspaces
}

struct Job {
  eg_request req{};
  eg_request_result res{};
  bool done = false;
  std::vector<double> state;
};

}  // namespace

struct eg_server {
  eg_server_opts o{};
  double t0 = 0.;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::deque<long long> queue;
  std::unordered_map<long long, Job> jobs;
  long long next_id = 0;
  long long resident = 0;  // bytes of running requests and idle pooled contexts
  int running = 0;
  long long pending = 0;
  bool stop = false;
  eg_server_stats stats{};
  std::map<ShapeKey, long long> measured;  // bytes of contexts of a shape
  struct Idle {
    ShapeKey key;
    eg_ctx *ctx;
    long long bytes;
  };
  std::deque<Idle> idle;  // pooled contexts, oldest first
  std::vector<std::thread> threads;

  // Bytes charged to a request: the estimate, or what a context of its shape
  // was measured to hold when that is larger.
  long long charge(const eg_request &r) {
    const auto it = measured.find(shape_of(r));
    const long long est = estimate_bytes(r);
    return it != measured.end() ? std::max(est, it->second) : est;
  }
  // Destroy idle pooled contexts (oldest first) until `need` more bytes fit.
  // Called with the lock held; returns the contexts to destroy outside it.
  std::vector<eg_ctx *> evict_for(long long need) {
    std::vector<eg_ctx *> out;
    while (!idle.empty() && resident + need > o.budget_bytes) {
      resident -= idle.front().bytes;
      out.push_back(idle.front().ctx);
      idle.pop_front();
    }
    return out;
  }
  eg_ctx *take_idle(const ShapeKey &key, long long &bytes) {
    for (auto it = idle.begin(); it != idle.end(); ++it)
      if (it->key == key) {
        eg_ctx *c = it->ctx;
        bytes = it->bytes;
        idle.erase(it);
        return c;
      }
    return nullptr;
  }

  void worker() {
    eg_set_device(o.device);
    for (;;) {
      long long id = -1, charged = 0;
      eg_ctx *ctx = nullptr;
      std::vector<eg_ctx *> evicted;
      {
        std::unique_lock<std::mutex> lk(m);
        for (;;) {
          if (stop && queue.empty()) return;
          if (!queue.empty()) {
            Job &j = jobs[queue.front()];
            long long reuse_bytes = 0;
            eg_ctx *reuse = take_idle(shape_of(j.req), reuse_bytes);
            if (reuse) {  // already resident: no new memory
              resident -= reuse_bytes;
              charged = reuse_bytes;
              ctx = reuse;
            } else {
              charged = charge(j.req);
            }
            evicted = evict_for(charged);
            if (resident + charged <= o.budget_bytes || running == 0) {
              id = queue.front();
              queue.pop_front();
              resident += charged;
              ++running;
              stats.peak_running = std::max(stats.peak_running, running);
              stats.peak_bytes = std::max(stats.peak_bytes, resident);
              j.res.start_s = now_s() - t0;
              break;
            }
            if (ctx) {  // give the pooled context back and wait for memory
              idle.push_front({shape_of(j.req), ctx, charged});
              resident += charged;
              ctx = nullptr;
            }
          }
          if (!evicted.empty()) break;  // free evicted contexts outside the lock, then retry
          cv_work.wait(lk);
        }
      }
      for (eg_ctx *c : evicted) eg_destroy(c);
      if (id < 0) continue;
      eg_request req;
      {
        std::lock_guard<std::mutex> lk(m);
        req = jobs[id].req;
      }
      eg_desc d{};
      int rc = eg_desc_simple_wave(&d, req.nx, req.ny, req.k, req.alpha_deg, 3.0, 1.1);
      if (rc == EG_OK && ctx) {
        rc = eg_set_desc(ctx, &d);  // a pooled context of this size: this request's geometry
      } else if (rc == EG_OK) {
        eg_opts eo{};
        eg_opts_default(&eo);
        eo.form = req.form;
        eo.precond = req.precond;
        eo.precision = req.precision;
        rc = eg_create(&d, &eo, &ctx);
      }
      eg_run_result rr{};
      std::vector<double> state;
      if (rc == EG_OK) {
        rc = run_schedule(ctx, schedule(req.steps, req.newton_steps, req.cfl, req.form, req.precond), rr);
        if (rc == EG_OK && o.keep_states) {
          int sz[7];
          eg_sizes(ctx, sz);
          state.resize((size_t)sz[5]);
          rc = eg_download(ctx, EG_SLOT_U, state.data());
        }
      }
      const long long actual = ctx ? eg_device_bytes(ctx) : 0;
      bool pooled = false;
      {
        std::lock_guard<std::mutex> lk(m);
        Job &j = jobs[id];
        j.res.status = rc;
        j.res.updates = rr.updates;
        j.res.final_time = rr.final_time;
        std::memcpy(j.res.errors, rr.errors, sizeof rr.errors);
        j.res.drift = rr.drift;
        j.res.bytes = std::max(charged, actual);
        j.res.finish_s = now_s() - t0;
        j.state = std::move(state);
        j.done = true;
        if (ctx) measured[shape_of(req)] = std::max(measured[shape_of(req)], actual);
        resident -= charged;
        --running;
        --pending;
        if (rc == EG_OK) ++stats.completed;
        else ++stats.failed;
        if (ctx && rc == EG_OK && o.keep_contexts) {
          idle.push_back({shape_of(req), ctx, actual});
          resident += actual;
          pooled = true;
        }
      }
      if (ctx && !pooled) eg_destroy(ctx);
      cv_work.notify_all();
      cv_done.notify_all();
    }
  }
};

extern "C" {

int eg_server_create(const eg_server_opts *o, eg_server **out) {
  if (!o || !out || o->workers <= 0 || o->budget_bytes <= 0) return EG_ERR_INVALID;
  *out = nullptr;
  const int rc = eg_set_device(o->device);
  if (rc != EG_OK) return rc;
  auto *s = new eg_server();
  s->o = *o;
  s->t0 = now_s();
  for (int i = 0; i < o->workers; ++i) s->threads.emplace_back([s] { s->worker(); });
  *out = s;
  return EG_OK;
}

double eg_server_clock(const eg_server *s) { return s ? now_s() - s->t0 : 0.; }

int eg_server_submit(eg_server *s, const eg_request *r, long long *id) {
  if (!s || !r || !id) return EG_ERR_INVALID;
  if (r->nx < 2 || r->ny < 2 || r->k < 0 || r->k > 8 || r->steps <= 0) return EG_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->m);
    if (s->stop) return EG_ERR_INVALID;
    *id = s->next_id++;
    Job &j = s->jobs[*id];
    j.req = *r;
    j.res.submit_s = now_s() - s->t0;
    s->queue.push_back(*id);
    ++s->pending;
  }
  s->cv_work.notify_one();
  return EG_OK;
}

int eg_server_poll(eg_server *s, long long id, eg_request_result *res) {
  if (!s) return EG_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->m);
  const auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return EG_ERR_INVALID;
  if (!it->second.done) return -1;
  if (res) *res = it->second.res;
  return EG_OK;
}

int eg_server_state(eg_server *s, long long id, double *u) {
  if (!s || !u) return EG_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->m);
  const auto it = s->jobs.find(id);
  if (it == s->jobs.end() || !it->second.done || it->second.state.empty()) return EG_ERR_INVALID;
  std::memcpy(u, it->second.state.data(), sizeof(double) * it->second.state.size());
  return EG_OK;
}

int eg_server_drain(eg_server *s, eg_server_stats *st) {
  if (!s) return EG_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->m);
  s->cv_done.wait(lk, [s] { return s->pending == 0; });
  if (st) *st = s->stats;
  return EG_OK;
}

void eg_server_destroy(eg_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto &t : s->threads) t.join();
  eg_set_device(s->o.device);
  for (auto &i : s->idle) eg_destroy(i.ctx);
  delete s;
}

}  // extern "C"
