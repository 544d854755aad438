// Serving loop: resident sessions solved and re-solved on concurrent streams.
//
// A session is one diagram kept on the device: its seeds and bins, its
// neighbour table, its results, and a device copy of its domain grid shared
// with every session on the same rpd_grid -- or its own domain, built on the
// device from a seeded blob or a sampled implicit function.  Requests (a new session's solve,
// or a weight-only re-solve of a session) wait in arrival order; a slot -- a
// host thread with its own context and CUDA stream -- takes the first one
// that can run: its session is not busy, and the device memory it needs fits
// in the budget next to the resident sessions and the requests in flight.
// Requests that arrive while others run are admitted as slots and memory
// free up, and the slots' kernels overlap on the device.  Every request ends
// with its stream synchronized, and a request's result depends only on its
// own inputs, so a result is the same alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Session {
  int id = 0;
  int n = 0;                     // seeds
  rpd_solver *solver = nullptr;
  bool ready = false;            // solved once
  bool failed = false;           // its first solve failed
  bool busy = false;             // a request runs on it
  bool released = false;         // freed once idle
  size_t resident = 0;           // device bytes kept between requests
  size_t reserved = 0;           // estimate reserved until the first solve ends
  int pending = 0;               // requests queued or running
};

struct Request {
  int ticket = 0;
  bool reweight = false;
  int session = 0;
  std::vector<float> data;  // seeds (xyzw) or weights
  int n = 0;
  const rpd_grid *grid = nullptr;
  // a domain built on the device by the session's own solver (no host grid)
  int dom_kind = 0;          // kDomHost (none, or `grid`), kDomBlob, kDomField
  int dom_size = 0, dom_nell = 0;
  uint64_t dom_seed = 0;
  std::vector<float> field;  // kDomField: (dom_size+1)^3 values, copied
  rpd_params params{};
  double *moments = nullptr;
  double *hessian = nullptr;  // --hessian rows (hessian_h > 0), user order
  int *hessian_ids = nullptr;
  size_t need = 0;          // transient device bytes while it runs
  size_t new_resident = 0;  // resident bytes it adds (a new session, a new grid)
  Clock::time_point submitted, admitted, done;
  bool finished = false;
  rpd_request_info info{};
};

constexpr int kDomHost = 0, kDomBlob = 1, kDomField = 2;

struct GridHolder {
  rpd_solver *solver = nullptr;  // owns the device grid
  bool loading = false;
  bool ready = false;
  bool failed = false;
};

size_t grid_bytes(const rpd_grid *g) {
  int size = 0, np = 0, nt = 0, nl = 0;
  if (!g || rpd_grid_info(g, &size, &np, &nt, &nl) != RPD_OK) return 0;
  const size_t S = size_t(size);
  // flags, offsets, summed-volume and summed-triangle tables, points,
  // triangles, lists
  return S * S * S * (1 + 4) + (S + 1) * (S + 1) * (S + 1) * 8 + size_t(np) * 16 + size_t(nt) * 12 +
         size_t(nl) * 4 + 4096;
}

// Device bytes of a domain built on the device at size^3 voxels: flags,
// offsets, summed tables, and for the reservation a surface of 48 size^2
// triangles (the session's actual bytes replace it after its solve).
size_t device_grid_bytes(int size) {
  const size_t S = size_t(size), S1 = S + 1;
  return S * S * S * (1 + 4) + S1 * S1 * S1 * 8 + 48 * S * S * (12 + 4) + 24 * S * S * 16 + 4096;
}

// The build's workspace: per lattice point the field, edge mask, counts and
// bases; per voxel the triangle counts; scan tiles.
size_t device_grid_build_bytes(int size) {
  const size_t S = size_t(size), S1 = S + 1;
  return S1 * S1 * S1 * (4 + 1 + 4 + 4) + (S * S * S + 1) * 4 + (size_t(1) << 20);
}

// Device bytes a session keeps: seeds (given and binned), permutation and
// inverse, neighbour table, results, status, bins.
size_t resident_bytes(int n, const rpd_params &p) {
  const size_t bins = size_t(double(n) / 3.1 * 1.2) + 64;
  return size_t(n) * (16 + 16 + 4 + 4 + 32 + 4 + 4 * size_t(p.K)) + bins * 4 + 4096;
}

// Device bytes a launch needs on top: binning workspace, failing-id lists,
// staging, parked boundary cells, neighbour rows of retry passes (caps grown
// x1.5 up to 5 times: bounded by 8x the first caps, which also bounds the
// first pass's slots for triangle overflows parked ahead).  Per work item of
// the parked cells: partial moments, failure, owning slot (40 bytes).
size_t transient_bytes(int n, const rpd_params &p) {
  const size_t cap = std::min<size_t>(size_t(n), std::max<size_t>(32768, size_t(n) / 8));
  const size_t P = size_t(std::min(255, p.P * 8)), V = size_t(std::min(256, p.V * 8)),
               T = size_t(std::min(4096, p.T * 8));
  const size_t slot = 144 + 32 * P + 44 * V + 4 * T;
  // --hessian: the rows on the device and their user-order staging
  const size_t hess = p.hessian_h > 0 ? 2 * size_t(n) * size_t(p.hessian_h) * (8 * size_t(p.hessian_hc) + 4) : 0;
  return size_t(n) * (12 + 16 + 32 + 12) + cap * (slot / 4 + 40 * (T / 32 + 1) / 4) +
         size_t(n) / 4 * size_t(p.K) * 8 * 4 + hess + (size_t(1) << 20);
}

}  // namespace

struct rpd_server {
  int device = 0;
  size_t budget = 0;
  std::vector<rpd_context *> ctx;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::unordered_map<int, std::unique_ptr<Request>> requests;
  std::unordered_map<int, std::unique_ptr<Session>> sessions;
  std::unordered_map<const rpd_grid *, std::unique_ptr<GridHolder>> grids;
  size_t resident = 0;  // sessions and grids
  size_t inflight = 0;  // admitted requests
  int next_ticket = 0, next_session = 0;
  bool stop = false;
  Clock::time_point created = Clock::now();

  // The first queued request that may run now, or null (mu held).  A new
  // session whose memory does not fit holds back the new sessions behind it
  // (no overtaking by size); re-solves of idle sessions still pass.  With
  // nothing running, the first runnable request runs even past the budget
  // (resident sessions alone may fill it until the caller releases some).
  Request *pick() {
    bool blocked_new = false;
    for (auto it = queue.begin(); it != queue.end(); ++it) {
      Request *r = *it;
      Session *s = sessions[r->session].get();
      if (r->reweight && !s->failed && (s->busy || !s->ready)) continue;
      if (!r->reweight && blocked_new) continue;
      const size_t want = r->need + r->new_resident;
      if (resident + inflight + want > budget && inflight > 0) {
        if (!r->reweight) blocked_new = true;
        continue;
      }
      queue.erase(it);
      return r;
    }
    return nullptr;
  }

  // The device grid of r's domain, uploaded by the first session on it.
  const rpd_solver *grid_for(GridHolder *gh, const rpd_grid *g, rpd_context *c) {
    std::unique_lock<std::mutex> lock(mu);
    cv_done.wait(lock, [&] { return !gh->loading; });
    if (!gh->ready && !gh->failed) {
      gh->loading = true;
      lock.unlock();
      int e = RPD_OK;
      rpd_solver *h = rpd_solver_create(c, &e);
      if (h) e = rpd_solver_set_grid(h, g);
      if (h) rpd::solver_trim(h);
      lock.lock();
      if (h && e == RPD_OK) {
        gh->solver = h;
        gh->ready = true;
        resident += rpd::solver_device_bytes(h);  // kept until the server goes
      } else {
        if (h) rpd_solver_destroy(h);
        gh->failed = true;
      }
      gh->loading = false;
      cv_done.notify_all();
    }
    return gh->ready ? gh->solver : nullptr;
  }

  void run(int slot) {
    rpd_context *c = ctx[size_t(slot)];
    for (;;) {
      Request *r = nullptr;
      Session *s = nullptr;
      GridHolder *gh = nullptr;
      {
        std::unique_lock<std::mutex> lock(mu);
        cv_work.wait(lock, [&] { return stop || (r = pick()) != nullptr; });
        if (!r) return;  // stopping, nothing runnable
        s = sessions[r->session].get();
        s->busy = true;
        inflight += r->need;
        if (!r->reweight) {
          resident += r->new_resident;
          s->reserved = r->new_resident;
        }
        if (r->grid) gh = grids[r->grid].get();
        r->admitted = Clock::now();
      }
      int rc = RPD_OK;
      rpd_stats st{};
      if (!r->reweight) {
        s->solver = rpd_solver_create(c, &rc);
        if (s->solver && gh) {
          const rpd_solver *g = grid_for(gh, r->grid, c);
          if (g) rpd::solver_share_grid(s->solver, g);
          else rc = RPD_ERR_CUDA;
        } else if (s->solver && r->dom_kind == kDomBlob) {
          rc = rpd_solver_set_grid_blob(s->solver, r->dom_size, r->dom_nell, r->dom_seed);
        } else if (s->solver && r->dom_kind == kDomField) {
          rc = rpd_solver_set_grid_field(s->solver, r->dom_size, r->field.data(), RPD_HOST);
          std::vector<float>().swap(r->field);
        }
        if (s->solver && rc == RPD_OK) rc = rpd_solver_set_points(s->solver, r->data.data(), r->n, RPD_HOST);
      } else if (!s->solver || s->failed) {
        rc = RPD_ERR_INVALID;  // the session's solve failed
      } else {
        rpd::solver_rebind(s->solver, c);
        rc = rpd_solver_set_weights(s->solver, r->data.data(), RPD_HOST);
      }
      if (rc == RPD_OK && s->solver) rc = rpd_solver_launch(s->solver, &r->params);
      if (rc == RPD_OK && r->moments) rc = rpd_solver_get_moments(s->solver, r->moments, RPD_HOST);
      if (rc == RPD_OK && r->hessian) rc = rpd_solver_get_hessian(s->solver, r->hessian, r->hessian_ids, RPD_HOST);
      if (s->solver) {
        rpd_solver_get_stats(s->solver, &st);
        rpd::solver_trim(s->solver);
      }
      {
        std::lock_guard<std::mutex> lock(mu);
        inflight -= r->need;
        if (!r->reweight) {
          resident -= s->reserved;
          s->reserved = 0;
          s->ready = rc == RPD_OK;
          s->failed = rc != RPD_OK;
          if (s->failed && s->solver) {
            rpd_solver_destroy(s->solver);
            s->solver = nullptr;
          }
        }
        resident -= s->resident;
        s->resident = s->solver ? rpd::solver_device_bytes(s->solver) : 0;
        resident += s->resident;
        s->busy = false;
        s->pending -= 1;
        r->done = Clock::now();
        r->info.status = rc;
        r->info.session = r->session;
        r->info.n = r->n;
        r->info.slot = slot;
        r->info.queue_ms = ms_between(r->submitted, r->admitted);
        r->info.latency_ms = ms_between(r->submitted, r->done);
        r->info.admitted_at_ms = ms_between(created, r->admitted);
        r->info.done_at_ms = ms_between(created, r->done);
        r->info.device_ms = st.total_ms;
        r->info.npasses = st.npasses;
        r->info.failed_cells = rc == RPD_OK ? r->n - st.status_hist[RPD_SUCCESS] - st.status_hist[RPD_EMPTY_CELL] : r->n;
        for (int k = 0; k < RPD_STATUS_NUM; ++k) r->info.status_hist[k] = rc == RPD_OK ? st.status_hist[k] : 0;
        r->info.last_caps[0] = st.npasses > 0 ? st.pass_K[std::min(st.npasses, 8) - 1] : 0;
        r->info.last_caps[1] = st.npasses > 0 ? st.pass_P[std::min(st.npasses, 8) - 1] : 0;
        r->info.last_caps[2] = st.npasses > 0 ? st.pass_V[std::min(st.npasses, 8) - 1] : 0;
        r->info.last_caps[3] = st.npasses > 0 ? st.pass_T[std::min(st.npasses, 8) - 1] : 0;
        if (rc != RPD_OK) {
          const char *msg = rpd_context_error(c);
          std::snprintf(r->info.error, sizeof(r->info.error), "%s", msg ? msg : "");
        }
        r->finished = true;
        std::vector<float>().swap(r->data);
        if (s->released && s->pending == 0) drop_session(s);
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  void drop_session(Session *s) {  // mu held, session idle
    if (s->solver) rpd_solver_destroy(s->solver);
    resident -= s->resident;
    sessions.erase(s->id);
  }

  int submit(std::unique_ptr<Request> r) {  // mu held
    r->ticket = next_ticket++;
    r->submitted = Clock::now();
    Request *raw = r.get();
    requests[raw->ticket] = std::move(r);
    queue.push_back(raw);
    cv_work.notify_one();
    return raw->ticket;
  }
};

extern "C" {

rpd_server *rpd_server_create(int device, int slots, size_t mem_budget, int *err) {
  if (slots < 1 || slots > 64) {
    if (err) *err = RPD_ERR_INVALID;
    return nullptr;
  }
  auto sv = std::make_unique<rpd_server>();
  sv->device = device;
  for (int i = 0; i < slots; ++i) {
    int e = RPD_OK;
    rpd_context *c = rpd_context_create(device, &e);
    if (!c) {
      for (rpd_context *x : sv->ctx) rpd_context_destroy(x);
      if (err) *err = e;
      return nullptr;
    }
    sv->ctx.push_back(c);
  }
  if (mem_budget == 0) {
    size_t fr = 0, tot = 0;
    cudaSetDevice(device);
    cudaMemGetInfo(&fr, &tot);
    mem_budget = size_t(double(fr) * 0.9);
  }
  sv->budget = mem_budget;
  rpd_server *raw = sv.get();
  for (int i = 0; i < slots; ++i)
    raw->threads.emplace_back([raw, i] {
      cudaSetDevice(raw->device);
      raw->run(i);
    });
  if (err) *err = RPD_OK;
  return sv.release();
}

void rpd_server_destroy(rpd_server *sv) {
  if (!sv) return;
  {
    std::unique_lock<std::mutex> lock(sv->mu);
    sv->cv_done.wait(lock, [&] {
      for (auto &kv : sv->requests)
        if (!kv.second->finished) return false;
      return true;
    });
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  for (auto &t : sv->threads) t.join();
  for (auto &kv : sv->sessions)
    if (kv.second->solver) rpd_solver_destroy(kv.second->solver);
  sv->sessions.clear();
  for (auto &kv : sv->grids)
    if (kv.second->solver) rpd_solver_destroy(kv.second->solver);
  sv->grids.clear();
  for (rpd_context *c : sv->ctx) rpd_context_destroy(c);
  delete sv;
}

int rpd_server_submit_solve(rpd_server *sv, const float *xyzw, int n, const rpd_grid *grid, const rpd_params *p,
                            double *moments, int *session) {
  if (p && p->hessian_h != 0) return RPD_ERR_INVALID;  // rows only through the _hessian form
  return rpd_server_submit_solve_hessian(sv, xyzw, n, grid, p, moments, nullptr, nullptr, session);
}

}  // extern "C"

namespace {

// A new session's solve; r carries its domain (a host grid, or one to build
// on the device, with the build's workspace in its transient bytes).
int submit_new(rpd_server *sv, std::unique_ptr<Request> r, const float *xyzw, int n, const rpd_params *p,
               double *moments, double *hessian, int *hessian_ids, int *session) {
  if (!sv || !xyzw || n <= 0) return RPD_ERR_INVALID;
  r->n = n;
  r->data.assign(xyzw, xyzw + size_t(n) * 4);
  if (p) r->params = *p;
  else rpd_params_default(&r->params);
  if (r->params.hessian_h < 0 || (r->params.hessian_h > 0 && (!hessian || !hessian_ids))) return RPD_ERR_INVALID;
  r->moments = moments;
  if (r->params.hessian_h > 0) {
    r->hessian = hessian;
    r->hessian_ids = hessian_ids;
  }
  r->need = transient_bytes(n, r->params);
  r->new_resident = resident_bytes(n, r->params);
  if (r->dom_kind != kDomHost) {
    r->need += device_grid_build_bytes(r->dom_size);
    r->new_resident += device_grid_bytes(r->dom_size);
  }
  std::lock_guard<std::mutex> lock(sv->mu);
  if (sv->stop) return RPD_ERR_INVALID;
  if (r->grid && !sv->grids.count(r->grid)) {
    sv->grids[r->grid] = std::make_unique<GridHolder>();
    r->new_resident += grid_bytes(r->grid);  // reserved with the first session on it
  }
  auto s = std::make_unique<Session>();
  s->id = sv->next_session++;
  s->n = n;
  s->pending = 1;
  r->session = s->id;
  if (session) *session = s->id;
  sv->sessions[s->id] = std::move(s);
  return sv->submit(std::move(r));
}

constexpr int kMaxDeviceGridSize = 1024;  // as rpd_solver_set_grid_blob / _field

}  // namespace

extern "C" {

int rpd_server_submit_solve_hessian(rpd_server *sv, const float *xyzw, int n, const rpd_grid *grid,
                                    const rpd_params *p, double *moments, double *hessian, int *hessian_ids,
                                    int *session) {
  auto r = std::make_unique<Request>();
  r->grid = grid;
  return submit_new(sv, std::move(r), xyzw, n, p, moments, hessian, hessian_ids, session);
}

int rpd_server_submit_solve_blob(rpd_server *sv, const float *xyzw, int n, int grid_size, int nellipsoids,
                                 uint64_t grid_seed, const rpd_params *p, double *moments, double *hessian,
                                 int *hessian_ids, int *session) {
  if (grid_size < 1 || grid_size > kMaxDeviceGridSize || nellipsoids < 1 || nellipsoids > 4096)
    return RPD_ERR_INVALID;
  auto r = std::make_unique<Request>();
  r->dom_kind = kDomBlob;
  r->dom_size = grid_size;
  r->dom_nell = nellipsoids;
  r->dom_seed = grid_seed;
  return submit_new(sv, std::move(r), xyzw, n, p, moments, hessian, hessian_ids, session);
}

int rpd_server_submit_solve_field(rpd_server *sv, const float *xyzw, int n, int grid_size, const float *field,
                                  const rpd_params *p, double *moments, double *hessian, int *hessian_ids,
                                  int *session) {
  if (grid_size < 1 || grid_size > kMaxDeviceGridSize || !field) return RPD_ERR_INVALID;
  auto r = std::make_unique<Request>();
  r->dom_kind = kDomField;
  r->dom_size = grid_size;
  const size_t S1 = size_t(grid_size) + 1;
  r->field.assign(field, field + S1 * S1 * S1);
  return submit_new(sv, std::move(r), xyzw, n, p, moments, hessian, hessian_ids, session);
}

int rpd_server_submit_reweight(rpd_server *sv, int session, const float *w, const rpd_params *p, double *moments) {
  if (p && p->hessian_h != 0) return RPD_ERR_INVALID;  // rows only through the _hessian form
  return rpd_server_submit_reweight_hessian(sv, session, w, p, moments, nullptr, nullptr);
}

int rpd_server_submit_reweight_hessian(rpd_server *sv, int session, const float *w, const rpd_params *p,
                                       double *moments, double *hessian, int *hessian_ids) {
  if (!sv || !w) return RPD_ERR_INVALID;
  auto r = std::make_unique<Request>();
  r->reweight = true;
  r->session = session;
  if (p) r->params = *p;
  else rpd_params_default(&r->params);
  if (r->params.hessian_h < 0 || (r->params.hessian_h > 0 && (!hessian || !hessian_ids))) return RPD_ERR_INVALID;
  r->moments = moments;
  if (r->params.hessian_h > 0) {
    r->hessian = hessian;
    r->hessian_ids = hessian_ids;
  }
  std::lock_guard<std::mutex> lock(sv->mu);
  if (sv->stop) return RPD_ERR_INVALID;
  auto it = sv->sessions.find(session);
  if (it == sv->sessions.end() || it->second->released || it->second->failed) return RPD_ERR_INVALID;
  Session *s = it->second.get();
  r->n = s->n;
  r->data.assign(w, w + size_t(s->n));
  r->need = transient_bytes(s->n, r->params);
  s->pending += 1;
  return sv->submit(std::move(r));
}

int rpd_server_wait(rpd_server *sv, int ticket, rpd_request_info *info) {
  if (!sv) return RPD_ERR_INVALID;
  std::unique_lock<std::mutex> lock(sv->mu);
  auto it = sv->requests.find(ticket);
  if (it == sv->requests.end()) return RPD_ERR_INVALID;
  Request *r = it->second.get();
  sv->cv_done.wait(lock, [&] { return r->finished; });
  if (info) *info = r->info;
  const int rc = r->info.status;
  sv->requests.erase(it);
  return rc;
}

int rpd_server_release(rpd_server *sv, int session) {
  if (!sv) return RPD_ERR_INVALID;
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->sessions.find(session);
  if (it == sv->sessions.end() || it->second->released) return RPD_ERR_INVALID;
  Session *s = it->second.get();
  s->released = true;
  if (s->pending == 0) sv->drop_session(s);
  sv->cv_work.notify_all();
  return RPD_OK;
}

size_t rpd_server_bytes_in_use(rpd_server *sv) {
  if (!sv) return 0;
  std::lock_guard<std::mutex> lock(sv->mu);
  return sv->resident + sv->inflight;
}

}  // extern "C"
