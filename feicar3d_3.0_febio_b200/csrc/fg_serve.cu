// fg_serve.cu -- serving engine: a stream of solve requests over many
// cases, admitted continuously as slots and device memory free up.
//
// A request is one problem (grid, body surface) and a run of time steps,
// each a right-hand side in and a pressure out, as the reference's time
// loop runs rhs_poisson -> solve_poisson per step with the pressure kept
// between steps (CORE_TIME_STEP.F90:171-178).  An engine thread owns every
// case.  It admits queued requests first come, first served while the
// number of active cases stays under max_active and their estimated device
// memory under the budget; it builds each admitted case (hierarchy,
// device tagging, lists, prepare) on the case's own stream; and it keeps
// one step of every active case queued on the device: the right-hand
// side's copy in, the whole FGMRES solve as one CUDA graph launch, the
// output finishing and the copy out, then an event.  Steps of different
// cases run concurrently on their streams.  When a step's event has fired
// the engine queues the case's next step (warm-started from the pressure
// left on the device), or, after the last one, releases the case (its
// stream has drained, so the device memory goes back to the block cache
// without a device-wide wait) and admits the next requests.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "fg_case.h"
#include "fg_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  fg_serve_request r{};
  std::vector<double> xn, yn, zn, xyz;
  std::vector<int32_t> tri;
  std::vector<const double *> div;
  std::vector<double *> p;
  size_t bytes = 0;
  double t_submit = 0.0;
};

struct Active {
  std::unique_ptr<Req> req;
  fg_case *c = nullptr;
  cudaEvent_t ev = nullptr;
  int step = 0;
  bool in_flight = false;
  fg_serve_result res{};
};

}  // namespace

struct fg_server {
  int device = 0;
  fg_solver_config cfg{};
  size_t budget = 0;
  int max_active = 1;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::unique_ptr<Req>> pending;
  std::vector<fg_serve_result> done;
  long long submitted = 0, finished = 0;
  size_t used = 0;  // estimated bytes of the active cases
  int active_now = 0, active_peak = 0;
  bool stop = false;
  std::thread engine;
  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// builds the case of a request on its own stream: grid and hierarchy,
// body, device tagging, ghost/dead lists, prepare
fg_status build_case(fg_server *S, Req &q, fg_case **out) {
  const fg_serve_request &r = q.r;
  fg_case *c = nullptr;
  fg_status st = fg_case_create(r.nx, r.ny, r.nz, q.xn.data(), q.yn.data(), q.zn.data(), &S->cfg,
                                S->device, &c);
  if (st != FG_OK) return st;
  if ((st = fg_case_add_body(c, r.nvert, r.ntri, q.xyz.data(), q.tri.data(), r.surface_type,
                             r.membrane_tkns, 3)) != FG_OK ||
      (st = fg_set_iblank_body_fast(c, nullptr)) != FG_OK ||
      (st = fg_gcm_set_internal_boundary(c, nullptr, nullptr, nullptr, nullptr, nullptr)) != FG_OK ||
      (st = fg_mg_prepare(c)) != FG_OK) {
    fg_case_destroy(c);
    return st;
  }
  *out = c;
  return FG_OK;
}

// queues step a.step of an active case: div in, solve, output finished and
// copied to the step's host field, event
fg_status enqueue_step(Active &a) {
  fg_case *c = a.c;
  const size_t nref = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  const Req &q = *a.req;
  if (a.step == 0) {
    if (q.r.p0) FG_CUDA(cudaMemcpyAsync(c->d_pin, q.r.p0, nref * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    else FG_CUDA(cudaMemsetAsync(c->d_pin, 0, nref * sizeof(double), c->stream));
  }
  FG_CUDA(cudaMemcpyAsync(c->d_fin, q.div[a.step], nref * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  fg_status st = fg::solve_enqueue(c, nullptr, nullptr, nullptr);
  if (st != FG_OK) return st;
  if (q.p[a.step])
    FG_CUDA(cudaMemcpyAsync(q.p[a.step], c->d_pin, nref * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FG_CUDA(cudaEventRecord(a.ev, c->stream));
  a.in_flight = true;
  return FG_OK;
}

void finish(fg_server *S, Active &a, fg_status st) {
  a.res.status = st == FG_NOT_CONVERGED && a.res.status == FG_OK ? FG_NOT_CONVERGED : st;
  a.res.t_done = S->now();
  if (a.c) {
    fg_case_destroy(a.c);
    a.c = nullptr;
  }
  if (a.ev) cudaEventDestroy(a.ev);
  a.ev = nullptr;
  std::lock_guard<std::mutex> lk(S->mu);
  S->used -= a.req->bytes;
  S->active_now--;
  S->done.push_back(a.res);
  S->finished++;
  S->cv.notify_all();
}

void engine_loop(fg_server *S) {
  cudaSetDevice(S->device);
  std::vector<std::unique_ptr<Active>> act;
  for (;;) {
    // admit: first come first served, within the slots and the budget
    for (;;) {
      std::unique_ptr<Req> q;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->pending.empty() || (int)act.size() >= S->max_active) break;
        if (S->used + S->pending.front()->bytes > S->budget && !act.empty()) break;
        q = std::move(S->pending.front());
        S->pending.pop_front();
        S->used += q->bytes;
        S->active_now++;
        S->active_peak = std::max(S->active_peak, S->active_now);
      }
      auto a = std::make_unique<Active>();
      a->res.id = q->r.id;
      a->res.t_submit = q->t_submit;
      a->res.t_admit = S->now();
      a->res.status = FG_OK;
      a->req = std::move(q);
      fg_status st = build_case(S, *a->req, &a->c);
      if (st == FG_OK && cudaEventCreateWithFlags(&a->ev, cudaEventDisableTiming) != cudaSuccess)
        st = FG_CUDA_ERROR;
      if (st == FG_OK) st = enqueue_step(*a);
      if (st != FG_OK) {
        finish(S, *a, st);
        continue;
      }
      act.push_back(std::move(a));
    }
    // completions: the next step of each case whose step has finished
    bool progressed = false;
    for (size_t i = 0; i < act.size();) {
      Active &a = *act[i];
      if (a.in_flight && cudaEventQuery(a.ev) == cudaSuccess) {
        progressed = true;
        a.in_flight = false;
        fg_solve_stats ss{};
        fg_status st = fg::solve_collect(a.c, &ss);
        a.res.steps_done++;
        a.res.cycles_max = std::max(a.res.cycles_max, ss.cycles);
        a.res.relres_max = std::max(a.res.relres_max, ss.relres);
        if (st == FG_NOT_CONVERGED) a.res.status = FG_NOT_CONVERGED;
        else if (st != FG_OK) {
          finish(S, a, st);
          act.erase(act.begin() + i);
          continue;
        }
        a.step++;
        if (a.step >= a.req->r.nsteps) {
          finish(S, a, a.res.status);
          act.erase(act.begin() + i);
          continue;
        }
        if ((st = enqueue_step(a)) != FG_OK) {
          finish(S, a, st);
          act.erase(act.begin() + i);
          continue;
        }
      }
      ++i;
    }
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (S->stop && S->pending.empty() && act.empty()) break;
      if (!progressed) {
        const bool can_admit = !S->pending.empty() && (int)act.size() < S->max_active &&
                               (act.empty() || S->used + S->pending.front()->bytes <= S->budget);
        if (!can_admit) {
          // nothing to admit and nothing finished yet: wait a little for a
          // step to complete or a request to arrive
          S->cv.wait_for(lk, std::chrono::microseconds(act.empty() ? 2000 : 50));
        }
      }
    }
  }
}

}  // namespace

extern "C" {

fg_status fg_server_create(int device, const fg_solver_config *cfg, size_t budget_bytes, int max_active,
                           fg_server **out) {
  if (!out || max_active < 1) return FG_BAD_INPUT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FG_NO_DEVICE;
  if (device < 0 || device >= ndev) return FG_BAD_INPUT;
  auto *S = new fg_server();
  S->device = device;
  if (cfg) S->cfg = *cfg; else fg_default_config(&S->cfg);
  S->cfg.outer = FG_OUTER_FGMRES;  // one graph launch per step
  S->budget = budget_bytes;
  S->max_active = max_active;
  S->t0 = Clock::now();
  S->engine = std::thread(engine_loop, S);
  *out = S;
  return FG_OK;
}

double fg_server_clock(const fg_server *S) { return S ? S->now() : 0.0; }

fg_status fg_server_submit(fg_server *S, const fg_serve_request *r) {
  if (!S || !r || r->nsteps < 1 || !r->xn || !r->yn || !r->zn || !r->xyz || !r->tri || !r->div)
    return FG_BAD_INPUT;
  auto q = std::make_unique<Req>();
  q->r = *r;
  q->xn.assign(r->xn, r->xn + r->nx);
  q->yn.assign(r->yn, r->yn + r->ny);
  q->zn.assign(r->zn, r->zn + r->nz);
  q->xyz.assign(r->xyz, r->xyz + 3 * (size_t)r->nvert);
  q->tri.assign(r->tri, r->tri + 3 * (size_t)r->ntri);
  q->div.assign(r->div, r->div + r->nsteps);
  if (r->p) q->p.assign(r->p, r->p + r->nsteps);
  else q->p.assign(r->nsteps, nullptr);
  for (const double *d : q->div)
    if (!d) return FG_BAD_INPUT;
  fg_status st = fg_case_estimate_bytes(r->nx, r->ny, r->nz, &S->cfg, &q->bytes);
  if (st != FG_OK) return st;
  if (q->bytes > S->budget) return FG_REJECTED;  // could never be admitted
  std::lock_guard<std::mutex> lk(S->mu);
  q->t_submit = S->now();
  S->pending.push_back(std::move(q));
  S->submitted++;
  S->cv.notify_all();
  return FG_OK;
}

fg_status fg_server_poll(fg_server *S, fg_serve_result *out, int capacity, int *count) {
  if (!S || !count || capacity < 0 || (capacity > 0 && !out)) return FG_BAD_INPUT;
  std::lock_guard<std::mutex> lk(S->mu);
  const int n = std::min(capacity, (int)S->done.size());
  for (int i = 0; i < n; ++i) out[i] = S->done[i];
  S->done.erase(S->done.begin(), S->done.begin() + n);
  *count = n;
  return FG_OK;
}

fg_status fg_server_wait_idle(fg_server *S, double timeout_s) {
  if (!S) return FG_BAD_INPUT;
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                 [&] { return S->finished == S->submitted; });
  return ok ? FG_OK : FG_TIMEOUT;
}

fg_status fg_server_info(const fg_server *S, fg_server_stats *out) {
  if (!S || !out) return FG_BAD_INPUT;
  auto *M = const_cast<fg_server *>(S);
  std::lock_guard<std::mutex> lk(M->mu);
  out->submitted = S->submitted;
  out->finished = S->finished;
  out->pending = (long long)S->pending.size();
  out->active = S->active_now;
  out->active_peak = S->active_peak;
  out->bytes_in_use = S->used;
  return FG_OK;
}

fg_status fg_server_destroy(fg_server *S) {
  if (!S) return FG_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv.notify_all();
  }
  if (S->engine.joinable()) S->engine.join();
  delete S;
  return FG_OK;
}

}  // extern "C"
