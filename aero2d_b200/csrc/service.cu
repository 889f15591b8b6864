// Continuous-batching service over one batched plan (the served-polar use of
// the Newton-Krylov path).  The plan's cases are slots, grouped in classes by
// grid size (ni, nc); a request is a sequence of freestreams (a polar sweep)
// on one grid of a class's size, solved point after point in one slot, each
// point started from the previous point's state (alpha continuation) or from
// the freestream.  Before every Newton step, queued requests are admitted in
// arrival order into free slots of their class (a request whose class is full
// waits without holding back requests of other classes); a slot freed by a
// finished request is refilled at the next step, so the batch stays full
// instead of draining to its slowest case.  A request may bring its own grid
// (a metrics blob of its class's size, kept alive by the caller until its
// result is taken): the slot is pointed at it on admission.
//
// Host code only: it drives the plan through the library's own C ABI
// (a2d_newton_step, a2d_case_status, a2d_case_forces, a2d_case_set_grid,
// a2d_case_restart, a2d_case_retire).  Requests and results live in host
// memory; the caller owns the device workspace, as for a plan.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "aero2d_b200.h"

namespace a2d {
int fail(int code, const std::string& msg);
}

struct a2d_service {
  a2d_plan* plan = nullptr;
  int slots = 0, max_iter = 0;
  struct Class {
    int ni = 0, nc = 0, first = 0, count = 0;
    const void* metrics = nullptr;   // the class's default grid
  };
  std::vector<Class> classes;
  struct Request {
    int cls = 0;
    const void* metrics = nullptr;
    int npts = 0;
    int continuation = 1;
    std::vector<double> winf;       // [npts][4]
    int next = 0;                   // next point to start
    int done_pts = 0;
    std::vector<double> coef;       // [npts][3]
    std::vector<double> cp;         // [npts][ni]
    std::vector<int> converged, nsteps;
    std::vector<double> drop;       // [npts] last finite residual norm / r0
  };
  std::map<long long, Request> reqs;
  std::deque<long long> queue;
  std::vector<int> slot_cls;             // class of each slot
  std::vector<long long> slot_cp;        // first wall entry of each slot in the plan's cp array
  std::vector<const void*> slot_metrics; // grid each slot points at
  std::vector<long long> slot_req;       // request in each slot, -1 if free
  std::vector<int> slot_pt;              // point of that request in the slot
  std::vector<long long> finished;       // finished since the last poll
  long long next_id = 1;
  long long total_ni = 0;
  long long newton_steps = 0;            // Newton steps taken by the plan since bind
  std::mutex mu;
};

using a2d::fail;

namespace {

int class_of(const a2d_service* S, int ni, int nc) {
  for (size_t c = 0; c < S->classes.size(); ++c)
    if (S->classes[c].ni == ni && S->classes[c].nc == nc) return (int)c;
  return -1;
}

int submit(a2d_service* S, int cls, const void* metrics, int npoints, const double* winf, int continuation,
           long long* id) {
  const int ni = S->classes[cls].ni;
  a2d_service::Request r;
  r.cls = cls;
  r.metrics = metrics != nullptr ? metrics : S->classes[cls].metrics;
  r.npts = npoints;
  r.continuation = continuation ? 1 : 0;
  r.winf.assign(winf, winf + 4 * (size_t)npoints);
  r.coef.assign(3 * (size_t)npoints, 0.0);
  r.cp.assign((size_t)npoints * ni, 0.0);
  r.converged.assign(npoints, 0);
  r.nsteps.assign(npoints, 0);
  r.drop.assign(npoints, NAN);
  std::lock_guard<std::mutex> lk(S->mu);
  const long long rid = S->next_id++;
  S->reqs.emplace(rid, std::move(r));
  S->queue.push_back(rid);
  *id = rid;
  return A2D_OK;
}

}  // namespace

extern "C" {

int a2d_service_create_ragged(int nclasses, const int* ni, const int* nc, const void* const* metrics,
                              const int* slots, const a2d_params* params, a2d_service** out) {
  if (out == nullptr || nclasses < 1 || ni == nullptr || nc == nullptr || metrics == nullptr || slots == nullptr)
    return fail(A2D_ERR_ARG, "service_create: bad arguments");
  a2d_params p;
  a2d_default_params(&p);
  if (params != nullptr) p = *params;
  p.retire = 1;   // a slot stops stepping as soon as its point is done
  a2d_service* S = new a2d_service();
  std::vector<int> vni, vnc;
  std::vector<const void*> vm;
  for (int c = 0; c < nclasses; ++c) {
    if (slots[c] < 1 || metrics[c] == nullptr || class_of(S, ni[c], nc[c]) >= 0) {
      delete S;
      return fail(A2D_ERR_ARG, "service_create: each class needs slots >= 1, a grid, and its own size");
    }
    a2d_service::Class k;
    k.ni = ni[c];
    k.nc = nc[c];
    k.first = (int)vni.size();
    k.count = slots[c];
    k.metrics = metrics[c];
    S->classes.push_back(k);
    for (int q = 0; q < slots[c]; ++q) {
      vni.push_back(ni[c]);
      vnc.push_back(nc[c]);
      vm.push_back(metrics[c]);
      S->slot_cls.push_back(c);
      S->slot_cp.push_back(S->total_ni);
      S->total_ni += ni[c];
    }
  }
  const int n = (int)vni.size();
  std::vector<double> winf(4 * (size_t)n);
  for (int k = 0; k < n; ++k) {   // placeholder freestream until a request is admitted
    winf[4 * k + 0] = 1.0;
    winf[4 * k + 1] = 0.5;
    winf[4 * k + 2] = 0.0;
    winf[4 * k + 3] = 1.0 / 1.4;
  }
  if (int e = a2d_plan_create(n, vni.data(), vnc.data(), vm.data(), winf.data(), &p, &S->plan)) {
    delete S;
    return e;
  }
  S->slots = n;
  S->max_iter = p.max_iter;
  S->slot_metrics = vm;
  S->slot_req.assign(n, -1);
  S->slot_pt.assign(n, 0);
  *out = S;
  return A2D_OK;
}

int a2d_service_create(int ni, int nc, const void* metrics, int slots, const a2d_params* params,
                       a2d_service** out) {
  return a2d_service_create_ragged(1, &ni, &nc, &metrics, &slots, params, out);
}

int a2d_service_workspace_bytes(const a2d_service* S, size_t* bytes) {
  if (S == nullptr) return fail(A2D_ERR_ARG, "null service");
  return a2d_plan_workspace_bytes(S->plan, bytes);
}

int a2d_service_bind(a2d_service* S, void* workspace, size_t bytes, void* stream) {
  if (S == nullptr) return fail(A2D_ERR_ARG, "null service");
  if (int e = a2d_plan_bind(S->plan, workspace, bytes, stream)) return e;
  // every slot starts idle
  std::vector<int> all(S->slots);
  for (int k = 0; k < S->slots; ++k) all[k] = k;
  return a2d_case_retire(S->plan, S->slots, all.data(), stream);
}

int a2d_service_submit(a2d_service* S, int npoints, const double* winf, int continuation, long long* id) {
  if (S == nullptr || npoints < 1 || winf == nullptr || id == nullptr)
    return fail(A2D_ERR_ARG, "service_submit: bad arguments");
  return submit(S, 0, nullptr, npoints, winf, continuation, id);
}

int a2d_service_submit_grid(a2d_service* S, int ni, int nc, const void* metrics, int npoints, const double* winf,
                            int continuation, long long* id) {
  if (S == nullptr || npoints < 1 || winf == nullptr || id == nullptr)
    return fail(A2D_ERR_ARG, "service_submit: bad arguments");
  const int cls = class_of(S, ni, nc);
  if (cls < 0) return fail(A2D_ERR_ARG, "service_submit: no slot class of this grid size");
  return submit(S, cls, metrics, npoints, winf, continuation, id);
}

int a2d_service_step(a2d_service* S, int* busy, void* stream) {
  if (S == nullptr) return fail(A2D_ERR_ARG, "null service");
  std::lock_guard<std::mutex> lk(S->mu);
  // admit queued requests, in arrival order, into free slots of their class
  std::vector<int> start, regrid;
  std::vector<double> start_w;
  std::vector<const void*> regrid_m;
  std::vector<int> free_in(S->classes.size(), 0);
  for (int k = 0; k < S->slots; ++k) free_in[S->slot_cls[k]] += S->slot_req[k] < 0;
  for (auto it = S->queue.begin(); it != S->queue.end();) {
    a2d_service::Request& r = S->reqs[*it];
    if (free_in[r.cls] == 0) {
      ++it;
      continue;
    }
    const a2d_service::Class& c = S->classes[r.cls];
    int k = c.first;
    while (S->slot_req[k] >= 0) ++k;
    S->slot_req[k] = *it;
    S->slot_pt[k] = 0;
    r.next = 1;
    free_in[r.cls] -= 1;
    start.push_back(k);
    start_w.insert(start_w.end(), r.winf.begin(), r.winf.begin() + 4);
    if (S->slot_metrics[k] != r.metrics) {
      S->slot_metrics[k] = r.metrics;
      regrid.push_back(k);
      regrid_m.push_back(r.metrics);
    }
    it = S->queue.erase(it);
  }
  if (!regrid.empty())
    if (int e = a2d_case_set_grid(S->plan, (int)regrid.size(), regrid.data(), regrid_m.data(), stream)) return e;
  if (!start.empty())
    if (int e = a2d_case_restart(S->plan, (int)start.size(), start.data(), start_w.data(), 0, stream)) return e;
  int nbusy = 0;
  for (int k = 0; k < S->slots; ++k) nbusy += S->slot_req[k] >= 0;
  if (busy != nullptr) *busy = nbusy;
  if (nbusy == 0) return A2D_OK;

  if (int e = a2d_newton_step(S->plan, stream)) return e;
  S->newton_steps += 1;
  std::vector<int> nsteps(S->slots), done(S->slots), frozen(S->slots);
  std::vector<double> lastrn(S->slots), r0(S->slots);
  if (int e = a2d_case_status(S->plan, nsteps.data(), done.data(), frozen.data(), lastrn.data(), r0.data(), stream))
    return e;
  std::vector<int> ended;
  for (int k = 0; k < S->slots; ++k)
    if (S->slot_req[k] >= 0 && (done[k] || frozen[k] || nsteps[k] >= S->max_iter)) ended.push_back(k);
  if (ended.empty()) return A2D_OK;

  // results of the points that ended, then the next points (or free slots)
  std::vector<double> coef(3 * (size_t)S->slots), cp((size_t)S->total_ni);
  if (int e = a2d_case_forces(S->plan, coef.data(), cp.data(), stream)) return e;
  std::vector<int> keep_k, fresh_k, retire_k;
  std::vector<double> keep_w, fresh_w;
  for (int k : ended) {
    const long long rid = S->slot_req[k];
    a2d_service::Request& r = S->reqs[rid];
    const int ni = S->classes[r.cls].ni;
    const int pt = S->slot_pt[k];
    for (int c = 0; c < 3; ++c) r.coef[3 * (size_t)pt + c] = coef[3 * (size_t)k + c];
    std::copy(cp.begin() + S->slot_cp[k], cp.begin() + S->slot_cp[k] + ni, r.cp.begin() + (size_t)pt * ni);
    // the reference's flag (aero2d/implicit.py:252): not frozen and three orders down
    r.converged[pt] = !frozen[k] && std::isfinite(lastrn[k]) && lastrn[k] < 1e-3 * r0[k];
    r.nsteps[pt] = nsteps[k];
    r.drop[pt] = lastrn[k] / r0[k];
    r.done_pts += 1;
    if (r.next < r.npts) {
      const int np = r.next++;
      S->slot_pt[k] = np;
      std::vector<int>& lst = r.continuation ? keep_k : fresh_k;
      std::vector<double>& w = r.continuation ? keep_w : fresh_w;
      lst.push_back(k);
      w.insert(w.end(), r.winf.begin() + 4 * (size_t)np, r.winf.begin() + 4 * (size_t)np + 4);
    } else {
      S->finished.push_back(rid);
      S->slot_req[k] = -1;
      retire_k.push_back(k);
    }
  }
  if (!keep_k.empty())
    if (int e = a2d_case_restart(S->plan, (int)keep_k.size(), keep_k.data(), keep_w.data(), 1, stream)) return e;
  if (!fresh_k.empty())
    if (int e = a2d_case_restart(S->plan, (int)fresh_k.size(), fresh_k.data(), fresh_w.data(), 0, stream)) return e;
  if (!retire_k.empty()) {
    if (int e = a2d_case_retire(S->plan, (int)retire_k.size(), retire_k.data(), stream)) return e;
    // a freed slot goes back to its class's own grid: the finished request's grid belongs to
    // the caller, who may free it once the result is taken, and a2d_case_forces reads every slot
    std::vector<int> back;
    std::vector<const void*> back_m;
    for (int k : retire_k) {
      const void* m = S->classes[S->slot_cls[k]].metrics;
      if (S->slot_metrics[k] != m) {
        S->slot_metrics[k] = m;
        back.push_back(k);
        back_m.push_back(m);
      }
    }
    if (!back.empty())
      if (int e = a2d_case_set_grid(S->plan, (int)back.size(), back.data(), back_m.data(), stream)) return e;
  }
  return A2D_OK;
}

int a2d_service_poll(a2d_service* S, long long* ids, int max_ids, int* n) {
  if (S == nullptr || n == nullptr || (max_ids > 0 && ids == nullptr)) return fail(A2D_ERR_ARG, "service_poll: bad arguments");
  std::lock_guard<std::mutex> lk(S->mu);
  const int m = std::min<int>(max_ids, (int)S->finished.size());
  for (int q = 0; q < m; ++q) ids[q] = S->finished[q];
  S->finished.erase(S->finished.begin(), S->finished.begin() + m);
  *n = m;
  return A2D_OK;
}

int a2d_service_result(a2d_service* S, long long id, double* coef, double* cp, int* converged, int* nsteps) {
  if (S == nullptr) return fail(A2D_ERR_ARG, "null service");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return fail(A2D_ERR_ARG, "service_result: unknown request");
  const a2d_service::Request& r = it->second;
  if (r.done_pts < r.npts) return fail(A2D_ERR_STATE, "service_result: request not finished");
  if (coef != nullptr) std::copy(r.coef.begin(), r.coef.end(), coef);
  if (cp != nullptr) std::copy(r.cp.begin(), r.cp.end(), cp);
  if (converged != nullptr) std::copy(r.converged.begin(), r.converged.end(), converged);
  if (nsteps != nullptr) std::copy(r.nsteps.begin(), r.nsteps.end(), nsteps);
  S->reqs.erase(it);
  return A2D_OK;
}

int a2d_service_result_drop(a2d_service* S, long long id, double* drop) {
  if (S == nullptr || drop == nullptr) return fail(A2D_ERR_ARG, "service_result_drop: bad arguments");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return fail(A2D_ERR_ARG, "service_result_drop: unknown request");
  const a2d_service::Request& r = it->second;
  if (r.done_pts < r.npts) return fail(A2D_ERR_STATE, "service_result_drop: request not finished");
  std::copy(r.drop.begin(), r.drop.end(), drop);
  return A2D_OK;
}

int a2d_service_pending(a2d_service* S, int* queued, int* running) {
  if (S == nullptr) return fail(A2D_ERR_ARG, "null service");
  std::lock_guard<std::mutex> lk(S->mu);
  if (queued != nullptr) *queued = (int)S->queue.size();
  if (running != nullptr) {
    int nb = 0;
    for (long long r : S->slot_req) nb += r >= 0;
    *running = nb;
  }
  return A2D_OK;
}

int a2d_service_plan(a2d_service* S, a2d_plan** plan) {
  if (S == nullptr || plan == nullptr) return fail(A2D_ERR_ARG, "service_plan: bad arguments");
  *plan = S->plan;
  return A2D_OK;
}

int a2d_service_stats(a2d_service* S, int* kernels_per_step, long long* newton_steps) {
  if (S == nullptr) return fail(A2D_ERR_ARG, "null service");
  std::lock_guard<std::mutex> lk(S->mu);
  if (newton_steps != nullptr) *newton_steps = S->newton_steps;
  return a2d_plan_stats(S->plan, kernels_per_step, nullptr, nullptr);
}

int a2d_service_destroy(a2d_service* S) {
  if (S == nullptr) return A2D_OK;
  a2d_plan_destroy(S->plan);
  delete S;
  return A2D_OK;
}

}  // extern "C"
