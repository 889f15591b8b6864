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
// The slots may be split into lanes: one plan per lane, each class's slots dealt
// to the lanes in turn, and a Newton step of every busy lane launched on the
// lane's own stream, forked from and joined back into the caller's stream, so
// that the lanes' kernels run concurrently and the hardware fills the SMs that
// one batch's launches leave idle (a 64-case batch's sweep has 4 CTAs on some
// SMs and 3 on others; four 16-case lanes step it 6 % faster).  Every per-case
// result is independent of the batch it is stepped in, so a request's result
// does not depend on its lane or slot.
//
// Host code only: it drives the plans through the library's own C ABI
// (a2d_newton_step, a2d_case_status, a2d_case_forces, a2d_case_set_grid,
// a2d_case_restart, a2d_case_retire).  Requests and results live in host
// memory; the caller owns the device workspace, as for a plan.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
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
  struct Lane {
    a2d_plan* plan = nullptr;
    std::vector<int> slots;           // global slot of each of the plan's cases
    std::vector<long long> cp_off;    // first wall entry of each case in the plan's cp array
    long long total_ni = 0;
    size_t ws_off = 0, ws_bytes = 0;  // the plan's part of the workspace
    cudaStream_t stream = nullptr;    // concurrent lanes only
    cudaEvent_t done = nullptr;
  };
  std::vector<Lane> lanes;
  cudaEvent_t fork = nullptr;
  std::vector<int> slot_lane, slot_local;   // lane of each global slot and its case there
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
  std::vector<const void*> slot_metrics; // grid each slot points at
  std::vector<long long> slot_req;       // request in each slot, -1 if free
  std::vector<int> slot_pt;              // point of that request in the slot
  std::vector<long long> finished;       // finished since the last poll
  long long next_id = 1;
  long long newton_steps = 0;            // Newton steps taken by the service since bind
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

// the global slots of `ks` (with per-slot payload of `width` values each) as
// local case lists per lane
template <typename V>
void by_lane(const a2d_service* S, const std::vector<int>& ks, const std::vector<V>& payload, int width,
             std::vector<std::vector<int>>& lk, std::vector<std::vector<V>>& lp) {
  lk.assign(S->lanes.size(), {});
  lp.assign(S->lanes.size(), {});
  for (size_t q = 0; q < ks.size(); ++q) {
    const int l = S->slot_lane[ks[q]];
    lk[l].push_back(S->slot_local[ks[q]]);
    lp[l].insert(lp[l].end(), payload.begin() + q * width, payload.begin() + (q + 1) * width);
  }
}

int set_grid(a2d_service* S, const std::vector<int>& ks, const std::vector<const void*>& ms, void* stream) {
  std::vector<std::vector<int>> lk;
  std::vector<std::vector<const void*>> lm;
  by_lane(S, ks, ms, 1, lk, lm);
  for (size_t l = 0; l < S->lanes.size(); ++l)
    if (!lk[l].empty())
      if (int e = a2d_case_set_grid(S->lanes[l].plan, (int)lk[l].size(), lk[l].data(), lm[l].data(), stream)) return e;
  return A2D_OK;
}

int restart(a2d_service* S, const std::vector<int>& ks, const std::vector<double>& w, int keep, void* stream) {
  std::vector<std::vector<int>> lk;
  std::vector<std::vector<double>> lw;
  by_lane(S, ks, w, 4, lk, lw);
  for (size_t l = 0; l < S->lanes.size(); ++l)
    if (!lk[l].empty())
      if (int e = a2d_case_restart(S->lanes[l].plan, (int)lk[l].size(), lk[l].data(), lw[l].data(), keep, stream))
        return e;
  return A2D_OK;
}

int retire(a2d_service* S, const std::vector<int>& ks, void* stream) {
  std::vector<std::vector<int>> lk;
  std::vector<std::vector<int>> unused;
  by_lane(S, ks, std::vector<int>(ks.size()), 1, lk, unused);
  for (size_t l = 0; l < S->lanes.size(); ++l)
    if (!lk[l].empty())
      if (int e = a2d_case_retire(S->lanes[l].plan, (int)lk[l].size(), lk[l].data(), stream)) return e;
  return A2D_OK;
}

void destroy(a2d_service* S) {
  for (a2d_service::Lane& L : S->lanes) {
    a2d_plan_destroy(L.plan);
    if (L.done != nullptr) cudaEventDestroy(L.done);
    if (L.stream != nullptr) cudaStreamDestroy(L.stream);
  }
  if (S->fork != nullptr) cudaEventDestroy(S->fork);
  delete S;
}

}  // namespace

extern "C" {

int a2d_service_create_lanes(int nclasses, const int* ni, const int* nc, const void* const* metrics,
                             const int* slots, int lanes, const a2d_params* params, a2d_service** out) {
  if (out == nullptr || nclasses < 1 || ni == nullptr || nc == nullptr || metrics == nullptr || slots == nullptr ||
      lanes < 1)
    return fail(A2D_ERR_ARG, "service_create: bad arguments");
  a2d_params p;
  a2d_default_params(&p);
  if (params != nullptr) p = *params;
  p.retire = 1;   // a slot stops stepping as soon as its point is done
  a2d_service* S = new a2d_service();
  int most = 0;
  for (int c = 0; c < nclasses; ++c) {
    if (slots[c] < 1 || metrics[c] == nullptr || class_of(S, ni[c], nc[c]) >= 0) {
      delete S;
      return fail(A2D_ERR_ARG, "service_create: each class needs slots >= 1, a grid, and its own size");
    }
    a2d_service::Class k;
    k.ni = ni[c];
    k.nc = nc[c];
    k.first = S->slots;
    k.count = slots[c];
    k.metrics = metrics[c];
    S->classes.push_back(k);
    S->slots += slots[c];
    most = std::max(most, slots[c]);
  }
  // every lane gets a case: at most as many lanes as the largest class has slots
  const int nl = std::min(lanes, most);
  S->lanes.resize(nl);
  S->slot_lane.resize(S->slots);
  S->slot_local.resize(S->slots);
  for (int c = 0; c < nclasses; ++c) {
    for (int q = 0; q < slots[c]; ++q) {
      const int k = S->classes[c].first + q;
      a2d_service::Lane& L = S->lanes[q % nl];
      S->slot_cls.push_back(c);
      S->slot_lane[k] = q % nl;
      S->slot_local[k] = (int)L.slots.size();
      L.slots.push_back(k);
      L.cp_off.push_back(L.total_ni);
      L.total_ni += ni[c];
    }
  }
  for (a2d_service::Lane& L : S->lanes) {
    const int n = (int)L.slots.size();
    std::vector<int> vni(n), vnc(n);
    std::vector<const void*> vm(n);
    std::vector<double> winf(4 * (size_t)n);
    for (int q = 0; q < n; ++q) {
      const a2d_service::Class& k = S->classes[S->slot_cls[L.slots[q]]];
      vni[q] = k.ni;
      vnc[q] = k.nc;
      vm[q] = k.metrics;
      winf[4 * q + 0] = 1.0;   // placeholder freestream until a request is admitted
      winf[4 * q + 1] = 0.5;
      winf[4 * q + 2] = 0.0;
      winf[4 * q + 3] = 1.0 / 1.4;
    }
    if (int e = a2d_plan_create(n, vni.data(), vnc.data(), vm.data(), winf.data(), &p, &L.plan)) {
      destroy(S);
      return e;
    }
  }
  S->max_iter = p.max_iter;
  S->slot_metrics.resize(S->slots);
  for (int k = 0; k < S->slots; ++k) S->slot_metrics[k] = S->classes[S->slot_cls[k]].metrics;
  S->slot_req.assign(S->slots, -1);
  S->slot_pt.assign(S->slots, 0);
  *out = S;
  return A2D_OK;
}

int a2d_service_create_ragged(int nclasses, const int* ni, const int* nc, const void* const* metrics,
                              const int* slots, const a2d_params* params, a2d_service** out) {
  return a2d_service_create_lanes(nclasses, ni, nc, metrics, slots, 1, params, out);
}

int a2d_service_create(int ni, int nc, const void* metrics, int slots, const a2d_params* params,
                       a2d_service** out) {
  return a2d_service_create_ragged(1, &ni, &nc, &metrics, &slots, params, out);
}

int a2d_service_workspace_bytes(const a2d_service* S, size_t* bytes) {
  if (S == nullptr || bytes == nullptr) return fail(A2D_ERR_ARG, "null service");
  size_t total = 0;
  for (const a2d_service::Lane& L : S->lanes) {
    size_t b = 0;
    if (int e = a2d_plan_workspace_bytes(L.plan, &b)) return e;
    total += (b + 255) & ~size_t(255);
  }
  *bytes = total;
  return A2D_OK;
}

int a2d_service_bind(a2d_service* S, void* workspace, size_t bytes, void* stream) {
  if (S == nullptr) return fail(A2D_ERR_ARG, "null service");
  size_t need = 0;
  if (int e = a2d_service_workspace_bytes(S, &need)) return e;
  if (workspace == nullptr || bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return fail(A2D_ERR_ARG, "service_bind: workspace too small or not 256-byte aligned");
  size_t off = 0;
  for (a2d_service::Lane& L : S->lanes) {
    if (int e = a2d_plan_workspace_bytes(L.plan, &L.ws_bytes)) return e;
    L.ws_off = off;
    if (int e = a2d_plan_bind(L.plan, static_cast<unsigned char*>(workspace) + off, L.ws_bytes, stream)) return e;
    off += (L.ws_bytes + 255) & ~size_t(255);
    if (S->lanes.size() > 1 && L.stream == nullptr) {
      if (cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) != cudaSuccess)
        return fail(A2D_ERR_CUDA, "service_bind: lane stream");
    }
  }
  if (S->lanes.size() > 1 && S->fork == nullptr &&
      cudaEventCreateWithFlags(&S->fork, cudaEventDisableTiming) != cudaSuccess)
    return fail(A2D_ERR_CUDA, "service_bind: lane event");
  // every slot starts idle
  std::vector<int> all(S->slots);
  for (int k = 0; k < S->slots; ++k) all[k] = k;
  return retire(S, all, stream);
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
    if (int e = set_grid(S, regrid, regrid_m, stream)) return e;
  if (!start.empty())
    if (int e = restart(S, start, start_w, 0, stream)) return e;
  const int nl = (int)S->lanes.size();
  std::vector<int> lane_busy(nl, 0);
  int nbusy = 0;
  for (int k = 0; k < S->slots; ++k)
    if (S->slot_req[k] >= 0) {
      nbusy += 1;
      lane_busy[S->slot_lane[k]] += 1;
    }
  if (busy != nullptr) *busy = nbusy;
  if (nbusy == 0) return A2D_OK;

  // one Newton step of every busy lane: on the caller's stream for a single lane, else
  // each on its own stream, forked from and joined back into the caller's
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  if (nl == 1) {
    if (int e = a2d_newton_step(S->lanes[0].plan, stream)) return e;
  } else {
    if (cudaEventRecord(S->fork, cs) != cudaSuccess) return fail(A2D_ERR_CUDA, "service_step: fork");
    for (int l = 0; l < nl; ++l) {
      a2d_service::Lane& L = S->lanes[l];
      if (lane_busy[l] == 0) continue;
      if (cudaStreamWaitEvent(L.stream, S->fork, 0) != cudaSuccess) return fail(A2D_ERR_CUDA, "service_step: fork");
      if (int e = a2d_newton_step(L.plan, L.stream)) return e;
      if (cudaEventRecord(L.done, L.stream) != cudaSuccess || cudaStreamWaitEvent(cs, L.done, 0) != cudaSuccess)
        return fail(A2D_ERR_CUDA, "service_step: join");
    }
  }
  S->newton_steps += 1;
  std::vector<int> nsteps(S->slots, 0), done(S->slots, 0), frozen(S->slots, 0);
  std::vector<double> lastrn(S->slots, 0.0), r0(S->slots, 1.0);
  for (int l = 0; l < nl; ++l) {
    const a2d_service::Lane& L = S->lanes[l];
    if (lane_busy[l] == 0) continue;
    const size_t n = L.slots.size();
    std::vector<int> ns(n), dn(n), fz(n);
    std::vector<double> lr(n), rr(n);
    if (int e = a2d_case_status(L.plan, ns.data(), dn.data(), fz.data(), lr.data(), rr.data(), stream)) return e;
    for (size_t q = 0; q < n; ++q) {
      const int k = L.slots[q];
      nsteps[k] = ns[q];
      done[k] = dn[q];
      frozen[k] = fz[q];
      lastrn[k] = lr[q];
      r0[k] = rr[q];
    }
  }
  std::vector<int> ended;
  std::vector<int> lane_ended(nl, 0);
  for (int k = 0; k < S->slots; ++k)
    if (S->slot_req[k] >= 0 && (done[k] || frozen[k] || nsteps[k] >= S->max_iter)) {
      ended.push_back(k);
      lane_ended[S->slot_lane[k]] = 1;
    }
  if (ended.empty()) return A2D_OK;

  // results of the points that ended, then the next points (or free slots)
  std::vector<std::vector<double>> coef(nl), cp(nl);
  for (int l = 0; l < nl; ++l) {
    if (!lane_ended[l]) continue;
    const a2d_service::Lane& L = S->lanes[l];
    coef[l].resize(3 * L.slots.size());
    cp[l].resize((size_t)L.total_ni);
    if (int e = a2d_case_forces(L.plan, coef[l].data(), cp[l].data(), stream)) return e;
  }
  std::vector<int> keep_k, fresh_k, retire_k;
  std::vector<double> keep_w, fresh_w;
  for (int k : ended) {
    const long long rid = S->slot_req[k];
    a2d_service::Request& r = S->reqs[rid];
    const int ni = S->classes[r.cls].ni;
    const int pt = S->slot_pt[k];
    const int l = S->slot_lane[k], q = S->slot_local[k];
    for (int c = 0; c < 3; ++c) r.coef[3 * (size_t)pt + c] = coef[l][3 * (size_t)q + c];
    const long long o = S->lanes[l].cp_off[q];
    std::copy(cp[l].begin() + o, cp[l].begin() + o + ni, r.cp.begin() + (size_t)pt * ni);
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
    if (int e = restart(S, keep_k, keep_w, 1, stream)) return e;
  if (!fresh_k.empty())
    if (int e = restart(S, fresh_k, fresh_w, 0, stream)) return e;
  if (!retire_k.empty()) {
    if (int e = retire(S, retire_k, stream)) return e;
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
      if (int e = set_grid(S, back, back_m, stream)) return e;
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
  *plan = S->lanes[0].plan;
  return A2D_OK;
}

int a2d_service_lanes(const a2d_service* S, int* lanes) {
  if (S == nullptr || lanes == nullptr) return fail(A2D_ERR_ARG, "service_lanes: bad arguments");
  *lanes = (int)S->lanes.size();
  return A2D_OK;
}

int a2d_service_lane(a2d_service* S, int lane, a2d_plan** plan, int* nslots, int* slots) {
  if (S == nullptr || lane < 0 || lane >= (int)S->lanes.size())
    return fail(A2D_ERR_ARG, "service_lane: bad arguments");
  const a2d_service::Lane& L = S->lanes[lane];
  if (plan != nullptr) *plan = L.plan;
  if (nslots != nullptr) *nslots = (int)L.slots.size();
  if (slots != nullptr) std::copy(L.slots.begin(), L.slots.end(), slots);
  return A2D_OK;
}

int a2d_service_stats(a2d_service* S, int* kernels_per_step, long long* newton_steps) {
  if (S == nullptr) return fail(A2D_ERR_ARG, "null service");
  std::lock_guard<std::mutex> lk(S->mu);
  if (newton_steps != nullptr) *newton_steps = S->newton_steps;
  if (kernels_per_step != nullptr) {
    int total = 0;
    for (const a2d_service::Lane& L : S->lanes) {
      int k = 0;
      if (int e = a2d_plan_stats(L.plan, &k, nullptr, nullptr)) return e;
      total += k;
    }
    *kernels_per_step = total;
  }
  return A2D_OK;
}

int a2d_service_destroy(a2d_service* S) {
  if (S == nullptr) return A2D_OK;
  destroy(S);
  return A2D_OK;
}

}  // extern "C"
