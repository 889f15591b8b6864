"""Continuous-batching Euler service: served polar sweeps.

The slots of one batched Newton-Krylov plan are grouped in classes by grid
size.  A request is a polar sweep -- a Mach number and a list of angles of
attack -- on one grid, solved point after point in one slot of that grid's
size, each point started from the previous point's state (alpha continuation)
unless `continuation=False`.  Before every Newton step, queued requests are
admitted in arrival order into free slots of their class, so the batch stays
full instead of draining to its slowest case (the serving pattern of the
reference's polar callers, which loop over ImplicitEuler.solve:
aero2d/core.py:220-260).  A request can bring its own grid (a DeviceGrid of a
class's size, e.g. from gridgen.ogrid_batch for a new airfoil); the service
keeps it alive until the request's result is taken.  The work runs in the
library's C ABI (a2d_service_*, include/aero2d_b200.h); this class owns the
device workspace.

    svc = EulerService(grid, slots=64)                       # one grid size
    svc = EulerService(classes=[(g128, 16), (g256, 16)])     # ragged slots
    rid = svc.submit(0.5, np.arange(-4, 17, 1.0), grid=dg)   # dg: that request's grid
    done = svc.run()                 # or svc.step() in your own loop + svc.poll()
    res = svc.result(rid)            # dict: alpha, cl, cd, cm, cp, converged, nsteps, drop
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .euler import GAMMA, _precision_of
from .grid import OGrid
from .plan import DeviceGrid, _ptr, device_of, stream_handle


def freestream(mach, alpha_deg) -> np.ndarray:
    """Freestream primitives (rho, u, v, p) per point (aero2d/euler.py:253-256)."""
    mach = np.asarray(mach, np.float64)
    a = np.deg2rad(np.asarray(alpha_deg, np.float64))
    one = np.ones_like(mach)
    return np.stack([one, mach * np.cos(a), mach * np.sin(a), one / GAMMA], axis=-1)


def workspace_bytes_per_slot(ni: int, nc: int, gmres_restart: int = 30, dtype=np.float32) -> int:
    """Device bytes one slot of an ni x nc grid takes in a service workspace
    (host-side query: no device memory is touched)."""
    lib = _lib.load()
    p = _lib.default_params()
    p.gmres_restart = int(gmres_restart)
    p.precision = _precision_of(dtype)
    sizes = []
    for n in (1, 2):
        h = C.c_void_p()
        _lib.check(lib.a2d_plan_create(n, (C.c_int * n)(*[ni] * n), (C.c_int * n)(*[nc] * n),
                                       (C.c_void_p * n)(*[1] * n), (C.c_double * (4 * n))(*([1.0, 0.5, 0.0, 0.7] * n)),
                                       C.byref(p), C.byref(h)))
        b = C.c_size_t()
        _lib.check(lib.a2d_plan_workspace_bytes(h, C.byref(b)))
        lib.a2d_plan_destroy(h)
        sizes.append(b.value)
    return sizes[1] - sizes[0]


def slots_for_budget(shapes: Sequence[tuple[int, int]], hbm_bytes: int, share: Optional[Sequence[float]] = None,
                     gmres_restart: int = 30, dtype=np.float32) -> list[int]:
    """Slots per grid size that fit `hbm_bytes` of workspace, the budget split
    by `share` (default: equal bytes per size); at least one slot per size."""
    share = np.full(len(shapes), 1.0 / len(shapes)) if share is None else np.asarray(share, float) / np.sum(share)
    per = [workspace_bytes_per_slot(ni, nc, gmres_restart, dtype) for ni, nc in shapes]
    return [max(1, int(hbm_bytes * s // b)) for s, b in zip(share, per)]


class EulerService:
    def __init__(self, grid: OGrid | DeviceGrid | None = None, slots: int = 64, dtype=np.float32, device=None,
                 tol: float = 1e-8, max_iter: int = 200, gmres_restart: int = 30, cfl0: float = 10.0,
                 cfl_max: float = 300.0, gmres_tol: float = 0.01, jacobi_sweeps: int = 4,
                 max_update: float = 0.2, classes: Optional[Sequence[tuple]] = None, tuning="cached",
                 lanes: Optional[int] = None):
        """`grid` + `slots` for one grid size, or `classes` = [(grid, slots), ...]
        with one grid per size (the class's default grid).  `tuning` as for
        plan.Plan: "cached", "auto" (measured on the idle slots at creation on a
        cache miss), None, or a (jvp_tile, sweep) pair.  `lanes`: plans the slots
        are dealt to, stepped concurrently on their own streams (default: one per
        16 slots of the largest class, at most 4)."""
        if classes is None:
            if grid is None:
                raise ValueError("give a grid (and slots) or classes")
            classes = [(grid, slots)]
        self.device = device_of(device)
        self.classes = []
        for g, n in classes:
            dg = g if isinstance(g, DeviceGrid) else DeviceGrid(g, self.device)
            self.classes.append((dg, int(n)))
        shapes = [(dg.ni, dg.nc) for dg, _ in self.classes]
        if len(set(shapes)) != len(shapes):
            raise ValueError("each slot class needs its own grid size")
        self._shape = {s: k for k, s in enumerate(shapes)}
        p = _lib.default_params()
        p.precision = _precision_of(dtype)
        for k, v in dict(gmres_restart=int(gmres_restart), gmres_tol=float(gmres_tol), cfl0=float(cfl0),
                         cfl_max=float(cfl_max), max_update=float(max_update), tol=float(tol),
                         jacobi_sweeps=int(jacobi_sweeps), max_iter=int(max_iter), retire=1).items():
            setattr(p, k, v)
        self.lib = _lib.load()
        m = len(self.classes)
        if lanes is None:
            lanes = default_lanes([n for _, n in self.classes])
        h = C.c_void_p()
        _lib.check(self.lib.a2d_service_create_lanes(
            m, (C.c_int * m)(*[s[0] for s in shapes]), (C.c_int * m)(*[s[1] for s in shapes]),
            (C.c_void_p * m)(*[dg.ptr for dg, _ in self.classes]), (C.c_int * m)(*[n for _, n in self.classes]),
            int(lanes), C.byref(p), C.byref(h)))
        self.handle = h
        nl = C.c_int()
        _lib.check(self.lib.a2d_service_lanes(h, C.byref(nl)))
        self.lanes = nl.value
        n = C.c_size_t()
        _lib.check(self.lib.a2d_service_workspace_bytes(h, C.byref(n)))
        self.workspace_bytes = n.value
        self.workspace = torch.empty(n.value, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.a2d_service_bind(h, _ptr(self.workspace), n.value, self.stream))
        self._meta: dict[int, tuple] = {}
        self._params = p
        if tuning is not None:
            self._tune(tuning)

    def _tune(self, tuning) -> None:
        """Applies (or, with "auto" on a cache miss, measures on the first lane's
        plan) the launch configuration of every lane while every slot is idle,
        then retires every slot again."""
        from . import autotune
        view = _PlanView(self)
        if isinstance(tuning, str):
            measured = tuning == "auto" and autotune.TuningCache().get(autotune.plan_key(view)) is None
            autotune.apply(view, measure=(tuning == "auto"))
            if measured:
                view.retire_all()
        else:
            view.set_tuning(*tuning)

    def tuning(self) -> tuple[str, str]:
        return _PlanView(self).tuning()

    @property
    def stream(self) -> int:
        return stream_handle(self.device)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.a2d_service_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, mach: float, alphas, continuation: bool = True, grid: DeviceGrid | None = None) -> int:
        """Queues a sweep of `alphas` (degrees) at `mach` on `grid` (a DeviceGrid
        of a class's size; default: the first class's grid); returns the id."""
        alphas = np.atleast_1d(np.asarray(alphas, np.float64))
        if alphas.size == 0:
            raise ValueError("a request needs at least one angle of attack")
        dg = grid if grid is not None else self.classes[0][0]
        if (dg.ni, dg.nc) not in self._shape:
            raise ValueError(f"no slot class for a {dg.ni} x {dg.nc} grid")
        winf = np.ascontiguousarray(freestream(np.full(alphas.shape, float(mach)), alphas))
        rid = C.c_longlong()
        _lib.check(self.lib.a2d_service_submit_grid(self.handle, dg.ni, dg.nc, C.c_void_p(dg.ptr), alphas.size,
                                                    winf.ctypes.data_as(C.POINTER(C.c_double)),
                                                    int(bool(continuation)), C.byref(rid)))
        self._meta[rid.value] = (float(mach), alphas, dg)
        return rid.value

    def step(self) -> int:
        """Admits queued requests, takes one Newton step of the busy slots and
        collects finished points; returns the number of busy slots."""
        busy = C.c_int()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.a2d_service_step(self.handle, C.byref(busy), self.stream))
        return busy.value

    def poll(self, max_ids: int = 1024) -> list[int]:
        """Ids of the requests finished since the last poll."""
        ids = (C.c_longlong * max_ids)()
        n = C.c_int()
        _lib.check(self.lib.a2d_service_poll(self.handle, ids, max_ids, C.byref(n)))
        return [ids[q] for q in range(n.value)]

    def pending(self) -> tuple[int, int]:
        """(queued requests, busy slots)."""
        q, r = C.c_int(), C.c_int()
        _lib.check(self.lib.a2d_service_pending(self.handle, C.byref(q), C.byref(r)))
        return q.value, r.value

    def stats(self) -> tuple[int, int]:
        """(kernel launches of one Newton step, Newton steps taken since bind)."""
        k, n = C.c_int(), C.c_longlong()
        _lib.check(self.lib.a2d_service_stats(self.handle, C.byref(k), C.byref(n)))
        return k.value, n.value

    def result(self, rid: int) -> dict:
        """A finished request's per-point results; releases the request (and its grid)."""
        mach, alphas, dg = self._meta[rid]
        n = alphas.size
        coef = np.empty((n, 3))
        cp = np.empty((n, dg.ni))
        conv = np.empty(n, np.int32)
        steps = np.empty(n, np.int32)
        drop = np.empty(n)
        _lib.check(self.lib.a2d_service_result_drop(self.handle, C.c_longlong(rid),
                                                    drop.ctypes.data_as(C.POINTER(C.c_double))))
        _lib.check(self.lib.a2d_service_result(self.handle, C.c_longlong(rid),
                                               coef.ctypes.data_as(C.POINTER(C.c_double)),
                                               cp.ctypes.data_as(C.POINTER(C.c_double)),
                                               conv.ctypes.data_as(C.POINTER(C.c_int)),
                                               steps.ctypes.data_as(C.POINTER(C.c_int))))
        del self._meta[rid]
        return {"mach": mach, "alpha": alphas, "cl": coef[:, 0], "cd": coef[:, 1], "cm": coef[:, 2], "cp": cp,
                "converged": conv.astype(bool), "nsteps": steps, "drop": drop}

    def run(self, max_steps: Optional[int] = None) -> list[int]:
        """Steps until the queue and every slot are empty (or max_steps steps);
        returns the ids finished meanwhile."""
        done: list[int] = []
        k = 0
        while True:
            busy = self.step()
            done += self.poll()
            k += 1
            if busy == 0 and self.pending()[0] == 0:
                break
            if max_steps is not None and k >= max_steps:
                break
        return done


def default_lanes(class_slots: Sequence[int]) -> int:
    """Lanes of a service: one per 16 slots of its largest class, 1 to 4 (four
    16-case plans of the 256 x 64 benchmark step 6 % faster than one 64-case plan)."""
    return max(1, min(4, max(class_slots) // 16))


class _PlanView:
    """The service's lanes seen as one plan.Plan by the autotuner: a launch
    configuration is set on every lane, and a Newton step steps every lane
    concurrently on its own stream (as a2d_service_step does), so that the
    configuration is timed under the load it will serve.  `shapes` are the first
    lane's cases and `lanes` the lane count (both part of the tuning key)."""

    def __init__(self, svc: "EulerService"):
        self.lib, self.device, self.params = svc.lib, svc.device, svc._params
        slot_shape = [(dg.ni, dg.nc) for dg, n in svc.classes for _ in range(n)]
        self.handles, self.counts = [], []
        for lane in range(svc.lanes):
            h, n = C.c_void_p(), C.c_int()
            _lib.check(svc.lib.a2d_service_lane(svc.handle, lane, C.byref(h), C.byref(n), None))
            if lane == 0:
                ids = (C.c_int * n.value)()
                _lib.check(svc.lib.a2d_service_lane(svc.handle, 0, None, None, ids))
                self.shapes = [slot_shape[k] for k in ids]
            self.handles.append(h)
            self.counts.append(n.value)
        self.handle = self.handles[0]
        self.lanes = len(self.handles)
        self._streams = None

    def _each(self, name, *args):
        with torch.cuda.device(self.device):
            for h in self.handles:
                _lib.check(getattr(self.lib, name)(h, *args, stream_handle(self.device)))

    def set_tuning(self, jvp_tile: str = "32x16", sweep: str = "halves") -> None:
        self._each("a2d_plan_set_tuning", _lib.JVP_TILES[jvp_tile], _lib.SWEEP_VARIANTS[sweep])

    def tuning(self) -> tuple[str, str]:
        t, v = C.c_int(), C.c_int()
        _lib.check(self.lib.a2d_plan_get_tuning(self.handle, C.byref(t), C.byref(v)))
        return ({b: a for a, b in _lib.JVP_TILES.items()}[t.value],
                {b: a for a, b in _lib.SWEEP_VARIANTS.items()}[v.value])

    def init_freestream(self) -> None:
        self._each("a2d_init_freestream")

    def newton_step(self) -> None:
        with torch.cuda.device(self.device):
            if self.lanes == 1:
                _lib.check(self.lib.a2d_newton_step(self.handle, stream_handle(self.device)))
                return
            if self._streams is None:
                self._streams = [torch.cuda.Stream(self.device) for _ in self.handles]
            cur = torch.cuda.current_stream(self.device)
            fork = torch.cuda.Event()
            fork.record(cur)
            for h, st in zip(self.handles, self._streams):
                st.wait_event(fork)
                _lib.check(self.lib.a2d_newton_step(h, st.cuda_stream))
                cur.wait_stream(st)

    def retire_all(self) -> None:
        with torch.cuda.device(self.device):
            for h, n in zip(self.handles, self.counts):
                _lib.check(self.lib.a2d_case_retire(h, n, (C.c_int * n)(*range(n)), stream_handle(self.device)))
