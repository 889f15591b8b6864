"""Continuous-batching Euler service: served polar sweeps on one grid.

A fixed number of slots of one batched Newton-Krylov plan share an O-grid.  A
request is a polar sweep -- a Mach number and a list of angles of attack --
solved point after point in one slot, each point started from the previous
point's state (alpha continuation) unless `continuation=False`; a slot freed
by a finished request is refilled from the queue before the next Newton step,
so the batch stays full instead of draining to its slowest case (the serving
pattern of the reference's polar callers, which loop over
ImplicitEuler.solve: aero2d/core.py:220-260).  The work runs in the library's
C ABI (a2d_service_*, include/aero2d_b200.h); this class owns the device
workspace and converts (M, alpha) to freestreams with EulerSolver.freestream.

    svc = EulerService(grid, slots=64)
    rid = svc.submit(0.5, np.arange(-4, 17, 1.0))
    done = svc.run()                 # or svc.step() in your own loop + svc.poll()
    res = svc.result(rid)            # dict: alpha, cl, cd, cm, cp, converged, nsteps
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from .euler import EulerSolver
from .grid import OGrid
from .plan import DeviceGrid, _ptr, device_of, stream_handle


class EulerService:
    def __init__(self, grid: OGrid, slots: int = 64, dtype=np.float32, device=None, tol: float = 1e-8,
                 max_iter: int = 200, gmres_restart: int = 30, cfl0: float = 10.0, cfl_max: float = 300.0,
                 gmres_tol: float = 0.01, jacobi_sweeps: int = 4, max_update: float = 0.2):
        self.device = device_of(device)
        self.base = EulerSolver(grid, dtype=dtype, device=self.device)
        self.dgrid: DeviceGrid = self.base.dgrid
        self.slots = int(slots)
        p = self.base.params(gmres_restart=int(gmres_restart), gmres_tol=float(gmres_tol), cfl0=float(cfl0),
                             cfl_max=float(cfl_max), max_update=float(max_update), tol=float(tol),
                             jacobi_sweeps=int(jacobi_sweeps), max_iter=int(max_iter), retire=1)
        self.lib = _lib.load()
        h = C.c_void_p()
        _lib.check(self.lib.a2d_service_create(self.dgrid.ni, self.dgrid.nc, C.c_void_p(self.dgrid.ptr), self.slots,
                                               C.byref(p), C.byref(h)))
        self.handle = h
        n = C.c_size_t()
        _lib.check(self.lib.a2d_service_workspace_bytes(h, C.byref(n)))
        self.workspace = torch.empty(n.value, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.a2d_service_bind(h, _ptr(self.workspace), n.value, self.stream))
        self._meta: dict[int, tuple[float, np.ndarray]] = {}

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

    def submit(self, mach: float, alphas, continuation: bool = True) -> int:
        """Queues a sweep of `alphas` (degrees) at `mach`; returns the request id."""
        alphas = np.atleast_1d(np.asarray(alphas, np.float64))
        if alphas.size == 0:
            raise ValueError("a request needs at least one angle of attack")
        winf = np.ascontiguousarray(self.base.freestream(np.full(alphas.shape, float(mach)), alphas))
        rid = C.c_longlong()
        _lib.check(self.lib.a2d_service_submit(self.handle, alphas.size,
                                               winf.ctypes.data_as(C.POINTER(C.c_double)), int(bool(continuation)),
                                               C.byref(rid)))
        self._meta[rid.value] = (float(mach), alphas)
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

    def result(self, rid: int) -> dict:
        """A finished request's per-point results; releases the request."""
        mach, alphas = self._meta.pop(rid)
        n = alphas.size
        coef = np.empty((n, 3))
        cp = np.empty((n, self.dgrid.ni))
        conv = np.empty(n, np.int32)
        steps = np.empty(n, np.int32)
        _lib.check(self.lib.a2d_service_result(self.handle, C.c_longlong(rid),
                                               coef.ctypes.data_as(C.POINTER(C.c_double)),
                                               cp.ctypes.data_as(C.POINTER(C.c_double)),
                                               conv.ctypes.data_as(C.POINTER(C.c_int)),
                                               steps.ctypes.data_as(C.POINTER(C.c_int))))
        return {"mach": mach, "alpha": alphas, "cl": coef[:, 0], "cd": coef[:, 1], "cm": coef[:, 2], "cp": cp,
                "converged": conv.astype(bool), "nsteps": steps}

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
