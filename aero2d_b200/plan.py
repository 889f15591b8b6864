"""Device plumbing between the Python solvers and the C ABI: grids uploaded
with their metrics, and batch plans bound to a caller-owned workspace.

PyTorch is used here only to own device memory and to name the CUDA stream;
all arithmetic of the Euler path runs in libaero2d_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .grid import OGrid


def device_of(device=None) -> torch.device:
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None
    if device is None:
        raise _lib.ExtensionMissing("aero2d_b200 needs a CUDA device; none is available")
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError("aero2d_b200 runs on CUDA devices only")
    return device


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


class DeviceGrid:
    """An O-grid resident on the device: node coordinates and the metrics blob
    (cell areas, face vectors, wall and far-field face midpoints, FP64 and FP32)."""

    def __init__(self, grid: OGrid | None = None, device=None, *, nodes: tuple | None = None):
        """From a host OGrid, or from node coordinates already on the device
        (`nodes=(x, y)`, contiguous FP64 tensors (ni, nj), as the device grid
        generator writes them)."""
        lib = _lib.load()
        if nodes is not None:
            self.x, self.y = nodes
            self.device = self.x.device
            if self.x.dtype != torch.float64 or self.x.shape != self.y.shape or self.x.dim() != 2 \
                    or not (self.x.is_contiguous() and self.y.is_contiguous()):
                raise ValueError("nodes must be two contiguous float64 (ni, nj) device tensors")
            ni, nj = self.x.shape
        else:
            self.device = device_of(device)
            ni, nj = grid.shape
            self.x = torch.as_tensor(np.ascontiguousarray(grid.x, np.float64), device=self.device)
            self.y = torch.as_tensor(np.ascontiguousarray(grid.y, np.float64), device=self.device)
        self.ni, self.nj, self.nc = ni, nj, nj - 1
        n = C.c_size_t()
        _lib.check(lib.a2d_metrics_bytes(ni, nj, C.byref(n)))
        self.metrics = torch.empty(n.value, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(lib.a2d_metrics_build(ni, nj, _ptr(self.x), _ptr(self.y), _ptr(self.metrics),
                                             stream_handle(self.device)))

    @property
    def ptr(self) -> int:
        return _ptr(self.metrics)


class Plan:
    """A batch of cases bound to one device workspace (include/aero2d_b200.h).

    `tuning`: the launch configuration (aero2d_b200.autotune): "cached" (the
    default) applies the autotuner's stored choice for this plan's grid sizes
    and precision if there is one; "auto" also measures and stores it when there
    is none; None keeps the library's starting configuration (32x16 JVP tiles and
    the halves sweep; FP64 plans the lanes sweep); a (jvp_tile, sweep) pair sets it.
    Results do not depend on it."""

    def __init__(self, grids: list[DeviceGrid], winf: np.ndarray, params: _lib.Params, device=None,
                 tuning="cached"):
        lib = _lib.load()
        self.lib = lib
        self.device = device_of(device if device is not None else grids[0].device)
        self.grids = list(grids)
        self.B = len(grids)
        self.params = params
        winf = np.ascontiguousarray(np.asarray(winf, np.float64).reshape(self.B, 4))
        ni = (C.c_int * self.B)(*[g.ni for g in grids])
        nc = (C.c_int * self.B)(*[g.nc for g in grids])
        mp = (C.c_void_p * self.B)(*[g.ptr for g in grids])
        wv = (C.c_double * (4 * self.B))(*winf.ravel())
        h = C.c_void_p()
        _lib.check(lib.a2d_plan_create(self.B, ni, nc, mp, wv, C.byref(params), C.byref(h)))
        self.handle = h
        n = C.c_size_t()
        _lib.check(lib.a2d_plan_workspace_bytes(h, C.byref(n)))
        self.workspace = torch.empty(n.value, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(lib.a2d_plan_bind(h, _ptr(self.workspace), n.value, self.stream))
        self.total_ni = sum(g.ni for g in grids)
        if tuning is not None:
            from . import autotune
            if isinstance(tuning, str):
                autotune.apply(self, measure=(tuning == "auto"))
            else:
                self.set_tuning(*tuning)

    @property
    def shapes(self) -> list[tuple[int, int]]:
        return [(g.ni, g.nc) for g in self.grids]

    def set_tuning(self, jvp_tile: str = "32x16", sweep: str = "halves") -> None:
        """The launch configuration: the FP32 JVP's tile shape and the line
        sweep's kernel variant (include/aero2d_b200.h, A2D_JVP_TILE_*, A2D_SWEEP_*)."""
        with torch.cuda.device(self.device):
            _lib.check(self.lib.a2d_plan_set_tuning(self.handle, _lib.JVP_TILES[jvp_tile],
                                                    _lib.SWEEP_VARIANTS[sweep], self.stream))

    def tuning(self) -> tuple[str, str]:
        t, v = C.c_int(), C.c_int()
        _lib.check(self.lib.a2d_plan_get_tuning(self.handle, C.byref(t), C.byref(v)))
        inv_t = {b: a for a, b in _lib.JVP_TILES.items()}
        inv_v = {b: a for a, b in _lib.SWEEP_VARIANTS.items()}
        return inv_t[t.value], inv_v[v.value]

    @property
    def stream(self) -> int:
        return stream_handle(self.device)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.a2d_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- vector I/O in the reference layout (4, ni, nc) ----------------------
    def set_vec(self, slot: int, k: int, src: torch.Tensor) -> None:
        g = self.grids[k]
        src = torch.as_tensor(src, dtype=torch.float64, device=self.device).contiguous()
        if tuple(src.shape) != (4, g.ni, g.nc):
            raise ValueError(f"state of case {k} must have shape (4, {g.ni}, {g.nc}), got {tuple(src.shape)}")
        with torch.cuda.device(self.device):
            _lib.check(self.lib.a2d_vec_set(self.handle, slot, k, _ptr(src), self.stream))
        self._keep = src

    def get_vec(self, slot: int, k: int) -> torch.Tensor:
        g = self.grids[k]
        out = torch.empty((4, g.ni, g.nc), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.a2d_vec_get(self.handle, slot, k, _ptr(out), self.stream))
        return out

    def get_prim(self, slot: int, k: int) -> torch.Tensor:
        """Primitives (rho, u, v, p) of a slot's vector of case k, (4, ni, nc)."""
        g = self.grids[k]
        out = torch.empty((4, g.ni, g.nc), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.a2d_vec_get_prim(self.handle, slot, k, _ptr(out), self.stream))
        return out

    def local_dt(self, k: int, W) -> torch.Tensor:
        """Local time steps (ni, nc) of case k from primitives W (4, ni, nc)."""
        g = self.grids[k]
        W = torch.as_tensor(W, dtype=torch.float64, device=self.device).contiguous()
        if tuple(W.shape) != (4, g.ni, g.nc):
            raise ValueError(f"W of case {k} must have shape (4, {g.ni}, {g.nc}), got {tuple(W.shape)}")
        dt = torch.empty((g.ni, g.nc), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.a2d_local_dt(self.handle, k, _ptr(W), _ptr(dt), self.stream))
        return dt

    def set_batch(self, slot: int, U: torch.Tensor) -> None:
        for k in range(self.B):
            self.set_vec(slot, k, U[k])

    def get_batch(self, slot: int) -> torch.Tensor:
        return torch.stack([self.get_vec(slot, k) for k in range(self.B)])

    # -- operations ------------------------------------------------------------
    def call(self, name: str, *args) -> None:
        with torch.cuda.device(self.device):
            _lib.check(getattr(self.lib, name)(self.handle, *args, self.stream))

    def init_freestream(self):
        self.call("a2d_init_freestream")

    def reset(self):
        self.call("a2d_reset")

    def residual(self, circ: torch.Tensor | None = None):
        self.call("a2d_residual", None if circ is None else _ptr(circ))

    def jvp(self):
        self.call("a2d_jvp")

    def forces(self):
        coef = torch.empty((self.B, 3), dtype=torch.float64, device=self.device)
        cp = torch.empty(self.total_ni, dtype=torch.float64, device=self.device)
        self.call("a2d_forces", _ptr(coef), _ptr(cp))
        cps = []
        o = 0
        for g in self.grids:
            cps.append(cp[o:o + g.ni])
            o += g.ni
        return coef, cps

    def precond_setup(self):
        self.call("a2d_precond_setup")

    def precond_apply(self):
        self.call("a2d_precond_apply")

    def set_cfl(self, cfl):
        arr = (C.c_double * self.B)(*np.broadcast_to(np.asarray(cfl, np.float64), (self.B,)))
        self.call("a2d_set_cfl", arr)

    def set_circulation(self, circ):
        arr = (C.c_double * self.B)(*np.broadcast_to(np.asarray(circ, np.float64), (self.B,)))
        self.call("a2d_set_circulation", arr)

    def newton_step(self):
        self.call("a2d_newton_step")

    def newton_run(self, max_steps: int) -> int:
        n = C.c_int()
        self.call("a2d_newton_run", int(max_steps), C.byref(n))
        return n.value

    def live_count(self) -> int:
        n = C.c_int()
        self.call("a2d_live_count", C.byref(n))
        return n.value

    def factor_saturations(self, reset: bool = False) -> int:
        """Sweep-factor entries stored saturated in FP16 since bind (mixed plans)."""
        n = C.c_ulonglong()
        self.call("a2d_factor_saturations", C.byref(n), int(bool(reset)))
        return int(n.value)

    def stats(self):
        """(kernel launches per Newton step, Newton steps since reset)."""
        k, s = C.c_int(), C.c_int()
        _lib.check(self.lib.a2d_plan_stats(self.handle, C.byref(k), C.byref(s), None))
        return k.value, s.value

    def table_bytes(self) -> int:
        """Bytes of the case tables copied to the device at bind time."""
        n = C.c_size_t()
        _lib.check(self.lib.a2d_plan_stats(self.handle, None, None, C.byref(n)))
        return n.value

    def time_kernel(self, which: int, reps: int = 20) -> float:
        """Mean milliseconds per launch of one kernel on the plan's data (CUDA events)."""
        ms = C.c_float()
        self.call("a2d_time_kernel", int(which), int(reps), C.byref(ms))
        return float(ms.value)

    def status(self):
        B = self.B
        nsteps = (C.c_int * B)()
        done = (C.c_int * B)()
        frozen = (C.c_int * B)()
        lastrn = (C.c_double * B)()
        r0 = (C.c_double * B)()
        self.call("a2d_case_status", nsteps, done, frozen, lastrn, r0)
        return (np.array(nsteps[:], int), np.array(done[:], bool), np.array(frozen[:], bool),
                np.array(lastrn[:]), np.array(r0[:]))

    def scalars(self) -> np.ndarray:
        """(B, 8): rn, omega, cfl, r0, circulation, beta, Arnoldi vectors, committed."""
        out = np.zeros(8 * self.B)
        self.call("a2d_case_scalars", out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.reshape(self.B, 8)

    def history(self, steps: int):
        B = self.B
        rn = np.full(steps * B, np.nan)
        cl = np.full(steps * B, np.nan)
        if steps:
            self.call("a2d_history", int(steps), rn.ctypes.data_as(C.POINTER(C.c_double)),
                      cl.ctypes.data_as(C.POINTER(C.c_double)))
        return rn.reshape(steps, B), cl.reshape(steps, B)

    def rk_iterate(self, n: int) -> torch.Tensor:
        res = torch.empty(self.B, dtype=torch.float64, device=self.device)
        self.call("a2d_rk_iterate", int(n), _ptr(res))
        return res

    def smooth(self):
        self.call("a2d_smooth")


def hllc_flux_device(WL: torch.Tensor, WR: torch.Tensor, S: torch.Tensor) -> torch.Tensor:
    """Point-wise HLLC flux on the device: WL, WR (4, n), S (2, n) -> (4, n)."""
    lib = _lib.load()
    dev = WL.device
    WL = WL.to(torch.float64).contiguous()
    WR = WR.to(torch.float64).contiguous()
    S = S.to(torch.float64).contiguous()
    n = WL.shape[1]
    F = torch.empty((4, n), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        _lib.check(lib.a2d_hllc_flux(n, _ptr(WL), _ptr(WR), _ptr(S), _ptr(F), stream_handle(dev)))
    return F
