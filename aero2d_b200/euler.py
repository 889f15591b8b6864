"""Batched 2-D Euler solver on the O-grid, B200 implementation.

Drop-in for aero2d/euler.py: the same names (GAMMA, Metrics, compute_metrics,
cons_to_prim, prim_to_cons, hllc_flux, van_albada, wall_ghost-free residual,
EulerSolver, EulerResult) with the same arguments and error behaviour.  The
residual, forces, residual smoothing and the explicit RK4 iteration run in the
CUDA library through the C ABI; the batch of (M, alpha) cases on one grid is
one launch (the reference's jax.vmap axis, aero2d/euler.py:393-408).

Nondimensionalisation: rho_inf = 1, a_inf = 1, p_inf = 1/gamma, |V_inf| = M.
States are torch tensors on the CUDA device, shape (4, ni, nc) per case or
(B, 4, ni, nc) per batch; host arrays are accepted wherever states go in.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .grid import OGrid
from .plan import DeviceGrid, Plan, device_of, hllc_flux_device

GAMMA = 1.4
LIMITER = "smooth"    # the reference default; the CUDA residual implements this limiter


# ---------------------------------------------------------------------------
# metrics on the host (FP64), as aero2d/euler.py:33-60 returns them; the device
# computes the same arrays itself from the node coordinates
# ---------------------------------------------------------------------------
@dataclass
class Metrics:
    vol: np.ndarray      # (ni, nc)        cell areas
    Si: np.ndarray       # (2, ni, nc)     face between cells i-1 and i, toward +i
    Sj: np.ndarray       # (2, ni, nc+1)   face j (0 = wall), toward +j
    xc: np.ndarray       # (ni, nc)        cell centres
    yc: np.ndarray
    xw: np.ndarray       # (ni,)           wall face midpoints
    yw: np.ndarray


def compute_metrics(g: OGrid) -> Metrics:
    x, y = g.x.astype(np.float64), g.y.astype(np.float64)
    vol = g.cell_areas()
    dx = x[:, 1:] - x[:, :-1]
    dy = y[:, 1:] - y[:, :-1]
    Si = np.stack([-dy, dx])
    x1, y1 = np.roll(x, -1, 0), np.roll(y, -1, 0)
    Sj = np.stack([y1 - y, -(x1 - x)])
    xc = 0.25 * (x[:, :-1] + x[:, 1:] + x1[:, :-1] + x1[:, 1:])
    yc = 0.25 * (y[:, :-1] + y[:, 1:] + y1[:, :-1] + y1[:, 1:])
    xw = 0.5 * (x[:, 0] + x1[:, 0])
    yw = 0.5 * (y[:, 0] + y1[:, 0])
    return Metrics(vol, Si, Sj, xc, yc, xw, yw)


# ---------------------------------------------------------------------------
# thermodynamics and the point flux
# ---------------------------------------------------------------------------
def _stack(xs, like):
    if isinstance(like, torch.Tensor):
        return torch.stack(list(xs))
    return np.stack(list(xs))


def cons_to_prim(U):
    """(rho, rho u, rho v, E) -> (rho, u, v, p) along the first axis."""
    rho = U[0]
    u = U[1] / rho
    v = U[2] / rho
    p = (GAMMA - 1) * (U[3] - 0.5 * rho * (u * u + v * v))
    return _stack([rho, u, v, p], U)


def prim_to_cons(W):
    rho, u, v, p = W[0], W[1], W[2], W[3]
    return _stack([rho, rho * u, rho * v, p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v)], W)


def hllc_flux(WL, WR, S):
    """HLLC flux through faces with area vectors S (2, ...), evaluated by the
    CUDA point kernel; returns the input's array type (aero2d/euler.py:79-121)."""
    as_np = not isinstance(WL, torch.Tensor)
    dev = device_of(WL.device if isinstance(WL, torch.Tensor) else None)
    WLt = torch.as_tensor(np.asarray(WL) if as_np else WL, dtype=torch.float64, device=dev)
    WRt = torch.as_tensor(np.asarray(WR) if as_np else WR, dtype=torch.float64, device=dev)
    St = torch.as_tensor(np.asarray(S) if as_np else S, dtype=torch.float64, device=dev)
    shape = WLt.shape[1:]
    F = hllc_flux_device(WLt.reshape(4, -1), WRt.reshape(4, -1), St.reshape(2, -1)).reshape(4, *shape)
    return F.cpu().numpy() if as_np else F


def van_albada(a, b, eps):
    """Smooth van Albada slope (aero2d/euler.py:127-136, LIMITER = "smooth")."""
    eps = eps + 1e-20
    return ((b * b + eps) * a + (a * a + eps) * b) / (a * a + b * b + 2 * eps)


def _precision_of(dtype) -> int:
    """float64 -> all-FP64 path; float32 -> mixed precision for the implicit
    solver (FP32 linearisation and Krylov basis around an FP64 residual,
    factorisation and update) and the FP32 explicit iteration (residual, local
    time steps, smoothing and stage update in FP32)."""
    name = getattr(dtype, "__name__", None) or str(dtype)
    try:
        name = np.dtype(dtype).name
    except TypeError:
        pass
    if "float64" in name or name in ("double", "f8"):
        return _lib.A2D_FP64
    if "float32" in name or name in ("float", "f4"):
        return _lib.A2D_MIXED
    raise ValueError(f"unsupported dtype {dtype!r}: use float32 or float64")


@dataclass
class EulerResult:
    mach: np.ndarray
    alpha: np.ndarray
    cl: np.ndarray
    cd: np.ndarray
    cm: np.ndarray
    cp: np.ndarray        # (B, ni) on the wall faces
    res_hist: np.ndarray  # (n, B)
    U: torch.Tensor       # (B, 4, ni, nc) on the device
    converged: np.ndarray | None = None


class EulerSolver:
    """Finite-volume Euler discretisation and the explicit RK4 + IRS solver
    (aero2d/euler.py:218-435)."""

    def __init__(self, grid: OGrid, dtype=np.float32, cfl: float = 2.5, irs_eps: float = 0.6,
                 order: int = 2, vortex_correction: bool = True, mg_levels: int = 1,
                 lim_k: float = 0.02, device=None):
        self.dtype = dtype
        self.precision = _precision_of(dtype)
        self.grid = grid
        self.m_np = compute_metrics(grid)
        self.ni, self.nc = self.m_np.vol.shape
        self.cfl, self.irs_eps, self.order, self.lim_k = cfl, irs_eps, order, lim_k
        self.vortex = vortex_correction
        # FAS multigrid (experimental in the reference, unstable below M 0.6 there;
        # ImplicitEuler is the production solver): every other node in i and j,
        # first order (aero2d/euler.py:241-250)
        self.coarse = None
        if mg_levels > 1 and (self.ni % 2 or self.nc % 2):
            raise ValueError("multigrid needs an even number of cells in i and j")
        self.device = device_of(device)
        if mg_levels > 1:
            cg = OGrid(np.ascontiguousarray(grid.x[::2, ::2]), np.ascontiguousarray(grid.y[::2, ::2]))
            self.coarse = EulerSolver(cg, dtype, cfl, irs_eps, order=1, vortex_correction=vortex_correction,
                                      mg_levels=mg_levels - 1, device=self.device)
        self.dgrid = DeviceGrid(grid, self.device)
        self._plans = {}

    # -- configuration shared with the implicit solver -----------------------
    def params(self, **over) -> _lib.Params:
        p = _lib.default_params()
        p.cfl = float(self.cfl)
        p.irs_eps = float(self.irs_eps)
        p.lim_k = float(self.lim_k)
        p.order = int(self.order)
        p.vortex_correction = int(bool(self.vortex))
        p.precision = int(self.precision)
        for k, v in over.items():
            setattr(p, k, v)
        return p

    def _plan(self, winf: np.ndarray, **over) -> Plan:
        winf = np.asarray(winf, np.float64).reshape(-1, 4)
        key = (winf.tobytes(), tuple(sorted(over.items())))
        pl = self._plans.get(key)
        if pl is None:
            if len(self._plans) > 8:
                self._plans.clear()
            pl = Plan([self.dgrid] * len(winf), winf, self.params(**over), self.device)
            self._plans[key] = pl
        return pl

    # -- freestream ------------------------------------------------------------
    def freestream(self, mach, alpha_deg):
        """Freestream primitives (aero2d/euler.py:253-256); arrays give (B, 4)."""
        mach = np.asarray(mach, np.float64)
        a = np.deg2rad(np.asarray(alpha_deg, np.float64))
        one = np.ones_like(mach)
        w = np.stack([one, mach * np.cos(a), mach * np.sin(a), one / GAMMA], axis=-1)
        return w

    def init_state(self, winf):
        w = np.asarray(winf, np.float64)
        Uc = prim_to_cons(w.reshape(4, 1, 1) if w.ndim == 1 else w.T[:, :, None, None])
        if w.ndim == 1:
            return torch.as_tensor(np.broadcast_to(Uc, (4, self.ni, self.nc)).copy(), device=self.device)
        B = w.shape[0]
        U = np.broadcast_to(Uc, (4, B, self.ni, self.nc)).transpose(1, 0, 2, 3).copy()
        return torch.as_tensor(U, device=self.device)

    # -- single-case operations --------------------------------------------------
    def residual(self, U, winf, circ=None):
        """(R, W) for one case (aero2d/euler.py:259-287).  circ=None takes the
        circulation from U itself (Gamma = Cl M / 2, as ImplicitEuler does)."""
        pl = self._plan(winf)
        pl.set_vec(_lib.VEC_U, 0, U)
        c = None
        if circ is not None:
            c = torch.full((1,), float(circ), dtype=torch.float64, device=self.device)
        pl.residual(c)
        return pl.get_vec(_lib.VEC_R, 0), pl.get_prim(_lib.VEC_U, 0)

    def local_dt(self, W):
        """Local time steps (ni, nc) of one case from its primitives W (4, ni, nc):
        cfl * vol / (lambda_i + lambda_j) (aero2d/euler.py:289-296)."""
        pl = self._plan(np.array([1.0, 0.5, 0.0, 1 / GAMMA]))
        return pl.local_dt(0, W)

    def forces(self, U, winf):
        """(cl, cd, cm, cp) of one case (aero2d/euler.py:318-331)."""
        pl = self._plan(winf)
        pl.set_vec(_lib.VEC_U, 0, U)
        coef, cps = pl.forces()
        c = coef[0].cpu().numpy()
        return float(c[0]), float(c[1]), float(c[2]), cps[0]

    def smooth(self, R):
        """Implicit residual smoothing of one residual field (aero2d/euler.py:298-312)."""
        pl = self._plan(np.array([1.0, 0.5, 0.0, 1 / GAMMA]))
        pl.set_vec(_lib.VEC_R, 0, R)
        pl.smooth()
        return pl.get_vec(_lib.VEC_R, 0)

    def wall_pressure(self, W):
        return 1.5 * W[3, :, 0] - 0.5 * W[3, :, 1]

    # -- explicit batch solve -------------------------------------------------
    def solve(self, machs, alphas, n_iter=4000, chunk=200, tol=1e-7, verbose=True, U0=None,
              tol_cl=2e-5, tol_cd=2e-6) -> EulerResult:
        """Batch RK4 + IRS run with the reference's stop tests (aero2d/euler.py:386-435)."""
        machs = np.atleast_1d(np.asarray(machs, np.float64))
        alphas = np.atleast_1d(np.asarray(alphas, np.float64))
        if machs.shape != alphas.shape:
            raise ValueError("machs and alphas must have the same length")
        winf = self.freestream(machs, alphas)
        B = len(machs)
        pl = Plan([self.dgrid] * B, winf, self.params(), self.device)
        levels = [pl]                # FAS levels, finest first, linked fine -> coarse
        lvl = self.coarse
        while lvl is not None:
            levels.append(Plan([lvl.dgrid] * B, winf, lvl.params(), self.device))
            _lib.check(pl.lib.a2d_plan_set_coarse(levels[-2].handle, levels[-1].handle))
            lvl = lvl.coarse
        if U0 is None:
            pl.init_freestream()
        else:
            pl.set_batch(_lib.VEC_U, torch.as_tensor(U0, dtype=torch.float64, device=self.device))
        pl.set_circulation(np.zeros(B))
        hist, clh, cdh = [], [], []
        res0 = None
        self.iterations = 0
        for it in range(0, n_iter, chunk):
            res = pl.rk_iterate(chunk).cpu().numpy()
            self.iterations = it + chunk
            if res0 is None:
                res0 = res
            coef, _ = pl.forces()
            c = coef.cpu().numpy()
            cl, cd = c[:, 0], c[:, 1]
            hist.append(res)
            clh.append(cl)
            cdh.append(cd)
            if verbose:
                print(f"  iter {it + chunk:6d}  log10(res/res0) max {np.max(np.log10(res / res0)):+.2f}"
                      f"  Cl {np.array2string(cl, precision=4)}")
            if not np.all(np.isfinite(res)):
                break
            if np.all(res / res0 < tol):
                break
            if len(clh) > 2 and np.all(np.abs(clh[-1] - clh[-2]) < tol_cl) \
                    and np.all(np.abs(cdh[-1] - cdh[-2]) < tol_cd):
                break
        self.cl_history = np.array(clh)
        U = pl.get_batch(_lib.VEC_U)
        if not bool(torch.isfinite(U).all()):
            raise FloatingPointError("solution diverged (NaN)")
        coef, cps = pl.forces()
        c = coef.cpu().numpy()
        return EulerResult(machs, alphas, c[:, 0], c[:, 1], c[:, 2],
                           torch.stack(cps).cpu().numpy(), np.array(hist), U)
