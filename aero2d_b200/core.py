"""Polar scenario on the Euler path: the reference's `run_euler` and its
`Polar` record (aero2d/core.py:20-45, :220-260) on this backend.

`run_euler(af, alphas, mach, grid, n_iter, callback)` re-panels the contour to
the grid level's points per side (geometry.repanel, as aero2d/core.py:236
does for every input), marches the level's O-grid (far field 40 chords),
solves every angle of attack as one batch with ImplicitEuler in FP32 (tol
1e-6, all angles stepped in lockstep until every one is done, as the
reference's loop does) and returns a `Polar` with Cl, Cd, Cm, the wall Cp at
the wall-face midpoints and the per-angle convergence flags, with the
reference's notes for unconverged angles.  With `continuation=True` the angles
are instead solved one after another from the previous angle's state (alpha
continuation) through EulerService.  `af` is an Airfoil or a NACA 4-digit code
(built as naca4(code), the reference's default resolution, then re-panelled).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .geometry import Airfoil, naca4, repanel
from .grid import ogrid

# grid levels: (points per side of the contour, nodes along the normal, first spacing),
# the reference's table (aero2d/core.py:13-18) with its keys and English aliases
GRIDS = {
    "грубая (быстро)": (65, 49, 2e-3),
    "средняя": (97, 65, 1.5e-3),
    "мелкая (медленно)": (129, 97, 1e-3),
}
GRID_ALIASES = {"coarse": "грубая (быстро)", "medium": "средняя", "fine": "мелкая (медленно)"}
FARFIELD_RADIUS = 40.0


@dataclass
class Polar:
    """One polar (the fields of aero2d/core.py:20-45 that the Euler path fills)."""
    label: str
    method: str
    mach: float
    alpha: np.ndarray
    cl: np.ndarray
    cd: np.ndarray
    cm: np.ndarray
    ok: np.ndarray                      # converged
    cp_x: list = field(default_factory=list)
    cp: list = field(default_factory=list)
    notes: list = field(default_factory=list)
    re: float = float("nan")
    chord_ref: float = 1.0
    xref: tuple = (0.25, 0.0)
    nsteps: Optional[np.ndarray] = None  # Newton steps per angle


def _level(grid: str) -> tuple[int, int, float]:
    key = GRID_ALIASES.get(grid, grid)
    if key not in GRIDS:
        raise ValueError(f"unknown grid level {grid!r}; one of {list(GRIDS) + list(GRID_ALIASES)}")
    return GRIDS[key]


def euler_grid(af, grid: str = "грубая (быстро)"):
    """The re-panelled contour and O-grid of a grid level (aero2d/core.py:234-236)."""
    nside, nj, ds0 = _level(grid)
    if isinstance(af, str):
        af = naca4(af)
    if not isinstance(af, Airfoil):
        raise TypeError("af must be an Airfoil or a NACA 4-digit code")
    af = repanel(af, nside)
    return af, ogrid(af, nj=nj, ds0=ds0, radius=FARFIELD_RADIUS)


def run_euler(af, alphas, mach: float, grid: str = "грубая (быстро)", n_iter: int = 100, callback=None,
              continuation: bool = False, device=None) -> Polar:
    """All angles of attack in one batch (aero2d/core.py:220-260).
    callback(text, fraction) -> True stops early."""
    from .euler import EulerSolver
    from .implicit import ImplicitEuler

    if mach < 0.2:
        raise ValueError("the Euler solver does not run below M = 0.2 (no low-Mach preconditioning); "
                         "use the panel method")
    af, g = euler_grid(af, grid)
    alphas = np.asarray(alphas, float)
    if callback:
        callback("grid built", 0.0)
    if continuation:
        from .service import EulerService
        svc = EulerService(g, slots=1, dtype=np.float32, device=device, tol=1e-6, max_iter=n_iter)
        rid = svc.submit(mach, alphas, continuation=True)
        svc.run()
        r = svc.result(rid)
        cl, cd, cm, cp, ok, nsteps = r["cl"], r["cd"], r["cm"], r["cp"], r["converged"], r["nsteps"]
        svc.close()
        from .euler import compute_metrics
        xw = np.asarray(compute_metrics(g).xw)
    else:
        # lockstep like the reference's loop: every angle steps until all are done, so an angle
        # that converges early is iterated further exactly as the reference returns it
        solver = ImplicitEuler(EulerSolver(g, dtype=np.float32, device=device), retire=False)

        def cb(it, n, logres, clv):
            if callback is None:
                return False
            worst = np.nanmax(logres) if np.any(np.isfinite(logres)) else 0.0
            return callback(f"iteration {it}/{n}: residual down {-worst:.1f} orders (worst case)", it / n)

        r = solver.solve(np.full_like(alphas, mach), alphas, n_iter=n_iter, tol=1e-6, verbose=False, callback=cb)
        xw = np.asarray(solver.b.m_np.xw)
        cl, cd, cm, cp = r.cl, r.cd, r.cm, r.cp
        ok = np.asarray(r.converged, bool)
        nsteps = np.asarray(getattr(solver, "steps_taken", np.full(alphas.shape, -1)))
    notes = []
    if not np.all(ok):
        notes.append(f"not converged: alpha = {', '.join(f'{a:g}' for a in alphas[~ok])} deg; their values are "
                     "unreliable (usually transonic with strong shocks, or high alpha). Try a finer grid or more "
                     "iterations.")
    notes.append("Euler is inviscid: Cd is wave drag only (shocks); no friction and no stall.")
    name = af.name if getattr(af, "name", None) else "airfoil"
    return Polar(f"{name}, Euler ({GRID_ALIASES.get(grid, grid).split(' ')[0]}), M={mach:g}", "euler", float(mach),
                 alphas, np.asarray(cl), np.asarray(cd), np.asarray(cm), ok, [xw] * len(alphas),
                 [np.asarray(c) for c in cp], notes, nsteps=np.asarray(nsteps))


def critical_cp(mach: float, gamma: float = 1.4) -> float:
    """Pressure coefficient at which the local flow is sonic (isentropic)."""
    m2 = mach * mach
    return 2.0 / (gamma * m2) * (((2.0 + (gamma - 1.0) * m2) / (gamma + 1.0)) ** (gamma / (gamma - 1.0)) - 1.0)


def shock_position(xw, yw, cp, mach: float) -> float:
    """Chordwise position of the upper-surface shock: where the wall Cp (at the
    wall-face midpoints xw, yw) rises through the critical Cp* going aft, at the
    crossing with the steepest dCp/dx, linearly interpolated; NaN if the flow on
    the upper surface never turns supersonic.  The reference defines no shock
    position; this is the measure the transonic comparisons of mixed against
    FP64 solutions use."""
    xw, yw, cp = (np.asarray(a, float) for a in (xw, yw, cp))
    le = int(np.argmin(xw))
    a, b = np.arange(0, le + 1), np.arange(le, len(xw))
    upper = a if yw[a].mean() > yw[b].mean() else b
    order = upper[np.argsort(xw[upper])]
    x, c = xw[order], cp[order]
    cs = critical_cp(mach)
    best, best_slope = float("nan"), 0.0
    for q in range(len(x) - 1):
        if c[q] < cs <= c[q + 1] and x[q + 1] > x[q]:
            slope = (c[q + 1] - c[q]) / (x[q + 1] - x[q])
            if slope > best_slope:
                best_slope = slope
                best = x[q] + (cs - c[q]) / (c[q + 1] - c[q]) * (x[q + 1] - x[q])
    return best
