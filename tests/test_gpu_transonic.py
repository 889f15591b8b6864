"""Transonic accuracy of the mixed-precision path against FP64 (the shape of
the transonic configuration: random NACA 4-digit airfoils, each on its own
384 x 96 O-grid with first spacing 1e-3 chord and radius 20, M ~ U[0.70, 0.80],
alpha ~ U[0, 3] deg, one ragged batch per precision, Newton-Krylov to a 1e-10
drop, at most 300 steps).  Shocked cases often stall short of that drop (the
reference's own M 0.85 benchmark case stops at -4.6; on this draw five of the
eight do, and the three that fall 8 orders in both precisions all carry an
upper-surface shock); on every case whose residual fell 8 orders in both: |dCl| <= 1e-4, |dCd| <= 2e-6, and
an upper-surface shock, where there is one, within 2e-3 chord."""
import numpy as np
import pytest

from aero2d_b200.core import shock_position
from aero2d_b200.euler import EulerSolver, compute_metrics
from aero2d_b200.geometry import naca4_params
from aero2d_b200.grid import GridError, ogrid
from aero2d_b200.implicit import ImplicitEuler
from aero2d_b200.plan import Plan

pytestmark = pytest.mark.gpu


def test_transonic_mixed_vs_fp64(cuda):
    rng = np.random.default_rng(2025)
    grids, rejected = [], 0
    while len(grids) < 8:
        af = naca4_params(rng.uniform(0, 0.06), rng.uniform(0.2, 0.6), rng.uniform(0.08, 0.16), 193)
        try:
            grids.append(ogrid(af, nj=97, ds0=1e-3, radius=20.0))
        except GridError:
            rejected += 1
    B = len(grids)
    machs, alphas = rng.uniform(0.70, 0.80, B), rng.uniform(0.0, 3.0, B)
    out = {}
    for dt in (np.float64, np.float32):
        solvers = [EulerSolver(g, dtype=dt, device=cuda) for g in grids]
        imp = ImplicitEuler(solvers[0], gmres_restart=30)
        pl = Plan([s.dgrid for s in solvers], solvers[0].freestream(machs, alphas), imp.params(1e-10, 300), cuda)
        pl.init_freestream()
        pl.newton_run(300)
        nsteps, done, frozen, lastrn, r0 = pl.status()
        coef, cps = pl.forces()
        out[dt] = (~frozen & (lastrn < 1e-8 * r0), coef.cpu().numpy(), [c.cpu().numpy() for c in cps])
        pl.close()
    ok = out[np.float64][0] & out[np.float32][0]
    assert ok.sum() >= 3, f"only {ok.sum()} of {B} transonic cases fell 8 orders in both precisions"
    shocks = 0
    for k in np.nonzero(ok)[0]:
        c64, c32 = out[np.float64][1][k], out[np.float32][1][k]
        assert abs(c64[0] - c32[0]) <= 1e-4
        assert abs(c64[1] - c32[1]) <= 2e-6
        mt = compute_metrics(grids[k])
        s64 = shock_position(mt.xw, mt.yw, out[np.float64][2][k], machs[k])
        s32 = shock_position(mt.xw, mt.yw, out[np.float32][2][k], machs[k])
        assert np.isnan(s64) == np.isnan(s32)
        if not np.isnan(s64):
            shocks += 1
            assert abs(s64 - s32) <= 2e-3
    print(f"transonic: {ok.sum()} of {B} cases compared, {shocks} with an upper-surface shock, "
          f"{rejected} airfoils redrawn")
