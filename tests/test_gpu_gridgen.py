"""Device O-grid generation (aero2d/grid.py:50-81) against the reference's grids."""
import numpy as np
import pytest
import torch

from aero2d_b200.euler import EulerSolver
from aero2d_b200.geometry import naca4, naca4_params
from aero2d_b200.grid import GridError, ogrid
from aero2d_b200.gridgen import ogrid_batch
from aero2d_b200.implicit import ImplicitEuler
from tests.golden.make_golden import GRIDS

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("key", list(GRIDS))
def test_device_grid_matches_reference(cuda, ref_grids, key):
    """Layers 0 .. nj-2 bitwise; the outer circle within a few ulps of its radius."""
    code, ns, nj, ds0, rad = GRIDS[key]
    (g,) = ogrid_batch([naca4(code, ns)], nj=nj, ds0=ds0, radius=rad, device=cuda)
    x, y = g.x.cpu().numpy(), g.y.cpu().numpy()
    rx, ry = ref_grids[f"{key}_x"], ref_grids[f"{key}_y"]
    assert np.array_equal(x[:, :-1], rx[:, :-1]) and np.array_equal(y[:, :-1], ry[:, :-1])
    assert np.max(np.abs(x[:, -1] - rx[:, -1])) < 8 * np.finfo(float).eps * rad
    assert np.max(np.abs(y[:, -1] - ry[:, -1])) < 8 * np.finfo(float).eps * rad


def test_batch_of_mixed_airfoils(cuda):
    """Several airfoils and two ring sizes in one call: each grid as the host
    generator makes it (float NACA parameters, as random airfoil requests use)."""
    rng = np.random.default_rng(7)
    afs = [naca4_params(rng.uniform(0, 0.06), rng.uniform(0.2, 0.6), rng.uniform(0.08, 0.16), ns)
           for ns in (65, 97, 65, 97, 65)]
    grids = ogrid_batch(afs, nj=33, ds0=2e-3, radius=20.0, device=cuda)
    for af, g in zip(afs, grids):
        h = ogrid(af, nj=33, ds0=2e-3, radius=20.0)
        x, y = g.x.cpu().numpy(), g.y.cpu().numpy()
        assert np.array_equal(x[:, :-1], h.x[:, :-1]) and np.array_equal(y[:, :-1], h.y[:, :-1])
        assert np.max(np.abs(x[:, -1] - h.x[:, -1])) < 1e-13


def test_inverted_grid_raises_on_device(cuda):
    with pytest.raises(GridError):
        ogrid_batch([naca4("0012", 65), naca4("6412", 193)], nj=97, ds0=1e-3, radius=20.0, device=cuda)


def test_converged_forces_on_device_grid(cuda):
    """FP64 Newton-Krylov on the device-built grid and on the host grid: the
    outer-circle rounding moves the converged Cl by less than 1e-10."""
    af = naca4("2412", 33)
    host = ogrid(af, nj=25, ds0=2e-3, radius=20.0)
    (dg,) = ogrid_batch([af], nj=25, ds0=2e-3, radius=20.0, device=cuda)
    base = EulerSolver(host, dtype=np.float64, device=cuda)
    r_host = ImplicitEuler(base, gmres_restart=30).solve([0.5], [2.0], n_iter=200, tol=1e-11, verbose=False)
    base.dgrid = dg
    r_dev = ImplicitEuler(base, gmres_restart=30).solve([0.5], [2.0], n_iter=200, tol=1e-11, verbose=False)
    assert r_host.converged[0] and r_dev.converged[0]
    assert abs(r_host.cl[0] - r_dev.cl[0]) < 1e-10
    assert abs(r_host.cd[0] - r_dev.cd[0]) < 1e-10
