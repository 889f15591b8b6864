"""The polar scenario (aero2d/core.py:220-260) on the host: grid levels,
contour checks and argument errors, without a GPU."""
import numpy as np
import pytest

from aero2d_b200.core import GRIDS, GRID_ALIASES, Polar, euler_grid, run_euler
from aero2d_b200.geometry import naca4


def test_grid_levels_match_the_reference_table():
    assert GRIDS["грубая (быстро)"] == (65, 49, 2e-3)
    assert GRIDS["средняя"] == (97, 65, 1.5e-3)
    assert GRIDS["мелкая (медленно)"] == (129, 97, 1e-3)
    assert set(GRID_ALIASES.values()) == set(GRIDS)


def test_euler_grid_from_code_and_airfoil():
    af, g = euler_grid("0012", "coarse")
    assert g.x.shape == (128, 49) and len(af.x) == 129
    af2, g2 = euler_grid(naca4("0012"), "грубая (быстро)")
    assert np.array_equal(g.x, g2.x) and np.array_equal(g.y, g2.y)
    with pytest.raises(TypeError):
        euler_grid(np.zeros((10, 2)), "coarse")


def test_coarse_level_is_the_reference_polar_grid():
    """The reference's polar grid, ogrid(repanel(naca4("0012"), 65), ...), bitwise."""
    from tests.conftest import GOLDEN
    d = np.load(GOLDEN / "ref_repanel.npz")
    _, g = euler_grid("0012", "coarse")
    assert np.array_equal(g.x, d["polar_coarse_0012_x"]) and np.array_equal(g.y, d["polar_coarse_0012_y"])


def test_any_contour_is_repanelled_to_the_level():
    af, g = euler_grid(naca4("2412", 40), "medium")
    assert len(af.x) == 2 * 97 - 1 and g.x.shape == (192, 65)
    with pytest.raises(ValueError):
        euler_grid("0012", "extra fine")


def test_multigrid_odd_grid_rejected_before_any_device_work():
    """aero2d/euler.py:245-246."""
    from aero2d_b200.euler import EulerSolver
    from aero2d_b200.grid import ogrid
    with pytest.raises(ValueError):
        EulerSolver(ogrid(naca4("0012", 33), nj=26), dtype=np.float64, mg_levels=2)


def test_low_mach_rejected_before_any_device_work():
    with pytest.raises(ValueError):
        run_euler("0012", [0.0, 2.0], 0.15)


def test_polar_record_fields():
    p = Polar("x", "euler", 0.5, np.zeros(2), np.zeros(2), np.zeros(2), np.zeros(2), np.ones(2, bool))
    assert p.method == "euler" and p.xref == (0.25, 0.0) and np.isnan(p.re)


def test_service_slot_budget_on_host():
    """Slot sizing and the ragged service's argument checks need no GPU."""
    import ctypes as C
    from aero2d_b200 import _lib
    from aero2d_b200.service import slots_for_budget, workspace_bytes_per_slot
    per = [workspace_bytes_per_slot(ni, nc) for ni, nc in [(128, 32), (192, 48), (256, 64), (384, 96)]]
    assert all(b > 0 for b in per) and per == sorted(per)
    n = slots_for_budget([(128, 32), (384, 96)], 10 * per[3], share=[1, 1])
    assert n == [int(5 * per[3] // per[0]), 5]
    lib = _lib.load()
    h = C.c_void_p()
    two = (C.c_int * 2)
    st = lib.a2d_service_create_ragged(2, two(128, 128), two(32, 32), (C.c_void_p * 2)(1, 1), two(1, 1), None,
                                       C.byref(h))
    assert st == _lib.A2D_ERR_ARG          # two classes of one size
    _lib.check(lib.a2d_service_create_ragged(2, two(128, 192), two(32, 48), (C.c_void_p * 2)(1, 1), two(2, 1), None,
                                             C.byref(h)))
    rid = C.c_longlong()
    w = (C.c_double * 4)(1.0, 0.5, 0.0, 1 / 1.4)
    assert lib.a2d_service_submit_grid(h, 256, 64, None, 1, w, 1, C.byref(rid)) == _lib.A2D_ERR_ARG
    _lib.check(lib.a2d_service_submit_grid(h, 192, 48, None, 1, w, 1, C.byref(rid)))
    q, r = C.c_int(), C.c_int()
    _lib.check(lib.a2d_service_pending(h, C.byref(q), C.byref(r)))
    assert (q.value, r.value) == (1, 0)
    _lib.check(lib.a2d_service_destroy(h))


def test_shock_position_of_a_synthetic_distribution():
    from aero2d_b200.core import critical_cp, shock_position
    assert abs(critical_cp(1.0)) < 1e-15 and critical_cp(0.8) < 0
    # upper surface y > 0 from the trailing edge to the leading edge, lower back
    x = np.concatenate([np.linspace(1, 0, 41), np.linspace(0, 1, 41)[1:]])
    y = np.concatenate([np.full(41, 0.05), np.full(40, -0.05)])
    cs = critical_cp(0.8)
    cp = np.where(y > 0, np.where(x < 0.6, cs - 0.4, cs + 0.3), 0.0)
    xs = shock_position(x, y, cp, 0.8)
    assert 0.575 < xs < 0.6
    assert np.isnan(shock_position(x, y, np.zeros_like(x), 0.8))
