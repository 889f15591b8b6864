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
    assert g.x.shape == (128, 49)
    af2, g2 = euler_grid(naca4("0012", 65), "грубая (быстро)")
    assert np.array_equal(g.x, g2.x) and np.array_equal(g.y, g2.y)


def test_coarse_level_is_the_reference_benchmark_grid(ref_grids):
    _, g = euler_grid("0012", "coarse")
    assert np.array_equal(g.x, ref_grids["0012_65_49_x"]) and np.array_equal(g.y, ref_grids["0012_65_49_y"])


def test_euler_grid_rejects_other_resolutions():
    with pytest.raises(NotImplementedError):
        euler_grid(naca4("0012", 100), "coarse")
    with pytest.raises(ValueError):
        euler_grid("0012", "extra fine")


def test_low_mach_rejected_before_any_device_work():
    with pytest.raises(ValueError):
        run_euler("0012", [0.0, 2.0], 0.15)


def test_polar_record_fields():
    p = Polar("x", "euler", 0.5, np.zeros(2), np.zeros(2), np.zeros(2), np.zeros(2), np.ones(2, bool))
    assert p.method == "euler" and p.xref == (0.25, 0.0) and np.isnan(p.re)
