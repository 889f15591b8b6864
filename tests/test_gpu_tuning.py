"""The launch-configuration knobs on the GPU: every (JVP tile shape, sweep
variant) takes bitwise the same Newton step, in FP64 and mixed precision, on a
ragged batch (three grid sizes); the autotuner measures, stores and re-applies a
choice through its cache."""
import numpy as np
import pytest
import torch

from aero2d_b200 import _lib, autotune
from aero2d_b200.euler import EulerSolver
from aero2d_b200.implicit import ImplicitEuler
from aero2d_b200.plan import Plan
from tests.helpers import grid

pytestmark = pytest.mark.gpu


def ragged_plan(dtype, cuda, tuning=None):
    # 128 x 32, 96 x 24 and 80 x 42 cells: the last has a half-full line group and a
    # twist row (21) whose wall-side back substitution ends on a short pack of the
    # sweeps' ring (packs of four C blocks); the others end short on the far-field side
    ga, gb, gc = grid("2412", 65, 33), grid("0012", 49, 25), grid("4412", 41, 43)
    sa, sb, sc = (EulerSolver(g, dtype=dtype, device=cuda) for g in (ga, gb, gc))
    imp = ImplicitEuler(sa, gmres_restart=20)
    machs, alphas = np.array([0.5, 0.7, 0.6, 0.55]), np.array([2.0, 1.0, -1.0, 3.0])
    return Plan([sa.dgrid, sb.dgrid, sa.dgrid, sc.dgrid], sa.freestream(machs, alphas), imp.params(1e-10, 20), cuda,
                tuning=tuning)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_every_configuration_takes_the_same_step(cuda, dtype):
    pl = ragged_plan(dtype, cuda)
    ref = None
    for t, v in autotune.candidates(_lib.A2D_MIXED if dtype == np.float32 else _lib.A2D_FP64):
        pl.set_tuning(t, v)
        assert pl.tuning() == (t, v)
        pl.init_freestream()
        for _ in range(3):
            pl.newton_step()
        U = [pl.get_vec(_lib.VEC_U, k) for k in range(pl.B)]   # ragged: one tensor per case
        sc = pl.scalars()
        if ref is None:
            ref = (U, sc)
        else:
            assert all(torch.equal(a, b) for a, b in zip(U, ref[0])), (t, v)
            assert np.array_equal(sc, ref[1], equal_nan=True), (t, v)


def test_autotuner_measures_stores_and_reapplies(cuda, tmp_path, monkeypatch):
    monkeypatch.setenv("AERO2D_B200_TUNING", str(tmp_path / "tuning.json"))
    pl = ragged_plan(np.float32, cuda, tuning="auto")
    cache = autotune.TuningCache()
    key = autotune.plan_key(pl)
    choice = cache.get(key)
    assert choice is not None and pl.tuning() == choice
    assert len(cache.load()[key]["ms"]) == len(autotune.candidates(_lib.A2D_MIXED))
    pl2 = ragged_plan(np.float32, cuda, tuning="cached")
    assert pl2.tuning() == choice


def test_fp64_plans_start_on_lanes_and_refuse_rows(cuda):
    """The rows and halves sweeps run mixed-precision plans only: an FP64 plan starts
    with the lanes sweep and refuses them; a mixed plan starts with 32x16 tiles and
    the halves sweep."""
    p64 = ragged_plan(np.float64, cuda)
    assert p64.tuning()[1] == "lanes"
    for v in ("rows", "halves"):
        with pytest.raises(Exception, match="mixed-precision plans only"):
            p64.set_tuning("32x8", v)
    assert ragged_plan(np.float32, cuda).tuning() == ("32x16", "halves")
