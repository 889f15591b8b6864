"""The autotuner's host logic (no GPU): plan signatures, the candidate lists,
the on-disk cache (missing, corrupt and partial files, atomic writes) and the
choice of the fastest configuration, with a stand-in plan and timer."""
import json

import pytest

from aero2d_b200 import autotune


def test_signature_orders_sizes_and_rounds_counts():
    s = autotune.signature([(256, 64)] * 64 + [(128, 32)] * 3, precision=1)
    assert s == "mixed|128x32:4,256x64:64"
    assert autotune.signature([(256, 64)] * 33, 0) == "fp64|256x64:64"
    assert autotune.signature([(192, 48)], 0) == "fp64|192x48:1"


def test_candidates_by_precision():
    mixed = autotune.candidates(1)
    assert len(mixed) == len(autotune.JVP_TILES) * len(autotune.SWEEPS)
    assert set(t for t, _ in autotune.candidates(0)) == {"32x8"}
    assert not set(v for _, v in autotune.candidates(0)) & set(autotune.MIXED_ONLY_SWEEPS)
    assert autotune.DEFAULT in mixed


def test_cache_roundtrip_and_bad_files(tmp_path):
    path = tmp_path / "sub" / "tuning.json"
    cache = autotune.TuningCache(path)
    assert cache.load() == {} and cache.get("k") is None          # missing file
    cache.put("k", ("32x16", "rows"), {("32x16", "rows"): 1.5, ("32x8", "lanes"): 2.0})
    assert cache.get("k") == ("32x16", "rows")
    data = json.loads(path.read_text())
    assert data["k"]["ms"] == {"32x16/rows": 1.5, "32x8/lanes": 2.0}
    assert [p.name for p in path.parent.iterdir()] == ["tuning.json"]   # no temporary left behind
    cache.put("k2", ("64x4", "lanes"))
    assert cache.get("k") == ("32x16", "rows") and cache.get("k2") == ("64x4", "lanes")
    path.write_text("{not json")
    assert cache.load() == {}
    path.write_text(json.dumps({"a": {"jvp_tile": "7x7", "sweep": "lanes"}, "b": [1], "c": {"jvp_tile": "16x16",
                                                                                             "sweep": "rows"}}))
    assert cache.load() == {"c": {"jvp_tile": "16x16", "sweep": "rows"}}


def test_choose_takes_the_fastest_first_on_ties():
    t = {("32x8", "lanes"): 3.0, ("32x16", "lanes"): 2.0, ("32x16", "rows"): 2.0}
    assert autotune.choose(t) == ("32x16", "lanes")
    with pytest.raises(ValueError):
        autotune.choose({})


class FakeParams:
    precision = 1


class FakePlan:
    def __init__(self):
        self.params = FakeParams()
        self.config = autotune.DEFAULT
        self.inits = 0
        self.shapes = [(128, 32)] * 8

    def set_tuning(self, t, v):
        self.config = (t, v)

    def tuning(self):
        return self.config

    def init_freestream(self):
        self.inits += 1


def test_tune_and_apply_with_a_fake_timer(tmp_path, monkeypatch):
    cost = {("16x16", "rows"): 1.0}
    measure = lambda plan: cost.get(plan.config, 5.0)       # noqa: E731
    plan = FakePlan()
    best, timings = autotune.tune(plan, measure)
    assert best == ("16x16", "rows") and plan.config == best and plan.inits == 1
    assert len(timings) == len(autotune.candidates(1))

    monkeypatch.setattr(autotune, "plan_key", lambda p: "gpu|lib|" + autotune.signature(p.shapes, 1))
    cache = autotune.TuningCache(tmp_path / "t.json")
    fresh = FakePlan()
    assert autotune.apply(fresh, measure=False, cache=cache) == autotune.DEFAULT   # miss, not measured
    assert cache.load() == {}
    assert autotune.apply(fresh, measure=True, cache=cache, measure_fn=measure) == ("16x16", "rows")
    again = FakePlan()
    assert autotune.apply(again, measure=False, cache=cache) == ("16x16", "rows") and again.inits == 0


def test_plan_key_counts_lanes(monkeypatch):
    """A service's lanes are tuned stepping together: the lane count is part of
    the key, so a 4 x 16-case service and a lone 16-case plan keep separate
    configurations."""
    from types import SimpleNamespace
    monkeypatch.setattr(autotune, "device_key", lambda device: "gpu|lib")
    plan = SimpleNamespace(device=None, shapes=[(256, 64)] * 16, params=SimpleNamespace(precision=1))
    lone = autotune.plan_key(plan)
    plan.lanes = 4
    assert lone == "gpu|lib|mixed|256x64:16"
    assert autotune.plan_key(plan) == lone + "|lanes4"
