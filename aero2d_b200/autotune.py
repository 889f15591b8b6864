"""Autotuner of a plan's launch configuration.

Two knobs of a bound plan change how its kernels are launched, never what they
compute (every variant does the same arithmetic in the same order, so results
are bitwise the same; include/aero2d_b200.h, a2d_plan_set_tuning):

  jvp_tile  the tile shape (i x j cells per CTA) of the FP32 Jacobian-vector
            stencil, run gmres_restart + 1 times per Newton step: "32x8",
            "32x16", "64x4" or "16x16" (the halo is recomputed per tile, so
            taller tiles compute less and hold more shared memory);
  sweep     the line sweep's kernel, by warps per half line group: "lanes"
            (one warp, a lane solving all four block rows of its line),
            "pairs" (two warps, two lanes per line with two block rows each)
            or "rows" (four warps, a warp per block row).

The best configuration depends on the grid sizes in a batch, the batch size and
the precision.  `apply(plan, measure=True)` looks the plan's key up in the
cache; on a miss it times a few Newton steps of the plan under every candidate
(CUDA events on the plan's stream), keeps the fastest, stores it and leaves the
plan at the freestream.  The key is the GPU model, the library's version, the
precision and the plan's signature: its grid sizes with the number of cases of
each size rounded up to a power of two.

The cache is one JSON file, $AERO2D_B200_TUNING or
~/.cache/aero2d_b200/tuning.json, written atomically (a temporary file
renamed over it); a missing, unreadable or malformed file is an empty cache.
"""
from __future__ import annotations

import json
import os
import tempfile
from collections import Counter
from pathlib import Path
from typing import Callable, Iterable, Optional

JVP_TILES = ("32x8", "32x16", "64x4", "16x16")
SWEEPS = ("lanes", "rows", "pairs", "halves")
MIXED_ONLY_SWEEPS = ("rows", "halves")   # refused on FP64 plans
DEFAULT = ("32x16", "halves")   # a new plan's configuration (the library's defaults)


def default_path() -> Path:
    env = os.environ.get("AERO2D_B200_TUNING")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "aero2d_b200" / "tuning.json"


def _pow2(n: int) -> int:
    p = 1
    while p < n:
        p *= 2
    return p


def signature(shapes: Iterable[tuple[int, int]], precision: int) -> str:
    """'mixed|128x32:16,256x64:64': grid sizes in order, case counts rounded up
    to powers of two (batches of similar size share a configuration)."""
    cnt = Counter((int(a), int(b)) for a, b in shapes)
    prec = "mixed" if precision else "fp64"
    return prec + "|" + ",".join(f"{ni}x{nc}:{_pow2(n)}" for (ni, nc), n in sorted(cnt.items()))


def candidates(precision: int) -> list[tuple[str, str]]:
    """Every configuration worth timing: the JVP tile shapes matter only in
    the mixed precision (the FP64 JVP always runs 32 x 8 tiles), and the rows
    and halves sweeps run mixed-precision plans only."""
    if precision:
        return [(t, v) for t in JVP_TILES for v in SWEEPS]
    return [(JVP_TILES[0], v) for v in SWEEPS if v not in MIXED_ONLY_SWEEPS]


class TuningCache:
    """The on-disk store of chosen configurations: key -> {"jvp_tile", "sweep", "ms"}."""

    def __init__(self, path: Optional[Path] = None):
        self.path = Path(path) if path is not None else default_path()

    def load(self) -> dict:
        try:
            data = json.loads(self.path.read_text())
        except (OSError, ValueError):
            return {}
        if not isinstance(data, dict):
            return {}
        return {k: v for k, v in data.items()
                if isinstance(v, dict) and v.get("jvp_tile") in JVP_TILES and v.get("sweep") in SWEEPS}

    def get(self, key: str) -> Optional[tuple[str, str]]:
        v = self.load().get(key)
        return (v["jvp_tile"], v["sweep"]) if v else None

    def put(self, key: str, choice: tuple[str, str], timings: Optional[dict] = None) -> None:
        data = self.load()
        entry = {"jvp_tile": choice[0], "sweep": choice[1]}
        if timings:
            entry["ms"] = {f"{t}/{v}": round(float(ms), 4) for (t, v), ms in timings.items()}
        data[key] = entry
        self.path.parent.mkdir(parents=True, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=str(self.path.parent), prefix=".tuning", suffix=".json")
        try:
            with os.fdopen(fd, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except BaseException:
            try:
                os.unlink(tmp)
            except OSError:
                pass
            raise


def choose(timings: dict) -> tuple[str, str]:
    """The fastest configuration; ties keep the earlier candidate."""
    best, best_ms = None, float("inf")
    for cand, ms in timings.items():
        if ms < best_ms:
            best, best_ms = cand, ms
    if best is None:
        raise ValueError("no timings")
    return best


def device_key(device) -> str:
    import torch
    from . import _lib
    name = torch.cuda.get_device_name(device)
    return f"{name}|lib{_lib.load().a2d_version()}"


def plan_key(plan) -> str:
    """The cache key of a plan (a service's lanes: the first lane's cases and the
    lane count, since the lanes are timed stepping together)."""
    lanes = int(getattr(plan, "lanes", 1))
    return (device_key(plan.device) + "|" + signature(plan.shapes, plan.params.precision) +
            (f"|lanes{lanes}" if lanes > 1 else ""))


def time_newton_steps(plan, steps: int = 2) -> float:
    """Mean milliseconds per Newton step of the plan from the freestream, after
    one untimed step (graph capture); CUDA events on the plan's stream."""
    import torch
    plan.init_freestream()
    plan.newton_step()
    with torch.cuda.device(plan.device):
        s = torch.cuda.current_stream(plan.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            plan.newton_step()
        e1.record(s)
        e1.synchronize()
    return e0.elapsed_time(e1) / steps


def tune(plan, measure: Callable = time_newton_steps, cands: Optional[list] = None) -> tuple[tuple[str, str], dict]:
    """Times every candidate configuration on the plan; leaves the fastest set
    and the plan's state at the freestream.  Returns (choice, timings)."""
    cands = cands if cands is not None else candidates(plan.params.precision)
    timings = {}
    for t, v in cands:
        plan.set_tuning(t, v)
        timings[(t, v)] = float(measure(plan))
    best = choose(timings)
    plan.set_tuning(*best)
    plan.init_freestream()
    return best, timings


def apply(plan, measure: bool = False, cache: Optional[TuningCache] = None,
          measure_fn: Callable = time_newton_steps) -> tuple[str, str]:
    """Sets the plan's cached configuration; with `measure`, tunes and stores
    it on a cache miss.  Returns the configuration in use."""
    cache = cache if cache is not None else TuningCache()
    key = plan_key(plan)
    choice = cache.get(key)
    if choice is not None:
        plan.set_tuning(*choice)
        return choice
    if not measure:
        return plan.tuning()
    choice, timings = tune(plan, measure_fn)
    cache.put(key, choice, timings)
    return choice
