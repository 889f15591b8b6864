"""Replica bookkeeping for solving independent Euler cases on several GPUs.

Cases never exchange data (each O-grid solve is self-contained), so N GPUs run
N independent replicas, one process per GPU launched by torchrun: every rank
solves its own shard of the cases on its own device, and the only collectives
are host-side bookkeeping after the solve -- the slowest rank's time (a job is
done when its last rank is) and the gathering of per-case results in global
case order.  Nothing here touches the device data path.

The functions take the process group module (``torch.distributed``) or None
(one process), so the same code runs single-GPU, under NCCL on GPUs, and under
gloo on the CPU (the multi-rank tests).
"""
from __future__ import annotations

import datetime
import os
from typing import Any, Optional, Sequence

import numpy as np


def env_rank_world() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment (1 process if unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0):
    """Joins the process group of a torchrun launch; returns ``torch.distributed``
    or None for a single process.  The timeout bounds every later collective, so
    ranks that wait for a rank that died end with an error instead of hanging."""
    rank, world, local = env_rank_world()
    if world <= 1:
        return None
    import torch
    import torch.distributed as td
    if backend == "nccl":
        torch.cuda.set_device(local)
    td.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return td


def case_shard(n_total: int, rank: int, world: int) -> slice:
    """Contiguous share of a global case list for one rank: sizes differ by at
    most one, ranks in order, every case in exactly one shard."""
    if n_total < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("need n_total >= 0 and 0 <= rank < world")
    base, extra = divmod(n_total, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's own synthetic batch (weak scaling: distinct cases per rank)."""
    return seed + rank


def _tensor(x, dist, device):
    import torch
    return torch.tensor([float(x)], dtype=torch.float64, device=device)


def job_time_and_count(elapsed_ms: float, count: float, dist, device=None) -> tuple[float, float]:
    """Whole-job time = the slowest rank's time (MAX) and the summed count of
    finished units (SUM) over all ranks; identity for one process."""
    if dist is None:
        return float(elapsed_ms), float(count)
    t = _tensor(elapsed_ms, dist, device)
    c = _tensor(count, dist, device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def gather_cases(local: dict[str, np.ndarray], dist) -> dict[str, np.ndarray]:
    """Concatenates every rank's per-case arrays (leading axis = that rank's
    shard, see case_shard) in rank order, i.e. in global case order, on every
    rank.  Host objects only: one all_gather of pickled arrays per call."""
    if dist is None:
        return {k: np.asarray(v) for k, v in local.items()}
    parts: list[Optional[dict[str, Any]]] = [None] * dist.get_world_size()
    dist.all_gather_object(parts, {k: np.asarray(v) for k, v in local.items()})
    keys = list(local.keys())
    for p in parts:
        if p is None or list(p.keys()) != keys:
            raise RuntimeError("ranks returned different result fields")
    return {k: np.concatenate([p[k] for p in parts], axis=0) for k in keys}


def split_inputs(arrays: Sequence[np.ndarray], rank: int, world: int) -> list[np.ndarray]:
    """A rank's shard of aligned per-case input arrays (e.g. Mach numbers and
    angles of attack)."""
    arrays = [np.asarray(a) for a in arrays]
    n = len(arrays[0])
    if any(len(a) != n for a in arrays):
        raise ValueError("per-case inputs must have the same length")
    s = case_shard(n, rank, world)
    return [a[s] for a in arrays]
