"""The multi-GPU replica path on the CPU: two gloo ranks run the same host
bookkeeping that bench.py and a sharded solve run under NCCL (case shards,
slowest-rank job time, summed counts, results gathered in global case order).
Cases exchange no data, so this is the whole multi-rank logic of the path."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from aero2d_b200 import replicas


def test_case_shard_covers_every_case_once():
    for n in (0, 1, 5, 64, 97):
        for world in (1, 2, 3, 8):
            seen = []
            sizes = []
            for r in range(world):
                s = replicas.case_shard(n, r, world)
                seen.extend(range(n)[s])
                sizes.append(s.stop - s.start)
            assert seen == list(range(n))
            assert max(sizes) - min(sizes) <= 1


def test_case_shard_rejects_bad_ranks():
    with pytest.raises(ValueError):
        replicas.case_shard(10, 2, 2)
    with pytest.raises(ValueError):
        replicas.case_shard(10, 0, 0)


def test_single_process_is_identity():
    assert replicas.job_time_and_count(12.5, 3, None) == (12.5, 3.0)
    out = replicas.gather_cases({"cl": np.arange(3.0)}, None)
    assert np.array_equal(out["cl"], np.arange(3.0))
    assert replicas.rank_seed(2412, 0) == 2412


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    try:
        dist = replicas.init("gloo", timeout_s=60.0)
        # each rank "solves" its shard of 7 global cases: cl = 10 * global index
        machs = np.linspace(0.3, 0.75, 7)
        alphas = np.linspace(-4.0, 8.0, 7)
        m, a = replicas.split_inputs([machs, alphas], rank, world)
        s = replicas.case_shard(7, rank, world)
        cl = 10.0 * np.arange(s.start, s.stop, dtype=np.float64)
        steps = np.full(len(m), 100 + rank, dtype=np.int64)
        t, n = replicas.job_time_and_count(100.0 + 50.0 * rank, len(m), dist)
        out = replicas.gather_cases({"cl": cl, "mach": m, "alpha": a, "steps": steps}, dist)
        q.put((rank, t, n, out, replicas.rank_seed(2412, rank)))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, "error", repr(e), None, None))


@pytest.mark.timeout(180)
def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=150) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort(key=lambda g: g[0])
    for rank, t, n, out, seed in got:
        assert t != "error", n
        assert t == 150.0                  # the slowest rank's time
        assert n == 7.0                    # every case counted once
        assert np.array_equal(out["cl"], 10.0 * np.arange(7))
        assert np.allclose(out["mach"], np.linspace(0.3, 0.75, 7))
        assert np.allclose(out["alpha"], np.linspace(-4.0, 8.0, 7))
        assert list(out["steps"]) == [100] * 4 + [101] * 3
    assert got[0][4] != got[1][4]          # distinct synthetic batches per rank
