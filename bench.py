#!/usr/bin/env python
"""Benchmark of the batched Euler Newton-Krylov path on B200.

Headline workload: Euler cases on one shared 256 x 64 O-grid of NACA 2412
(ogrid(naca4("2412", 129), nj=65, ds0=2e-3, radius=20)), M ~ U[0.30, 0.75] and
alpha ~ U[-4, 8] deg from default_rng(2412) (64 cases), pseudo-transient
Newton-Krylov (GMRES restart 30, 4 line-Jacobi sweeps, reference defaults
otherwise) from the freestream to a residual drop of 1e-10 (at most 200 Newton
steps), mixed precision.  One "step" is those 64 cases.  The K timed steps are
served as one stream: all K x 64 cases are queued at once into the
continuous-batching service with 64 slots, which admits a queued case as soon
as a slot's case retires, so the batch stays full until the queue empties.
Inputs are synthetic (seeded), like the reference's own benchmark inputs.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line.  `value` is converged cases per second of that stream
with the grid resident in HBM (CUDA events); `e2e` is the same stream through
the public service API from a host grid and host arrays, results back to the
host, on the wall clock.  Beside it: the same 64 cases as one batch from t = 0
(the batch drains to its slowest case), the plain FP64 batch and per-case
paths, accuracy against the FP64 oracle's converged solutions
(tests/golden/oracle_configs.json), the roofline of the dominant kernel, and
the other configurations: the single FP64 case (192 x 48 NACA 0012), 128
transonic airfoils on 384 x 96 grids, the 512-case ragged batch, and served
polar requests.  Under torchrun every rank streams its own cases (seed 2412 +
rank, weak scaling, no collective on the data path) and only the headline
runs.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from aero2d_b200 import replicas  # noqa: E402  (host-only module: no torch or CUDA import)

METRIC = "converged Euler cases/sec + p50/p99 latency, mixed vs plain FP64 on 1 B200 at |ΔCl|≤1e-4"
GRID = dict(code="2412", n_side=129, nj=65, ds0=2e-3, radius=20.0)
CASES = 64
MACH = (0.30, 0.75)
ALPHA = (-4.0, 8.0)
SEED = 2412
TOL = 1e-10
RESTART = 30
MAX_ITER = 200
FIXTURES = ROOT / "tests" / "golden" / "oracle_configs.json"


def draw_cases(seed: int, n: int):
    rng = np.random.default_rng(seed)
    machs = rng.uniform(MACH[0], MACH[1], n)
    alphas = rng.uniform(ALPHA[0], ALPHA[1], n)
    return machs, alphas


def make_grid():
    from aero2d_b200.geometry import naca4
    from aero2d_b200.grid import ogrid
    return ogrid(naca4(GRID["code"], GRID["n_side"]), nj=GRID["nj"], ds0=GRID["ds0"], radius=GRID["radius"])


def workload_config(cases: int, tol: float, max_iter: int, restart: int) -> dict:
    """The `config` of both arms: the workload only (precision and parallelism
    are reported beside it), so the two lines carry the same config."""
    return {"workload": f"{cases} cases on one 256x64 O-grid of NACA 2412, M~U[0.30,0.75], alpha~U[-4,8] deg, "
                        f"seed {SEED}(+rank), Newton-Krylov from the freestream to residual drop {tol:g}",
            "cases_per_gpu": cases, "grid": "256x64 (ogrid naca4('2412',129), nj=65, ds0=2e-3, radius=20)",
            "gmres_restart": restart, "jacobi_sweeps": 4, "max_newton_steps": max_iter, "tol": tol,
            "l2": "working set ~2 GB per 64 cases, larger than the 126 MB L2 (no flush needed)"}


def oracle_fixtures() -> dict:
    if not FIXTURES.exists():
        return {}
    return json.load(open(FIXTURES)).get("cases", {})


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 oracle (NumPy restatement of aero2d/euler.py and
# aero2d/implicit.py), one process per case stepping along the case's own
# Newton trajectory from the freestream
# ---------------------------------------------------------------------------
def _oracle_worker(case: int, seed: int, conn):
    """Holds one case of the workload and takes one Newton step (with the
    solve loop's SER CFL update, aero2d/implicit.py:216-244) per request."""
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, str(ROOT))
    from oracle.euler_oracle import EulerModel
    from oracle.implicit_oracle import ImplicitModel
    g = make_grid()
    machs, alphas = draw_cases(seed, CASES)
    im = ImplicitModel(EulerModel(g.x, g.y), gmres_restart=RESTART)
    w = im.b.freestream(machs[case], alphas[case])
    U = im.b.init_state(w)
    cfl, r0 = im.cfl0, None
    conn.send("ready")
    while conn.recv() == "step":
        t = time.perf_counter()
        Un, rn, om, _ = im.step(U, w, cfl)
        dt = time.perf_counter() - t
        if np.isfinite(rn) and np.all(np.isfinite(Un)):
            U = Un
            r0 = rn if r0 is None else r0
            cfl = float(np.clip(im.cfl0 * r0 / max(rn, 1e-30), im.cfl0, im.cfl_max))
            if om < 1.0:
                cfl = max(cfl * 0.5, 1.0)
        else:
            cfl = 1.0
        conn.send(dt)
    conn.close()


class OracleBaseline:
    """`procs` spawned processes, each holding one case of the workload; a
    sample is one further Newton step of every case (steps 1, 2, ... of the
    real trajectories).  Converged cases/s = processes / mean step time /
    Newton steps per case x converged fraction, the last two from the oracle's
    own converged runs of this workload (tests/golden/oracle_configs.json)."""

    def __init__(self, procs: int, seed: int = SEED):
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        self.conns, self.procs = [], []
        # one BLAS thread per process: the children inherit the environment and
        # read it when they import numpy, before the worker function runs
        threads = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")
        saved = {v: os.environ.get(v) for v in threads}
        os.environ.update({v: "1" for v in threads})
        try:
            for k in range(procs):
                a, b = ctx.Pipe()
                p = ctx.Process(target=_oracle_worker, args=(k % CASES, seed, b), daemon=True)
                p.start()
                self.conns.append(a)
                self.procs.append(p)
        finally:
            for v, old in saved.items():
                if old is None:
                    os.environ.pop(v, None)
                else:
                    os.environ[v] = old
        for c in self.conns:
            c.recv()
        fx = [v for k, v in oracle_fixtures().items() if k.startswith("c2_")]
        if not fx:
            raise RuntimeError("tests/golden/oracle_configs.json has no c2 cases")
        self.steps_per_case = float(np.mean([v["newton_steps"] for v in fx]))
        self.converged_frac = float(np.mean([v["log10_drop"] <= np.log10(v["tol"]) for v in fx]))
        self.n_fixture = len(fx)
        self.steps_done = 0

    def sample(self):
        for c in self.conns:
            c.send("step")
        times = [c.recv() for c in self.conns]
        self.steps_done += 1
        per_step = float(np.mean(times))
        rate = len(self.conns) / per_step / self.steps_per_case * self.converged_frac
        return rate, per_step

    def describe(self, per_step: float, first: int, last: int) -> str:
        return (f"Newton steps {first}..{last} of the first {len(self.conns)} cases of this workload "
                f"(one spawned process per case, one BLAS thread each), {per_step:.2f} s per step; "
                f"x {self.steps_per_case:.1f} Newton steps per case and {self.converged_frac:.3f} converged "
                f"fraction from the FP64 oracle's own runs of {self.n_fixture} cases of this workload")

    def close(self):
        for c in self.conns:
            try:
                c.send("stop")
            except Exception:
                pass
        for p in self.procs:
            p.join(timeout=10)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = [ln.split(",") for ln in open(self.file.name).read().splitlines() if ln.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        if not sm:
            return None
        busy = [v for v in sm if v > 0.5 * (smax or max(sm))] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def pct(a, qs=(50, 95, 99), nd=3):
    a = np.asarray(a, float)
    if a.size == 0:
        return None
    return {f"p{q}": round(float(np.percentile(a, q)), nd) for q in qs}


# ---------------------------------------------------------------------------
# the GPU arm: streamed cases through the service, and the batch from t = 0
# ---------------------------------------------------------------------------
def stream_solve(svc, machs, alphas, slots: int):
    """Queues every case (one single-point request each) at once and steps the
    service until all are done; CUDA events after every Newton step.  Returns
    (elapsed ms, per-case results in submission order, per-case service time
    ms from admission to retirement, Newton steps taken, kernel launches)."""
    import torch
    ids = [svc.submit(float(m), [float(a)], continuation=False) for m, a in zip(machs, alphas)]
    pos = {rid: q for q, rid in enumerate(ids)}
    n = len(ids)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    evs, end_step, finished = [], {}, 0
    admit_step = np.zeros(n, int)
    admitted = 0
    while finished < n:
        # requests are admitted in queue order into the slots freed so far
        free_before = slots + finished
        while admitted < n and admitted < free_before:
            admit_step[admitted] = len(evs)
            admitted += 1
        busy = svc.step()
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        evs.append(e)
        for rid in svc.poll():
            end_step[pos[rid]] = len(evs) - 1
            finished += 1
        if busy == 0 and finished < n and svc.pending()[0] == 0:
            raise RuntimeError("service idle with unfinished requests")
    evs[-1].synchronize()
    t = np.array([ev0.elapsed_time(e) for e in evs])
    t_start = np.concatenate([[0.0], t])
    res = [svc.result(rid) for rid in ids]
    svc_ms = np.array([t[end_step[q]] - t_start[admit_step[q]] for q in range(n)])
    return float(t[-1]), res, svc_ms, len(evs)


def batch_solve(plan, max_iter):
    """One batch solve from the freestream; CUDA events after every Newton step.
    Returns (elapsed_ms, per-case latency ms, nsteps, converged, frozen, steps)."""
    import torch
    ev0 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    plan.init_freestream()
    evs = []
    for _ in range(max_iter):
        plan.newton_step()
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        evs.append(e)
        if plan.live_count() == 0:
            break
    evs[-1].synchronize()
    t_steps = np.array([ev0.elapsed_time(e) for e in evs])
    nsteps, done, frozen, lastrn, r0 = plan.status()
    conv = done & ~frozen
    lat = np.array([t_steps[n - 1] if n > 0 else 0.0 for n in nsteps])
    batch_solve.last_step_ms = np.diff(np.concatenate([[0.0], t_steps]))
    batch_solve.last_live = np.array([(nsteps > s).sum() for s in range(len(evs))])
    return float(t_steps[-1]), lat, nsteps, conv, frozen, len(evs)


def step_profile(step_ms, live, B):
    return {f"{lo}-{hi}": round(float(step_ms[(live >= lo) & (live <= hi)].mean()), 3)
            for lo, hi in ((B * 3 // 4 + 1, B), (B // 4 + 1, B * 3 // 4), (2, B // 4), (1, 1))
            if ((live >= lo) & (live <= hi)).any()}


def algorithmic_bytes(kernel: str, cells: int, restart: int, mixed: bool) -> float:
    """Bytes a kernel must move per launch for the whole batch (cells = total
    cells); counts the matrix and vector words of the kernel's definition once."""
    f = 4 if mixed else 8
    h = 2 if mixed else 8   # sweep factors G, C, P, Q (FP16 in the mixed path)
    v = 4 if mixed else 8   # intermediate vectors of the sweeps (FP32 in the mixed path)
    kb = 2 if mixed else 8  # Krylov basis entries (BF16 in the mixed path)
    d = 8
    half = max(1, restart // 2)
    per_cell = {
        # coupled line sweep: e0, x_prev, P, Q, G, C, x (store); the d_j written by
        # the forward recurrence and read back by the backward one is not counted
        "sweep": 4 * v + 4 * v + 4 * 16 * h + 4 * v,
        # first sweep: r, inv, G, C, e0 (store), x (store)
        "sweep_first": 4 * d + 16 * f + 2 * 16 * h + 4 * v + 4 * v,
        # U, V, diag, z, face vectors (2 i-face + 2 j-face components)
        "jvp": 4 * d + 4 * kb + d + 4 * d + 4 * f,
        # Gram-Schmidt pass 1: w, restart/2 basis vectors
        "dots": 4 * d + half * 4 * kb,
        # pass 2: w, restart/2 basis vectors read once (kept on chip for the re-projection)
        "project": 4 * d + half * 4 * kb,
        # pass 3: w, restart/2 basis vectors, the next basis vector written
        "update": 4 * d + half * 4 * kb + 4 * kb,
    }[kernel]
    return float(per_cell) * cells


def launches_per_step(kernel: str, restart: int, sweeps: int = 4) -> int:
    napp = restart + 2
    return {"sweep": (sweeps - 1) * napp, "sweep_first": napp, "jvp": restart + 1,
            "dots": restart, "project": restart, "update": restart}[kernel]


def read_traffic(kernel: str):
    """DRAM bytes per cell of a kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "dram_traffic.txt"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        parts = ln.split()
        if len(parts) >= 2 and parts[0] == kernel and not ln.startswith("#"):
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def cpu_model() -> str:
    """The host CPU's model name (Linux), for the CPU-baseline lines."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def gpu_arm(args, rank: int, world: int, dist):
    import torch
    from aero2d_b200 import _lib
    from aero2d_b200.euler import EulerSolver
    from aero2d_b200.implicit import ImplicitEuler
    from aero2d_b200.plan import DeviceGrid, Plan
    from aero2d_b200.service import EulerService

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    B = args.cases
    seed = replicas.rank_seed(SEED, rank)
    machs, alphas = draw_cases(seed, B)
    grid = make_grid()
    dgrid = DeviceGrid(grid, dev)
    tol_log = np.log10(args.tol)

    def make_plan(dtype, cases_m, cases_a):
        base = EulerSolver(grid, dtype=dtype, device=dev)
        s = ImplicitEuler(base, gmres_restart=args.restart)
        winf = base.freestream(cases_m, cases_a)
        return Plan([base.dgrid] * len(cases_m), winf, s.params(args.tol, args.max_iter), dev, tuning="auto"), base

    def make_service(g, dtype=np.float32):
        return EulerService(g, slots=B, dtype=dtype, device=dev, tol=args.tol, max_iter=args.max_iter,
                            gmres_restart=args.restart, tuning="auto", lanes=args.lanes)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- headline: K x 64 cases streamed through the 64-slot service --------
    svc = make_service(dgrid)
    tuning = svc.tuning()
    if args.warmup > 0:
        stream_solve(svc, np.tile(machs, args.warmup), np.tile(alphas, args.warmup), B)
    sm, sa = np.tile(machs, args.steps), np.tile(alphas, args.steps)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    steps_before = svc.stats()[1]
    elapsed_ms, res, svc_ms, nsteps_run = stream_solve(svc, sm, sa, B)
    barrier()
    clk = clocks.stop()
    reached = np.array([r["drop"][0] < args.tol for r in res])
    converged = int(reached.sum())
    kps, steps_after = svc.stats()
    # per Newton step: the graph's kernels and the service's status/forces/restart kernels
    launches = (steps_after - steps_before) * (kps + 3 * svc.lanes)
    elapsed_ms, converged_all = replicas.job_time_and_count(elapsed_ms, converged, dist, dev)
    converged_all = int(converged_all)
    value = converged_all / (elapsed_ms / 1e3)
    coef_mix = np.array([[r["cl"][0], r["cd"][0], r["cm"][0]] for r in res[:B]])
    conv_mix = reached[:B]
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "cases/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(elapsed_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64",
        "data": "synthetic (seeded NACA 2412 cases; random (M, alpha) per case)",
        "config": workload_config(B, args.tol, args.max_iter, args.restart),
        "precision": "mixed: FP64 residual/factorisation/Gram-Schmidt/update; FP32 JVP, face Jacobians, sweep "
                     "arithmetic; FP16 sweep factors; BF16 Krylov basis",
        "parallelism": f"replicas x{world}, case sharding",
        "mode": f"served stream: the {args.steps} steps' {args.steps * B} cases queued at once into a {B}-slot "
                f"continuous-batching service ({svc.lanes} lanes of {B // svc.lanes} slots, each lane's plan stepped "
                "on its own stream, concurrently; a case is admitted as soon as a slot retires; the batch drains "
                "once, at the end of the stream)",
        "tuning": {"jvp_tile": tuning[0], "sweep": tuning[1],
                   "note": "chosen by aero2d_b200.autotune on this GPU (timed Newton steps of every configuration)"},
        "converged_cases": converged_all,
        "cases_total": B * args.steps * world,
        "newton_steps_mean": round(float(np.mean([r["nsteps"][0] for r in res])), 2),
        "service_steps": int(nsteps_run),
        "ms_per_service_step": round(elapsed_ms / max(1, nsteps_run), 3),
        "latency_ms": dict(pct(svc_ms[reached], nd=2) or {},
                           note="per converged case, from its admission into a slot to its retirement"),
    }
    svc.close()
    del svc
    if rank != 0 or world > 1:
        return out if rank == 0 else None

    # ---- the same 64 cases as one batch from t = 0 (drains) -----------------
    plan, base = make_plan(np.float32, machs, alphas)
    batch_solve(plan, args.max_iter)
    rb = batch_solve(plan, args.max_iter)
    out["batch_from_t0"] = {
        "value": round(int(rb[3].sum()) / (rb[0] / 1e3), 3), "unit": "cases/s", "ms_per_batch": round(rb[0], 1),
        "ms_per_newton_step_by_live_cases": step_profile(batch_solve.last_step_ms, batch_solve.last_live, B),
        "latency_ms": pct(rb[1][rb[3]], nd=2),
        "note": f"the {B} cases started together and stepped until the slowest retires"}

    # ---- plain FP64 batch and the per-case FP64 path -----------------------
    plan64, _ = make_plan(np.float64, machs, alphas)
    batch_solve(plan64, args.max_iter)
    r64 = batch_solve(plan64, args.max_iter)
    coef64 = plan64.forces()[0].cpu().numpy()
    conv64 = r64[3]
    out["fp64_batched"] = {"value": round(int(conv64.sum()) / (r64[0] / 1e3), 3), "unit": "cases/s",
                           "ms_per_batch": round(r64[0], 1), "newton_steps_mean": round(float(r64[2].mean()), 2)}
    del plan64
    t_single, n_single, lat_single = 0.0, 0, []
    for k in range(args.single_sample):
        pk, _ = make_plan(np.float64, machs[k:k + 1], alphas[k:k + 1])
        batch_solve(pk, 2)
        r1 = batch_solve(pk, args.max_iter)
        t_single += r1[0]
        n_single += int(r1[3].sum())
        lat_single.append(r1[0])
        del pk
    per_case_rate = n_single / (t_single / 1e3) if n_single else 0.0
    out["fp64_per_case"] = {"value": round(per_case_rate, 3), "unit": "cases/s",
                            "sample": f"cases 0..{args.single_sample - 1} solved one at a time (B=1 plans)",
                            "latency_ms": pct(lat_single, nd=1),
                            "ratio_mixed_served_over_this": round(value / per_case_rate, 2) if per_case_rate else None}

    # ---- accuracy: against the FP64 oracle's converged solutions -----------
    fx = oracle_fixtures()
    ocases = [(k, fx.get(f"c2_{k}")) for k in range(B) if fx.get(f"c2_{k}") is not None and seed == SEED]
    d_or, n_or = [], 0
    for k, c in ocases:
        if c["log10_drop"] <= tol_log and conv_mix[k]:
            d_or.append(np.abs(coef_mix[k] - [c["cl"], c["cd"], c["cm"]]))
            n_or += 1
    d_or = np.array(d_or) if d_or else np.full((1, 3), np.nan)
    both = conv_mix & conv64
    dd = np.abs(coef_mix - coef64)[both]
    out["accuracy"] = {
        "vs_fp64_oracle": {"max_abs_dCl": float(d_or[:, 0].max()), "max_abs_dCd": float(d_or[:, 1].max()),
                           "max_abs_dCm": float(d_or[:, 2].max()), "cases_compared": n_or,
                           "reference": "tests/golden/oracle_configs.json c2_0..c2_7 (FP64 oracle, same grid and "
                                        "cases, converged to 1e-10)"},
        "vs_fp64_gpu": {"max_abs_dCl": float(dd[:, 0].max()) if both.any() else None,
                        "max_abs_dCd": float(dd[:, 1].max()) if both.any() else None,
                        "max_abs_dCm": float(dd[:, 2].max()) if both.any() else None,
                        "cases_compared": int(both.sum())},
        "gate": "|dCl| <= 1e-4 and |dCd| <= 2e-6"}

    # ---- roofline of the dominant kernel (CUDA events on the plan's stream) --
    cells = B * 256 * 64
    kernels = {"sweep": _lib.K_SWEEP, "sweep_first": _lib.K_SWEEP_FIRST, "jvp": _lib.K_JVP, "dots": _lib.K_DOTS,
               "project": _lib.K_PROJECT, "update": _lib.K_UPDATE}
    ktimes = {k: plan.time_kernel(v, reps=20) for k, v in kernels.items()}
    share = {k: ktimes[k] * launches_per_step(k, args.restart) for k in kernels}
    dom = max(share, key=share.get)
    peak, peak_kind = measured_peak()
    achieved = algorithmic_bytes(dom, cells, args.restart, True) / (ktimes[dom] / 1e3) / 1e9
    traffic_per_cell = read_traffic(dom)
    out["roofline"] = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                       "unit": "GB/s", "frac": round(achieved / peak, 3), "peak_source": peak_kind,
                       "traffic": (round(traffic_per_cell * cells) if traffic_per_cell else None),
                       "algorithmic_bytes_per_launch": algorithmic_bytes(dom, cells, args.restart, True),
                       "ms_per_launch": round(ktimes[dom], 4)}
    out["kernels_ms_per_launch"] = {k: round(v, 4) for k, v in ktimes.items()}
    out["kernels_ms_per_newton_step"] = {k: round(v, 3) for k, v in share.items()}
    del plan

    # ---- end to end through the public service API ---------------------------
    torch.cuda.synchronize()
    t = time.perf_counter()
    svc_e = EulerService(grid, slots=B, dtype=np.float32, device=dev, tol=args.tol, max_iter=args.max_iter,
                         gmres_restart=args.restart, lanes=args.lanes)
    ids = [svc_e.submit(float(m), [float(a)], continuation=False) for m, a in zip(sm, sa)]
    svc_e.run()
    res_e = [svc_e.result(rid) for rid in ids]
    te = time.perf_counter() - t
    conv_e2e = int(sum(r["drop"][0] < args.tol for r in res_e))
    ni, nj = grid.shape
    h2d = (2 * ni * nj * 8 + len(ids) * (4 * 8 + 4 * 2)) / args.steps
    d2h = sum(sum(v.nbytes for v in r.values() if isinstance(v, np.ndarray)) for r in res_e) / args.steps
    out["e2e"] = {"value": round(conv_e2e / te, 3), "unit": "cases/s", "h2d_bytes_per_step": int(h2d),
                  "d2h_bytes_per_step": int(d2h), "seconds": round(te, 3), "converged_cases": conv_e2e,
                  "call": "EulerService(host OGrid, slots=64, dtype=float32, tol=1e-10).submit(M, [alpha]) for every "
                          "case, .run(), .result(id) -> numpy (service creation, grid upload and graph capture "
                          "inside the timed region)"}
    svc_e.close()
    del svc_e
    out["gpu_launches"] = int(launches)
    out["clocks"] = clk

    # ---- the other configurations -----------------------------------------------
    if "c1" in args.sections:
        out["c1_single_fp64"] = c1_arm(args, dev, fx)
    if "c3" in args.sections:
        out["c3_transonic"] = c3_arm(args, dev, fx)
    if "c4" in args.sections:
        out["c4_ragged"] = c4_arm(args, dev)
    if "served" in args.sections and args.served_window > 0:
        out["c5_served"] = served_arm(args, dev)

    # ---- CPU baseline ---------------------------------------------------------
    if not args.no_cpu_baseline:
        procs = max(1, min(os.cpu_count() or 1, args.cpu_procs))
        ob = OracleBaseline(procs)
        t0 = time.perf_counter()
        samples = [ob.sample() for _ in range(args.cpu_samples)]
        cpu_wall = time.perf_counter() - t0
        ob.close()
        per_step = float(np.mean([s[1] for s in samples]))
        rate = float(np.mean([s[0] for s in samples]))
        out["cpu_baseline"] = {"value": round(rate, 5), "unit": "cases/s", "cores": procs, "kind": "port",
                               "cpu": f"{cpu_model()}, {os.cpu_count()} logical CPUs",
                               "sample": ob.describe(per_step, 1, args.cpu_samples), "wall_s": round(cpu_wall, 1)}
    return out


# ---------------------------------------------------------------------------
# the other configurations of the path
# ---------------------------------------------------------------------------
def c1_arm(args, dev, fx):
    """Single case, plain FP64: NACA 0012, ogrid(naca4("0012", 97), nj=49,
    ds0=2e-3, radius=20) (192 x 48), M 0.5, alpha 1.25 deg, restart 30, to a
    1e-10 drop; time to converge and Cl/Cd/Cm against the FP64 oracle."""
    from aero2d_b200.euler import EulerSolver
    from aero2d_b200.geometry import naca4
    from aero2d_b200.grid import ogrid
    from aero2d_b200.implicit import ImplicitEuler
    from aero2d_b200.plan import Plan
    g = ogrid(naca4("0012", 97), nj=49, ds0=2e-3, radius=20.0)
    base = EulerSolver(g, dtype=np.float64, device=dev)
    s = ImplicitEuler(base, gmres_restart=args.restart)
    pl = Plan([base.dgrid], base.freestream([0.5], [1.25]), s.params(1e-10, 200), dev)
    batch_solve(pl, 200)
    runs = [batch_solve(pl, 200) for _ in range(3)]
    coef = pl.forces()[0].cpu().numpy()[0]
    o = fx.get("c1")
    out = {"workload": "NACA 0012 192x48 (ogrid naca4('0012',97), nj=49, ds0=2e-3, radius=20; growth ratio 1.167 "
                       "so the far field is at 20 chords), M 0.5, alpha 1.25 deg, FP64, restart 30, drop 1e-10",
           "seconds_to_converge": pct([r[0] / 1e3 for r in runs]), "newton_steps": int(runs[-1][2][0]),
           "converged": bool(runs[-1][3][0]), "cl": float(coef[0]), "cd": float(coef[1]), "cm": float(coef[2])}
    if o is not None:
        out["vs_fp64_oracle"] = {"abs_dCl": float(abs(coef[0] - o["cl"])), "abs_dCd": float(abs(coef[1] - o["cd"])),
                                 "abs_dCm": float(abs(coef[2] - o["cm"])), "oracle_newton_steps": o["newton_steps"]}
    pl.close()
    return out


def c3_arm(args, dev, fx):
    """128 transonic random NACA 4-digit airfoils, each on its own 384 x 96
    O-grid (ds0 1e-3, radius 20, generated on the device), M ~ U[0.70, 0.80],
    alpha ~ U[0, 3] deg, mixed precision, restart 30, drop 1e-10, at most 300
    Newton steps, one ragged batch.  The first 8 cases are the oracle's
    transonic fixtures (tests/golden/oracle_configs.json c3_*), the other 120
    a second seeded draw of the same distribution."""
    import torch
    from aero2d_b200.core import shock_position
    from aero2d_b200.euler import EulerSolver, compute_metrics
    from aero2d_b200.geometry import naca4_params
    from aero2d_b200.grid import GridError
    from aero2d_b200.gridgen import ogrid_batch
    from aero2d_b200.implicit import ImplicitEuler
    from aero2d_b200.plan import Plan
    from tests.helpers import transonic_draw
    p8, grids8, m8, a8, _ = transonic_draw(8, 2025)
    rng = np.random.default_rng(2026)
    params, machs, alphas, rejected = list(p8), list(m8), list(a8), 0
    while len(params) < args.c3_cases:
        m, p, t = rng.uniform(0, 0.06), rng.uniform(0.2, 0.6), rng.uniform(0.08, 0.16)
        mach, al = rng.uniform(0.70, 0.80), rng.uniform(0.0, 3.0)
        try:
            ogrid_batch([naca4_params(m, p, t, 193)], nj=97, ds0=1e-3, radius=20.0, device=dev)
        except GridError:
            rejected += 1
            continue
        params.append((m, p, t))
        machs.append(mach)
        alphas.append(al)
    dgrids = ogrid_batch([naca4_params(m, p, t, 193) for m, p, t in params], nj=97, ds0=1e-3, radius=20.0,
                         device=dev)
    base = EulerSolver(grids8[0], dtype=np.float32, device=dev)
    s = ImplicitEuler(base, gmres_restart=args.restart)
    winf = base.freestream(np.array(machs), np.array(alphas))
    pl = Plan(dgrids, winf, s.params(1e-10, 300), dev, tuning="auto")
    torch.cuda.synchronize()
    t_ms, lat, nsteps, conv, frozen, nst = batch_solve(pl, 300)
    coef, cps = pl.forces()
    coef = coef.cpu().numpy()
    sat = pl.factor_saturations()
    pl.close()
    acc = []
    for k in range(8):
        o = fx.get(f"c3_{k}")
        if o is None or not (o["log10_drop"] <= -8 and conv[k]):
            continue
        m = compute_metrics(grids8[k])
        xs = shock_position(m.xw, m.yw, cps[k].cpu().numpy(), machs[k])
        acc.append([abs(coef[k, 0] - o["cl"]), abs(coef[k, 1] - o["cd"]), abs(coef[k, 2] - o["cm"]),
                    abs(xs - o["shock_x"]) if not (np.isnan(xs) or np.isnan(o["shock_x"])) else np.nan])
    acc = np.array(acc) if acc else np.full((1, 4), np.nan)
    return {"workload": f"{len(params)} random NACA 4-digit airfoils (m~U[0,0.06], p~U[0.2,0.6], t~U[0.08,0.16]) on "
                        "their own 384x96 O-grids (ds0 1e-3, growth 1.08, radius 20, built on the device), "
                        "M~U[0.70,0.80], alpha~U[0,3] deg, mixed precision, drop 1e-10, at most 300 Newton steps",
            "value": round(int(conv.sum()) / (t_ms / 1e3), 3), "unit": "cases/s", "seconds": round(t_ms / 1e3, 2),
            "converged_cases": int(conv.sum()), "frozen": int(frozen.sum()), "airfoils_redrawn": rejected,
            "latency_s": pct(lat[conv] / 1e3), "fp16_factor_saturations": sat,
            "vs_fp64_oracle": {"max_abs_dCl": float(np.nanmax(acc[:, 0])), "max_abs_dCd": float(np.nanmax(acc[:, 1])),
                               "max_abs_dCm": float(np.nanmax(acc[:, 2])),
                               "max_shock_shift_chord": (float(np.nanmax(acc[:, 3]))
                                                         if np.isfinite(acc[:, 3]).any() else None),
                               "cases_compared": int(np.isfinite(acc[:, 0]).sum()),
                               "reference": "the oracle's c3_* cases that fell 8 orders"}}


def c4_arm(args, dev):
    """512 cases with grid sizes drawn uniformly from {128x32, 192x48, 256x64,
    384x96} (ds0 2e-3, 1e-3 for 384x96, radius 20, grids built on the device),
    random NACA 4-digit geometry, M ~ U[0.3, 0.8], alpha ~ U[-4, 10] deg, mixed
    precision, drop 1e-10, at most 200 Newton steps: one ragged batch whose
    every kernel launch covers all cases (one CUDA graph per Newton step),
    against the same cases stepped with one plan (one launch per kernel) per
    case, measured on a sample."""
    import torch
    from aero2d_b200.euler import EulerSolver
    from aero2d_b200.geometry import naca4_params
    from aero2d_b200.grid import GridError
    from aero2d_b200.gridgen import ogrid_batch
    from aero2d_b200.implicit import ImplicitEuler
    from aero2d_b200.plan import Plan
    sizes = [(65, 33, 2e-3), (97, 49, 2e-3), (129, 65, 2e-3), (193, 97, 1e-3)]
    rng = np.random.default_rng(SEED + 4)
    cases, rejected = [], 0
    while len(cases) < args.c4_cases:
        m, p, t = rng.uniform(0, 0.06), rng.uniform(0.2, 0.6), rng.uniform(0.08, 0.16)
        size = int(rng.integers(len(sizes)))
        mach, al = rng.uniform(0.3, 0.8), rng.uniform(-4.0, 10.0)
        ns, nj, ds0 = sizes[size]
        try:
            (g,) = ogrid_batch([naca4_params(m, p, t, ns)], nj=nj, ds0=ds0, radius=20.0, device=dev)
        except GridError:
            rejected += 1
            continue
        cases.append((g, mach, al))
    from aero2d_b200.geometry import naca4
    from aero2d_b200.grid import ogrid
    base = EulerSolver(ogrid(naca4("0012", 65), nj=33, ds0=2e-3, radius=20.0), dtype=np.float32, device=dev)
    s = ImplicitEuler(base, gmres_restart=args.restart)
    machs = np.array([c[1] for c in cases])
    alphas = np.array([c[2] for c in cases])
    params = s.params(1e-10, 200)
    pl = Plan([c[0] for c in cases], base.freestream(machs, alphas), params, dev, tuning="auto")
    tuning = pl.tuning()
    cells = sum(c[0].ni * c[0].nc for c in cases)
    batch_solve(pl, 3)   # graph capture and first launches
    t_ms, lat, nsteps, conv, frozen, nst = batch_solve(pl, 200)
    step_ms, live = batch_solve.last_step_ms, batch_solve.last_live
    full = step_ms[live == len(cases)]
    kps, _ = pl.stats()
    pl.close()
    del pl
    # one plan per case: Newton steps of a sample, cases taken in order
    n_s = min(args.c4_sample, len(cases))
    per_case_ms, sample_cells = 0.0, 0
    for c, m, a in cases[:n_s]:
        p1 = Plan([c], base.freestream([m], [a]), params, dev)
        p1.init_freestream()
        p1.newton_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.c4_steps):
            p1.newton_step()
        e1.record()
        e1.synchronize()
        per_case_ms += e0.elapsed_time(e1) / args.c4_steps
        sample_cells += c.ni * c.nc
        p1.close()
    batch_case_steps = len(cases) / (float(full[:args.c4_steps].mean()) / 1e3) if full.size else None
    single_case_steps = n_s / (per_case_ms / 1e3)
    return {"workload": f"{len(cases)} cases, grid sizes uniform over 128x32/192x48/256x64/384x96 (device-built), "
                        "random NACA 4-digit sections, M~U[0.3,0.8], alpha~U[-4,10] deg, mixed precision, drop 1e-10, "
                        "at most 200 Newton steps, one ragged batch",
            "value": round(int(conv.sum()) / (t_ms / 1e3), 3), "unit": "cases/s", "seconds": round(t_ms / 1e3, 2),
            "converged_cases": int(conv.sum()), "frozen": int(frozen.sum()), "airfoils_redrawn": rejected,
            "cells": int(cells), "kernel_launches_per_newton_step": kps,
            "tuning": {"jvp_tile": tuning[0], "sweep": tuning[1]},
            "ms_per_newton_step_all_live": round(float(full.mean()), 2) if full.size else None,
            "case_steps_per_s": {"one_launch_per_kernel_for_all_cases": round(batch_case_steps, 1)
                                 if batch_case_steps else None,
                                 "one_plan_per_case": round(single_case_steps, 1),
                                 "sample": f"{args.c4_steps} Newton steps of each of the first {n_s} cases "
                                           "alone (B=1 plans, one graph per step each)",
                                 "ratio": round(batch_case_steps / single_case_steps, 2) if batch_case_steps else None},
            "latency_s": pct(lat[conv] / 1e3)}


# served polar requests: the grid sizes of the ragged set (n_side, nj, ds0), radius 20
SERVED_SIZES = [(65, 33, 2e-3), (97, 49, 2e-3), (129, 65, 2e-3), (193, 97, 1e-3)]
SERVED_ALPHAS = np.arange(-4.0, 17.0, 1.0)


def split_chains(alphas, chains: int):
    """An alpha sweep cut into `chains` contiguous pieces, each solved by
    continuation from its own cold first point (in parallel slots)."""
    return [a for a in np.array_split(np.asarray(alphas), chains) if a.size]


def served_arm(args, dev):
    """Served polar requests on one GPU: a seeded Poisson stream at
    `served_rate` requests/s for `served_window` seconds, each request a
    21-point alpha sweep (-4 .. 16 deg) at one random NACA 4-digit airfoil
    (airfoils whose grid folds are redrawn) on one grid size of the ragged set,
    M ~ U[0.2, 0.75], mixed precision, residual drop 1e-8 per point (at most
    `served_max_iter` Newton steps), the sweep cut into `served_chains`
    continuation chains run in parallel slots.  Each request's grid is
    generated on the device when it arrives; slots per grid size come from the
    HBM budget.  Latency = arrival to the last point's result (wall clock: the
    requests arrive in real time)."""
    import torch
    from aero2d_b200.geometry import naca4, naca4_params
    from aero2d_b200.grid import GridError
    from aero2d_b200.gridgen import ogrid_batch
    from aero2d_b200.service import EulerService, slots_for_budget
    rng = np.random.default_rng(SEED + 7)
    n = max(1, int(round(args.served_rate * args.served_window)))
    arrivals = np.cumsum(rng.exponential(1.0 / args.served_rate, n))
    reqs = []
    for _ in range(n):
        m, pp, t = rng.uniform(0, 0.06), rng.uniform(0.2, 0.6), rng.uniform(0.08, 0.16)
        size = int(rng.integers(len(SERVED_SIZES)))
        mach = rng.uniform(0.2, 0.75)
        reqs.append((naca4_params(m, pp, t, SERVED_SIZES[size][0]), size, mach))
    shapes = [(2 * ns - 2, nj - 1) for ns, nj, _ in SERVED_SIZES]
    slots = slots_for_budget(shapes, args.served_hbm_gb * 1e9)
    defaults = [ogrid_batch([naca4("0012", ns)], nj=nj, ds0=ds0, radius=20.0, device=dev)[0]
                for ns, nj, ds0 in SERVED_SIZES]
    svc = EulerService(classes=list(zip(defaults, slots)), dtype=np.float32, device=dev, tol=1e-8,
                       max_iter=args.served_max_iter, gmres_restart=RESTART, tuning="auto", lanes=args.lanes)
    w = svc.submit(0.5, [2.0], grid=defaults[0])
    svc.run()
    svc.result(w)
    chains = split_chains(SERVED_ALPHAS, args.served_chains)
    parts_of, arr_of, grid_of, done_at, left = {}, {}, {}, {}, {}
    part_done = {}
    rejected, steps, nxt, busy_sum, qmax = 0, 0, 0, 0, 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while len(done_at) < n:
        now = time.perf_counter() - t0
        if now > args.served_wall_cap:
            break
        while nxt < n and arrivals[nxt] <= now:
            af, size, mach = reqs[nxt]
            ns, nj, ds0 = SERVED_SIZES[size]
            while True:
                try:
                    (g,) = ogrid_batch([af], nj=nj, ds0=ds0, radius=20.0, device=dev)
                    break
                except GridError:
                    rejected += 1
                    af = naca4_params(rng.uniform(0, 0.06), rng.uniform(0.2, 0.6), rng.uniform(0.08, 0.16), ns)
            ids = [svc.submit(mach, ch, continuation=True, grid=g) for ch in chains]
            for rid in ids:
                parts_of[rid] = nxt
            left[nxt] = len(ids)
            arr_of[nxt], grid_of[nxt] = arrivals[nxt], (g, mach)
            nxt += 1
        busy = svc.step()
        steps += busy > 0
        busy_sum += busy
        qmax = max(qmax, svc.pending()[0])
        for rid in svc.poll():
            q = parts_of[rid]
            part_done[rid] = svc.result(rid)
            left[q] -= 1
            if left[q] == 0:
                done_at[q] = time.perf_counter() - t0
        if busy == 0 and svc.pending()[0] == 0 and nxt < n:
            time.sleep(max(0.0, arrivals[nxt] - (time.perf_counter() - t0)))
    wall = time.perf_counter() - t0
    queued_at_end, running_at_end = svc.pending()
    svc.close()
    by_req: dict = {}
    for rid, r in part_done.items():
        by_req.setdefault(parts_of[rid], []).append((rid, r))
    res = {q: by_req[q] for q in done_at}
    lat = np.array([done_at[q] - arr_of[q] for q in done_at])
    conv = sum(int(r["converged"].sum()) for parts in res.values() for _, r in parts)
    reach = sum(int((r["drop"] < 1e-8).sum()) for parts in res.values() for _, r in parts)
    pts = sum(r["converged"].size for parts in res.values() for _, r in parts)
    span = max(done_at.values()) - float(arrivals[0]) if done_at else float("nan")
    # accuracy: the first two finished requests again in FP64, same grids and chains
    acc_ids = sorted(done_at, key=done_at.get)[:2]
    by_shape: dict = {}
    for q in acc_ids:
        by_shape.setdefault((grid_of[q][0].ni, grid_of[q][0].nc), []).append(q)
    ref = EulerService(classes=[(grid_of[qs[0]][0], len(qs) * len(chains)) for qs in by_shape.values()],
                       dtype=np.float64, device=dev, tol=1e-8, max_iter=args.served_max_iter, gmres_restart=RESTART)
    rid64 = {q: [ref.submit(grid_of[q][1], ch, continuation=True, grid=grid_of[q][0]) for ch in chains]
             for q in acc_ids}
    ref.run()
    dcl, dcd, ncmp = [], [], 0
    for q, r64s in rid64.items():
        mine = [r for _, r in sorted(res[q], key=lambda x: x[0])]
        for a, r64 in zip(mine, r64s):
            b = ref.result(r64)
            both = (a["drop"] < 1e-8) & (b["drop"] < 1e-8)
            ncmp += int(both.sum())
            if both.any():
                dcl.append(np.abs(a["cl"] - b["cl"])[both].max())
                dcd.append(np.abs(a["cd"] - b["cd"])[both].max())
    ref.close()
    return {
        "workload": f"{n} requests, Poisson arrivals at {args.served_rate:g}/s (seeded) for {args.served_window:g} s, "
                    "21-point alpha sweep -4..16 deg each at a random NACA 4-digit airfoil and grid size "
                    "(128x32, 192x48, 256x64, 384x96), M~U[0.2,0.75], mixed precision, drop 1e-8, at most "
                    f"{args.served_max_iter} Newton steps per point, the sweep as {len(chains)} continuation chains "
                    "in parallel slots, grids generated on the device on arrival",
        "slots": dict(zip([f"{a}x{b}" for a, b in shapes], slots)), "lanes": svc.lanes,
        "hbm_budget_gb": args.served_hbm_gb,
        "requests_done": len(done_at), "requests_offered": n, "grid_rejections": rejected,
        "latency_s": pct(lat), "points": pts, "points_reached_1e-8": reach, "converged_points": conv,
        "converged_points_per_s": round(conv / span, 3) if done_at else None,
        "requests_per_s_served": round(len(done_at) / span, 3) if done_at else None,
        "max_queue": qmax, "left_at_cut": {"queued": queued_at_end, "running": running_at_end},
        "mean_busy_slots": round(busy_sum / max(1, steps), 1),
        "newton_steps": steps, "wall_s": round(wall, 2),
        "accuracy_vs_fp64": {"max_abs_dCl": float(max(dcl)) if dcl else None,
                             "max_abs_dCd": float(max(dcd)) if dcd else None, "points_compared": ncmp,
                             "sample": "the first two finished requests re-served in FP64; points that reached "
                                       "the 1e-8 drop in both"},
    }


def reference_arm(args):
    """The reference's CPU path: JAX is not installable in this image, so its
    FP64 NumPy restatement (oracle/) runs on all host cores, one process per
    case along the cases' own Newton trajectories."""
    procs = max(1, os.cpu_count() or 1)
    ob = OracleBaseline(procs)
    for _ in range(max(0, min(args.warmup, 1))):
        ob.sample()
    first = ob.steps_done + 1
    vals, per = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rate, per_step = ob.sample()
        vals.append(rate)
        per.append(per_step)
    wall = time.perf_counter() - t0
    ob.close()
    value = statistics.mean(vals)
    return {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "cases/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * wall / args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded NACA 2412 cases; random (M, alpha) per case)",
            "config": workload_config(CASES, TOL, MAX_ITER, RESTART),
            "precision": "fp64 (the reference's FP64 mode, restated in NumPy)",
            "parallelism": f"{procs} host processes, one case each",
            "cpu_baseline": {"value": round(value, 5), "unit": "cases/s", "cores": procs, "kind": "port",
                             "cpu": f"{cpu_model()}, {os.cpu_count()} logical CPUs",
                             "sample": ob.describe(statistics.mean(per), first, first + args.steps - 1) +
                                       "; the JAX reference cannot be installed in this image (no jax wheel, "
                                       "no network)"},
            "e2e": {"value": round(value, 5), "unit": "cases/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def profile_driver(args):
    """A short run for ncu: the plan of the bench workload (--cases of it),
    `--profile` Newton steps from the freestream."""
    import torch
    from aero2d_b200.euler import EulerSolver
    from aero2d_b200.implicit import ImplicitEuler
    from aero2d_b200.plan import Plan
    dev = torch.device("cuda", 0)
    machs, alphas = draw_cases(SEED, args.cases)
    base = EulerSolver(make_grid(), dtype=np.float64 if args.fp64 else np.float32, device=dev)
    s = ImplicitEuler(base, gmres_restart=args.restart)
    plan = Plan([base.dgrid] * args.cases, base.freestream(machs, alphas), s.params(args.tol, args.max_iter), dev)
    plan.init_freestream()
    for _ in range(args.profile):
        plan.newton_step()
    torch.cuda.synchronize()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--cases", type=int, default=CASES)
    ap.add_argument("--restart", type=int, default=RESTART)
    ap.add_argument("--lanes", type=int, default=None,
                    help="service lanes (plans stepped concurrently; default: the service's, 4 for 64 slots)")
    ap.add_argument("--tol", type=float, default=TOL)
    ap.add_argument("--max-iter", type=int, default=MAX_ITER)
    ap.add_argument("--single-sample", type=int, default=4)
    ap.add_argument("--cpu-procs", type=int, default=16)
    ap.add_argument("--cpu-samples", type=int, default=3, help="Newton steps per CPU process")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sections", default="c1,c3,c4,served",
                    help="comma list of the extra configurations to measure (c1, c3, c4, served)")
    ap.add_argument("--c3-cases", type=int, default=128)
    ap.add_argument("--c4-cases", type=int, default=512)
    ap.add_argument("--c4-sample", type=int, default=16, help="cases stepped one plan at a time")
    ap.add_argument("--c4-steps", type=int, default=10, help="Newton steps timed per sampled case")
    ap.add_argument("--served-rate", type=float, default=50.0, help="request arrivals per second")
    ap.add_argument("--served-window", type=float, default=2.0, help="seconds of arrivals (0 skips)")
    ap.add_argument("--served-chains", type=int, default=3, help="continuation chains per alpha sweep")
    ap.add_argument("--served-hbm-gb", type=float, default=8.0,
                    help="workspace budget of the service (slots beyond those that saturate the GPU only "
                         "add latency)")
    ap.add_argument("--served-max-iter", type=int, default=100, help="Newton steps per point at most")
    ap.add_argument("--served-wall-cap", type=float, default=150.0, help="seconds before the stream is cut")
    ap.add_argument("--profile", type=int, default=0, metavar="STEPS",
                    help="profiling driver: build the mixed plan, run STEPS Newton steps, print nothing")
    ap.add_argument("--fp64", action="store_true", help="with --profile: the all-FP64 plan")
    args = ap.parse_args()
    args.sections = set(s for s in args.sections.split(",") if s)
    if args.profile:
        profile_driver(args)
        return

    rank, world, _ = replicas.env_rank_world()
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(args)))
        return
    dist = replicas.init("nccl", timeout_s=300.0)
    try:
        out = gpu_arm(args, rank, world, dist)
        if rank == 0 and out is not None:
            print(json.dumps(out))
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
