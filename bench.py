#!/usr/bin/env python
"""Benchmark of the batched Euler Newton-Krylov path on B200.

Workload (one "step" = one batch solve): 64 Euler cases on one shared 256 x 64
O-grid of NACA 2412 (ogrid(naca4("2412", 129), nj=65, ds0=2e-3, radius=20)),
M ~ U[0.30, 0.75] and alpha ~ U[-4, 8] deg from default_rng(2412), every case
its own state in one batched plan, pseudo-transient Newton-Krylov (GMRES
restart 30, 4 line-Jacobi sweeps, reference defaults otherwise) from the
freestream to a residual drop of 1e-10 (at most 200 Newton steps).  Inputs are
synthetic (seeded), like the reference's own benchmark inputs.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line.  `value` is converged cases per second of the
mixed-precision batch solve with grid and plan resident in HBM; `e2e` is the
same metric through the public API (ImplicitEuler.solve with host arrays in and
host results out).  Under torchrun every rank solves its own 64-case batch
(seed 2412 + rank, weak scaling, no collective on the data path).
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
# Newton steps per converged case of this workload, FP64, as measured by the
# CUDA path (which follows the oracle step for step); converts the reference
# arm's timed Newton steps into converged cases per second.
NEWTON_STEPS_PER_CASE = 145.5


def draw_cases(seed: int, n: int):
    rng = np.random.default_rng(seed)
    machs = rng.uniform(MACH[0], MACH[1], n)
    alphas = rng.uniform(ALPHA[0], ALPHA[1], n)
    return machs, alphas


def make_grid():
    from aero2d_b200.geometry import naca4
    from aero2d_b200.grid import ogrid
    return ogrid(naca4(GRID["code"], GRID["n_side"]), nj=GRID["nj"], ds0=GRID["ds0"], radius=GRID["radius"])


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 oracle (NumPy restatement of aero2d/euler.py and
# aero2d/implicit.py), one Newton step per process
# ---------------------------------------------------------------------------
def _oracle_newton_step(args):
    k, seed = args
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, str(ROOT))
    from oracle.euler_oracle import EulerModel
    from oracle.implicit_oracle import ImplicitModel
    g = make_grid()
    machs, alphas = draw_cases(seed, CASES)
    im = ImplicitModel(EulerModel(g.x, g.y), gmres_restart=RESTART)
    w = im.b.freestream(machs[k], alphas[k])
    U = im.b.init_state(w)
    t = time.perf_counter()
    im.step(U, w, im.cfl0)
    return time.perf_counter() - t


def cpu_oracle_rate(procs: int, seed: int = SEED):
    """Converged cases/s of the oracle on `procs` host processes, from one
    timed Newton step per process (BLAS threads 1 per process)."""
    import multiprocessing as mp
    os.environ["OMP_NUM_THREADS"] = "1"
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        t0 = time.perf_counter()
        step_times = pool.map(_oracle_newton_step, [(k % CASES, seed) for k in range(procs)])
        wall = time.perf_counter() - t0
    per_step = statistics.mean(step_times)
    rate = procs / per_step / NEWTON_STEPS_PER_CASE
    return rate, per_step, wall


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


# ---------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------
def batch_solve(plan, max_iter):
    """One batch solve from the freestream; CUDA events after every Newton step.
    Returns (elapsed_ms, per-case latency ms, nsteps, converged, frozen)."""
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
    from aero2d_b200.plan import Plan

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    B = args.cases
    seed = replicas.rank_seed(SEED, rank)
    machs, alphas = draw_cases(seed, B)
    grid = make_grid()

    def make_plan(dtype, cases_m, cases_a):
        base = EulerSolver(grid, dtype=dtype, device=dev)
        s = ImplicitEuler(base, gmres_restart=args.restart)
        winf = base.freestream(cases_m, cases_a)
        return Plan([base.dgrid] * len(cases_m), winf, s.params(args.tol, args.max_iter), dev), base

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- headline: mixed-precision batch solve, device resident ------------
    plan, base = make_plan(np.float32, machs, alphas)
    for _ in range(args.warmup):
        batch_solve(plan, args.max_iter)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    t0 = time.perf_counter()
    runs = [batch_solve(plan, args.max_iter) for _ in range(args.steps)]
    barrier()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    elapsed_ms = sum(r[0] for r in runs)
    converged = sum(int(r[3].sum()) for r in runs)
    kps, _ = plan.stats()
    launches = sum(r[5] * (kps + 1) + 2 for r in runs)
    elapsed_ms, converged = replicas.job_time_and_count(elapsed_ms, converged, dist, dev)
    converged = int(converged)
    step_ms, live = batch_solve.last_step_ms, batch_solve.last_live
    step_profile = {"ms_per_newton_step_by_live_cases": {
        f"{lo}-{hi}": round(float(step_ms[(live >= lo) & (live <= hi)].mean()), 3)
        for lo, hi in ((B * 3 // 4 + 1, B), (B // 4 + 1, B * 3 // 4), (2, B // 4), (1, 1))
        if ((live >= lo) & (live <= hi)).any()}}
    lat = np.concatenate([r[1][r[3]] for r in runs]) if converged else np.array([np.nan])
    nsteps_mix = runs[-1][2]
    coef_mix = plan.forces()[0].cpu().numpy()
    conv_mix = runs[-1][3]
    value = converged / (elapsed_ms / 1e3)
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "cases/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(elapsed_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64",
        "data": "synthetic (seeded NACA 2412 cases; random (M, alpha) per case)",
        "config": {"workload": f"{B} cases on one 256x64 O-grid of NACA 2412, M~U[0.30,0.75], alpha~U[-4,8] deg, "
                               f"seed {SEED}+rank, Newton-Krylov to residual drop {args.tol:g}",
                   "cases_per_gpu": B, "grid": "256x64 (ogrid naca4('2412',129), nj=65, ds0=2e-3, radius=20)",
                   "gmres_restart": args.restart, "jacobi_sweeps": 4, "max_newton_steps": args.max_iter,
                   "precision": "mixed: FP64 residual/factorisation/Gram-Schmidt/update; FP32 JVP, face Jacobians, sweep arithmetic; FP16 sweep factors; BF16 Krylov basis",
                   "l2": "working set ~2 GB per batch, larger than the 126 MB L2 (no flush needed)",
                   "parallelism": f"replicas x{world}, case sharding"},
        "converged_cases": converged,
        "cases_total": B * args.steps * world,
        "newton_steps_mean": round(float(nsteps_mix.mean()), 2),
        "step_profile": step_profile,
        "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 2), "p95": round(float(np.percentile(lat, 95)), 2),
                       "p99": round(float(np.percentile(lat, 99)), 2),
                       "note": "per converged case, from batch start to its retirement"},
    }
    if rank != 0:
        return None

    # ---- plain FP64 batch and the per-case FP64 path -----------------------
    plan64, _ = make_plan(np.float64, machs, alphas)
    batch_solve(plan64, args.max_iter)
    r64 = batch_solve(plan64, args.max_iter)
    coef64 = plan64.forces()[0].cpu().numpy()
    conv64 = r64[3]
    out["fp64_batched"] = {"value": round(int(conv64.sum()) / (r64[0] / 1e3), 3), "unit": "cases/s",
                           "ms_per_batch": round(r64[0], 1), "newton_steps_mean": round(float(r64[2].mean()), 2)}
    single, _ = make_plan(np.float64, machs[:1], alphas[:1])
    batch_solve(single, args.max_iter)
    t_single, n_single = 0.0, 0
    for k in range(args.single_sample):
        pk, _ = make_plan(np.float64, machs[k:k + 1], alphas[k:k + 1])
        batch_solve(pk, 2)
        r1 = batch_solve(pk, args.max_iter)
        t_single += r1[0]
        n_single += int(r1[3].sum())
        del pk
    per_case_rate = n_single / (t_single / 1e3) if n_single else 0.0
    out["fp64_per_case"] = {"value": round(per_case_rate, 3), "unit": "cases/s",
                            "sample": f"cases 0..{args.single_sample - 1} solved one at a time (B=1 plans)",
                            "ratio_mixed_batched_over_this": round(value / per_case_rate, 2) if per_case_rate else None}
    both = conv_mix & conv64
    dcl = np.abs(coef_mix[:, 0] - coef64[:, 0])[both]
    dcd = np.abs(coef_mix[:, 1] - coef64[:, 1])[both]
    dcm = np.abs(coef_mix[:, 2] - coef64[:, 2])[both]
    out["accuracy_vs_fp64"] = {"max_abs_dCl": float(dcl.max()) if both.any() else None,
                               "max_abs_dCd": float(dcd.max()) if both.any() else None,
                               "max_abs_dCm": float(dcm.max()) if both.any() else None,
                               "cases_compared": int(both.sum()),
                               "gate": "|dCl| <= 1e-4 and |dCd| <= 2e-6 against the FP64 path "
                                       "(parity-pinned to the FP64 oracle)"}

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

    # ---- end to end through the public API ---------------------------------
    def e2e_once():
        torch.cuda.synchronize()
        t = time.perf_counter()
        s = ImplicitEuler(EulerSolver(grid, dtype=np.float32, device=dev), gmres_restart=args.restart)
        r = s.solve(machs, alphas, n_iter=args.max_iter, tol=args.tol, verbose=False)
        torch.cuda.synchronize()
        return time.perf_counter() - t, r, s
    e2e_once()
    te, r, s = e2e_once()
    conv_e2e = int((s.done & ~s.frozen).sum())
    ni, nj = grid.shape
    h2d = 2 * ni * nj * 8 + B * 4 * 8 + plan.table_bytes()
    d2h = (r.cl.nbytes + r.cd.nbytes + r.cm.nbytes + r.cp.nbytes + r.res_hist.nbytes
           + s.cl_history.nbytes + B * (3 * 4 + 2 * 8))
    out["e2e"] = {"value": round(conv_e2e / te, 3), "unit": "cases/s", "h2d_bytes_per_step": int(h2d),
                  "d2h_bytes_per_step": int(d2h), "seconds": round(te, 3),
                  "call": "ImplicitEuler(EulerSolver(grid, dtype=float32), gmres_restart=30).solve(machs, alphas, "
                          "n_iter=200, tol=1e-10) with host arrays in and numpy results out"}
    out["e2e"]["converged_cases"] = conv_e2e
    out["gpu_launches"] = int(launches)
    out["clocks"] = clk

    # ---- served polar requests (continuous batching, ragged grids) ----------
    if world == 1 and args.served_requests > 0:
        out["served"] = served_arm(args, dev)

    # ---- CPU baseline ---------------------------------------------------------
    if world == 1 and not args.no_cpu_baseline:
        procs = max(1, min(os.cpu_count() or 1, args.cpu_procs))
        rate, per_step, cpu_wall = cpu_oracle_rate(procs)
        out["cpu_baseline"] = {"value": round(rate, 5), "unit": "cases/s", "cores": procs, "kind": "port",
                               "cpu": f"{cpu_model()}, {os.cpu_count()} logical CPUs",
                               "sample": f"one Newton step (restart {RESTART}, 4 sweeps) of {procs} cases of this "
                                         f"workload, one spawned process per case with one BLAS thread, "
                                         f"{per_step:.2f} s per step; cases/s = processes / step time / "
                                         f"{NEWTON_STEPS_PER_CASE} Newton steps per converged case",
                               "wall_s": round(cpu_wall, 1)}
    return out


# served polar requests: the grid sizes of the ragged set (n_side, nj, ds0), radius 20
SERVED_SIZES = [(65, 33, 2e-3), (97, 49, 2e-3), (129, 65, 2e-3), (193, 97, 1e-3)]
SERVED_ALPHAS = np.arange(-4.0, 17.0, 1.0)


def served_arm(args, dev):
    """Served polar requests on one GPU: a seeded Poisson stream of requests,
    each a 21-point alpha sweep (-4 .. 16 deg) at one random NACA 4-digit
    airfoil (m ~ U[0, 0.06], p ~ U[0.2, 0.6], t ~ U[0.08, 0.16]; airfoils whose
    grid folds are redrawn) on one grid size of the ragged set (128x32 ..
    384x96, radius 20), M ~ U[0.2, 0.75], alpha continuation inside the
    request, mixed precision, residual drop 1e-8 per point (at most
    `served_max_iter` Newton steps).  Each request's grid is generated on the
    device when it arrives; slots per grid size come from an HBM budget split
    equally between the sizes.  Latency = arrival to the last point's result
    (host wall clock: requests arrive in real time)."""
    import torch
    from aero2d_b200.geometry import naca4, naca4_params
    from aero2d_b200.grid import GridError
    from aero2d_b200.gridgen import ogrid_batch
    from aero2d_b200.service import EulerService, slots_for_budget
    rng = np.random.default_rng(SEED + 7)
    n = args.served_requests
    arrivals = np.cumsum(rng.exponential(1.0 / args.served_rate, n))
    reqs, rejected = [], 0
    while len(reqs) < n:
        m, pp, t = rng.uniform(0, 0.06), rng.uniform(0.2, 0.6), rng.uniform(0.08, 0.16)
        size = int(rng.integers(len(SERVED_SIZES)))
        mach = rng.uniform(0.2, 0.75)
        reqs.append((naca4_params(m, pp, t, SERVED_SIZES[size][0]), size, mach))
    shapes = [(2 * ns - 2, nj - 1) for ns, nj, _ in SERVED_SIZES]
    slots = slots_for_budget(shapes, args.served_hbm_gb * 1e9)
    defaults = [ogrid_batch([naca4("0012", ns)], nj=nj, ds0=ds0, radius=20.0, device=dev)[0]
                for ns, nj, ds0 in SERVED_SIZES]
    svc = EulerService(classes=list(zip(defaults, slots)), dtype=np.float32, device=dev, tol=1e-8,
                       max_iter=args.served_max_iter, gmres_restart=RESTART)
    # warm the service (graph capture, first launches) with one short request
    w = svc.submit(0.5, [2.0], grid=defaults[0])
    svc.run()
    svc.result(w)
    rid_of, arr_of, grid_of, done_at = {}, {}, {}, {}
    steps = 0
    nxt = 0
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
            rid = svc.submit(mach, SERVED_ALPHAS, continuation=True, grid=g)
            rid_of[nxt], arr_of[rid], grid_of[rid] = rid, arrivals[nxt], (g, mach)
            nxt += 1
        busy = svc.step()
        steps += busy > 0
        for rid in svc.poll():
            done_at[rid] = time.perf_counter() - t0
        if busy == 0 and svc.pending()[0] == 0 and nxt < n:
            time.sleep(max(0.0, arrivals[nxt] - (time.perf_counter() - t0)))
    wall = time.perf_counter() - t0
    res = {rid: svc.result(rid) for rid in done_at}
    lat = np.array([done_at[r] - arr_of[r] for r in done_at])
    conv = sum(int(r["converged"].sum()) for r in res.values())
    pts = sum(r["converged"].size for r in res.values())
    span = max(done_at.values()) - float(arrivals[0]) if done_at else float("nan")
    svc.close()
    # accuracy: the first two finished requests again in FP64, same grids and sweeps
    acc_ids = sorted(done_at, key=done_at.get)[:2]
    by_shape: dict = {}
    for r in acc_ids:
        by_shape.setdefault((grid_of[r][0].ni, grid_of[r][0].nc), []).append(r)
    ref = EulerService(classes=[(grid_of[rs[0]][0], len(rs)) for rs in by_shape.values()], dtype=np.float64,
                       device=dev, tol=1e-8, max_iter=args.served_max_iter, gmres_restart=RESTART)
    rid64 = {r: ref.submit(grid_of[r][1], SERVED_ALPHAS, continuation=True, grid=grid_of[r][0]) for r in acc_ids}
    ref.run()
    dcl, dcd, ncmp = [], [], 0
    for r, r64 in rid64.items():
        a, b = res[r], ref.result(r64)
        # points that reached the 1e-8 drop in both (the reference's converged flag asks only 1e-3)
        both = a["converged"] & b["converged"] & (a["nsteps"] < args.served_max_iter) & \
            (b["nsteps"] < args.served_max_iter)
        ncmp += int(both.sum())
        if both.any():
            dcl.append(np.abs(a["cl"] - b["cl"])[both].max())
            dcd.append(np.abs(a["cd"] - b["cd"])[both].max())
    ref.close()
    return {
        "workload": f"{n} requests, Poisson arrivals at {args.served_rate:g}/s (seeded), 21-point alpha sweep "
                    "-4..16 deg each with continuation, random NACA 4-digit airfoil and grid size "
                    "(128x32, 192x48, 256x64, 384x96), M~U[0.2,0.75], mixed precision, drop 1e-8, "
                    f"at most {args.served_max_iter} Newton steps per point, grids generated on the device",
        "slots": dict(zip([f"{a}x{b}" for a, b in shapes], slots)),
        "hbm_budget_gb": args.served_hbm_gb,
        "requests_done": len(done_at), "grid_rejections": rejected,
        "latency_s": {"p50": round(float(np.percentile(lat, 50)), 3), "p95": round(float(np.percentile(lat, 95)), 3),
                      "p99": round(float(np.percentile(lat, 99)), 3)} if len(lat) else None,
        "points": pts, "converged_points": conv,
        "converged_points_per_s": round(conv / span, 3) if done_at else None,
        "newton_steps": steps, "wall_s": round(wall, 2),
        "accuracy_vs_fp64": {"max_abs_dCl": float(max(dcl)) if dcl else None,
                             "max_abs_dCd": float(max(dcd)) if dcd else None, "points_compared": ncmp,
                             "sample": "the first two finished requests re-served in FP64; points that reached "
                                       "the 1e-8 drop in both"},
    }


def reference_arm(args):
    """The reference's CPU path: JAX is not installable here, so its FP64
    NumPy restatement (oracle/) runs on all host cores."""
    procs = max(1, os.cpu_count() or 1)
    for _ in range(args.warmup if args.warmup < 1 else 1):
        cpu_oracle_rate(procs)
    vals, per = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rate, per_step, _ = cpu_oracle_rate(procs)
        vals.append(rate)
        per.append(per_step)
    wall = time.perf_counter() - t0
    value = statistics.mean(vals)
    return {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "cases/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * wall / args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded NACA 2412 cases)",
            "config": {"workload": f"{CASES} cases on one 256x64 O-grid of NACA 2412, M~U[0.30,0.75], "
                                   f"alpha~U[-4,8] deg, seed {SEED}, Newton-Krylov to residual drop {TOL:g}",
                       "gmres_restart": RESTART},
            "cpu_baseline": {"value": round(value, 5), "unit": "cases/s", "cores": procs, "kind": "port",
                             "cpu": f"{cpu_model()}, {os.cpu_count()} logical CPUs",
                             "sample": f"per step: one Newton step of {procs} cases on {procs} spawned processes "
                                       f"({statistics.mean(per):.2f} s per Newton step); the JAX reference "
                                       "cannot be installed in this image (no jax wheel, no network)"},
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
    ap.add_argument("--tol", type=float, default=TOL)
    ap.add_argument("--max-iter", type=int, default=MAX_ITER)
    ap.add_argument("--single-sample", type=int, default=4)
    ap.add_argument("--cpu-procs", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--served-requests", type=int, default=24, help="0 skips the served-requests measurement")
    ap.add_argument("--served-rate", type=float, default=8.0, help="request arrivals per second")
    ap.add_argument("--served-hbm-gb", type=float, default=2.0, help="workspace budget of the service")
    ap.add_argument("--served-max-iter", type=int, default=100, help="Newton steps per point at most")
    ap.add_argument("--served-wall-cap", type=float, default=150.0, help="seconds before the stream is cut")
    ap.add_argument("--profile", type=int, default=0, metavar="STEPS",
                    help="profiling driver: build the mixed plan, run STEPS Newton steps, print nothing")
    ap.add_argument("--fp64", action="store_true", help="with --profile: the all-FP64 plan")
    args = ap.parse_args()
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
