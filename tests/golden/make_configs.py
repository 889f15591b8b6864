"""Generates tests/golden/oracle_configs.json: converged FP64 oracle solutions of
the benchmark configurations, the known answers that the GPU parity tests and
the bench's accuracy report compare against.  Run by hand in the build
container (CPU only, about an hour on 8 cores; one spawned process per case):

    python tests/golden/make_configs.py [--procs 8] [--only c1,c2,c3] [--force]

(cases already in the file are kept unless --force)

Cases (all with the reference's ImplicitEuler defaults except GMRES restart 30,
aero2d/implicit.py:68-70, from the uniform freestream, one case per solve):
  c1        NACA 0012, ogrid(naca4("0012", 97), nj=49, ds0=2e-3, radius=20)
            (192 x 48 cells), M 0.5, alpha 1.25 deg, residual drop 1e-10,
            at most 200 Newton steps
  c2_<k>    the first 8 cases of the 64-case batch on one 256 x 64 O-grid of
            NACA 2412 (ogrid(naca4("2412", 129), nj=65, ds0=2e-3, radius=20)),
            M ~ U[0.30, 0.75] then alpha ~ U[-4, 8] deg from default_rng(2412),
            drop 1e-10, at most 200 Newton steps
  c3_<k>    the 8 transonic cases of tests.helpers.transonic_draw(): random NACA
            4-digit sections on their own 384 x 96 O-grids (ds0 1e-3, radius 20),
            M ~ U[0.70, 0.80], alpha ~ U[0, 3] deg, drop 1e-10, at most 300 steps

Per case: Cl, Cd, Cm, the wall Cp, the residual history, the Newton steps taken,
the reference's converged flag (drop below 1e-3 and not frozen,
aero2d/implicit.py:252) and, for c3, the upper-surface shock position
(aero2d_b200.core.shock_position, Cp rising through Cp*), plus the oracle's
mean seconds per Newton step on this machine (informational: the processes
share the cores).
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "oracle_configs.json"

C2_SEED, C2_BATCH, C2_SAMPLE = 2412, 64, 8


def case_list(only):
    import numpy as np
    cases = []
    if "c1" in only:
        cases.append(dict(name="c1", grid=dict(code="0012", n_side=97, nj=49, ds0=2e-3, radius=20.0),
                          mach=0.5, alpha=1.25, tol=1e-10, n_iter=200))
    if "c2" in only:
        rng = np.random.default_rng(C2_SEED)
        machs = rng.uniform(0.30, 0.75, C2_BATCH)
        alphas = rng.uniform(-4.0, 8.0, C2_BATCH)
        for k in range(C2_SAMPLE):
            cases.append(dict(name=f"c2_{k}", grid=dict(code="2412", n_side=129, nj=65, ds0=2e-3, radius=20.0),
                              mach=float(machs[k]), alpha=float(alphas[k]), tol=1e-10, n_iter=200))
    if "c3" in only:
        from tests.helpers import transonic_draw
        params, _, machs, alphas, _ = transonic_draw()
        for k, (m, p, t) in enumerate(params):
            cases.append(dict(name=f"c3_{k}", grid=dict(m=m, p=p, t=t, n_side=193, nj=97, ds0=1e-3, radius=20.0),
                              mach=float(machs[k]), alpha=float(alphas[k]), tol=1e-10, n_iter=300))
    return cases


def make_grid(g):
    from aero2d_b200.geometry import naca4, naca4_params
    from aero2d_b200.grid import ogrid
    af = naca4(g["code"], g["n_side"]) if "code" in g else naca4_params(g["m"], g["p"], g["t"], g["n_side"])
    return ogrid(af, nj=g["nj"], ds0=g["ds0"], radius=g["radius"])


def solve_case(c):
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, str(ROOT))
    import numpy as np
    from aero2d_b200.core import shock_position
    from aero2d_b200.euler import compute_metrics
    from oracle.euler_oracle import EulerModel
    from oracle.implicit_oracle import ImplicitModel
    g = make_grid(c["grid"])
    im = ImplicitModel(EulerModel(g.x, g.y), gmres_restart=30)
    t = time.perf_counter()
    r = im.solve([c["mach"]], [c["alpha"]], n_iter=c["n_iter"], tol=c["tol"])
    sec = time.perf_counter() - t
    hist = np.asarray(r["res_hist"])[:, 0]
    out = dict(c, cl=float(r["cl"][0]), cd=float(r["cd"][0]), cm=float(r["cm"][0]),
               cp=[float(v) for v in r["cp"][0]], res_hist=[float(v) for v in hist],
               r0=float(r["r0"][0]), newton_steps=int(im.steps_taken[0]),
               log10_drop=float(np.log10(hist[np.isfinite(hist)][-1] / r["r0"][0])),
               converged=bool(r["converged"][0]), frozen=bool(im.frozen[0]),
               seconds_per_step=sec / max(1, int(im.steps_taken[0])))
    if c["name"].startswith("c3"):
        m = compute_metrics(g)
        out["shock_x"] = float(shock_position(m.xw, m.yw, r["cp"][0], c["mach"]))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", default="c1,c2,c3")
    ap.add_argument("--force", action="store_true", help="recompute cases already in the file")
    a = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    only = set(a.only.split(","))
    old = json.load(open(OUT)) if OUT.exists() else {"cases": {}}
    cases = [c for c in case_list(only) if a.force or c["name"] not in old["cases"]]
    # longest cases first so the pool's tail is short
    cases.sort(key=lambda c: -c["grid"]["n_side"] * c["grid"]["nj"] * c["n_iter"])
    with mp.get_context("spawn").Pool(a.procs) as pool:
        for res in pool.imap_unordered(solve_case, cases):
            old["cases"][res["name"]] = res
            old["generator"] = ("tests/golden/make_configs.py: oracle/implicit_oracle.py ImplicitModel "
                                "(gmres_restart=30, reference defaults otherwise), one case per solve")
            json.dump(old, open(OUT, "w"), indent=0)
            print(f"{res['name']}: {res['newton_steps']} steps, drop {res['log10_drop']:.2f}, "
                  f"Cl {res['cl']:.10f}", flush=True)


if __name__ == "__main__":
    main()
