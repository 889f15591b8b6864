"""Generates the golden fixtures under tests/golden/ from the reference
implementation and the oracle.  Needs the reference source tree (it imports
aero2d.grid, aero2d.geometry and aero2d.panel, which are pure NumPy) and is run
by hand in the build container:

    python tests/golden/make_golden.py [--reference /path/to/Aero2d] [--converged]

Outputs
  ref_grids.npz            O-grid nodes from aero2d.grid.ogrid for several airfoils
  ref_known_answers.json   panel-method Cl used by the reference's subsonic test
                           (tests/test_euler.py:55-60) and the FP64 Cl/Cd values
                           of benchmarks/results.json
  naca0012_128x48_r40_converged.npz  (--converged; ~10 min of CPU)
                           converged FP64 oracle states of the results.json cases
                           M 0.5 a 2 deg and M 0.8 a 1.25 deg (80 Newton steps)
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

GRIDS = {
    # key: (code, n_side, nj, ds0, radius)
    "0012_33_25": ("0012", 33, 25, 2e-3, 40.0),       # tests/test_euler.py:34 freestream test
    "0012_49_41": ("0012", 49, 41, 3e-3, 40.0),       # tests/test_euler.py:45 subsonic fixture
    "0012_65_49": ("0012", 65, 49, 2e-3, 40.0),       # benchmarks/results.json grid (128 x 48)
    "0012_97_49": ("0012", 97, 49, 2e-3, 20.0),       # 192 x 48, single-case FP64 workload
    "2412_65_33": ("2412", 65, 33, 2e-3, 20.0),       # cambered, 128 x 32
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--converged", action="store_true")
    a = ap.parse_args()
    sys.path.insert(0, a.reference)
    from aero2d.geometry import naca4          # noqa: E402  (reference)
    from aero2d.grid import ogrid              # noqa: E402  (reference)
    from aero2d.panel import PanelSolver       # noqa: E402  (reference)

    out = {}
    for key, (code, ns, nj, ds0, rad) in GRIDS.items():
        g = ogrid(naca4(code, ns), nj=nj, ds0=ds0, radius=rad)
        out[f"{key}_x"] = g.x
        out[f"{key}_y"] = g.y
    np.savez_compressed(HERE / "ref_grids.npz", **out)

    res = json.load(open(Path(a.reference) / "benchmarks" / "results.json"))
    known = {
        "panel_cl_0012_121_a2": float(PanelSolver(naca4("0012", 121)).solve(2.0).cl),
        "results_json": {
            "grid": res["euler"]["grid"],
            "cases": [{k: c[k] for k in ("mach", "alpha", "cl_fp64", "cd_fp64")}
                      for c in res["euler"]["cases"]],
            "log10_res_drop_fp64": res["euler"]["log10_res_drop_fp64"],
            "newton_its_fp64": res["euler"]["newton_its_fp64"],
        },
    }
    json.dump(known, open(HERE / "ref_known_answers.json", "w"), indent=1)

    if a.converged:
        sys.path.insert(0, str(ROOT))
        from oracle.euler_oracle import EulerModel
        from oracle.implicit_oracle import ImplicitModel
        g = ogrid(naca4("0012", 65), nj=49, ds0=2e-3, radius=40.0)
        im = ImplicitModel(EulerModel(g.x, g.y))
        states, cls = {}, []
        for name, m, al in (("U_m05_a2", 0.5, 2.0), ("U_m08_a125", 0.8, 1.25)):
            r = im.solve([m], [al], n_iter=80, tol=0.0)
            states[name] = r["U"][0]
            cls.append(r["cl"][0])
        np.savez_compressed(HERE / "naca0012_128x48_r40_converged.npz", cl=np.array(cls), **states)
    print("written to", HERE)


if __name__ == "__main__":
    main()
