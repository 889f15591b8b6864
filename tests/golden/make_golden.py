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
  ref_repanel.npz          contours re-panelled by aero2d.geometry.repanel (several
                           inputs: NACA sections, a blunt trailing edge, a contour with
                           corners, two-halves input, a mirrored unnormalised contour,
                           viscous spacing) and the grid of the polar scenario's coarse
                           level, ogrid(repanel(naca4("0012"), 65), nj=49, ds0=2e-3, radius=40)
  polar_known_answer.json  (--polar; ~2 min of CPU) FP64 oracle Cl, Cd of NACA 0012 at
                           M 0.5, alpha 2 deg on that polar grid, 80 Newton steps (residual
                           down 13 orders): the known answer of the polar scenario
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


# re-panelling cases: key -> (input contour, repanel keyword arguments); the tests
# rebuild the inputs from the stored coordinates and pass the same arguments
REPANEL_KW = {
    "naca0012_65": dict(n_side=65), "naca0012_97": dict(n_side=97), "naca0012_129": dict(n_side=129),
    "naca2412_65": dict(n_side=65), "naca4415_97": dict(n_side=97), "blunt0012_65": dict(n_side=65),
    "corners_49": dict(n_side=49), "halves2412_65": dict(n_side=65), "mirrored2412_65": dict(n_side=65),
    "viscous2412_65": dict(n_side=65, spacing="viscous"),
}


def repanel_inputs(naca4, Airfoil):
    def diamond():
        # a double-wedge section: sharp leading edge and shoulder corners
        xs = np.concatenate([np.linspace(1, 0.5, 15), np.linspace(0.5, 0, 15)[1:],
                             np.linspace(0, 0.5, 15)[1:], np.linspace(0.5, 1, 15)[1:]])
        ys = np.concatenate([np.linspace(0, 0.06, 15), np.linspace(0.06, 0, 15)[1:],
                             np.linspace(0, -0.06, 15)[1:], np.linspace(-0.06, 0, 15)[1:]])
        return Airfoil(xs, ys, "diamond")

    def halves():
        a = naca4("2412", 60)
        n = 60
        up_x, up_y = a.x[:n][::-1], a.y[:n][::-1]          # leading edge -> trailing edge, upper
        lo_x, lo_y = a.x[n - 1:], a.y[n - 1:]                # leading edge -> trailing edge, lower
        return Airfoil(np.concatenate([up_x, lo_x]), np.concatenate([up_y, lo_y]), "halves")

    def mirrored():
        a = naca4("2412", 70)
        ang = np.deg2rad(5.0)
        x, y = 2.0 * a.x + 0.3, 2.0 * a.y - 0.1
        xr, yr = x * np.cos(ang) - y * np.sin(ang), x * np.sin(ang) + y * np.cos(ang)
        return Airfoil(xr[::-1].copy(), yr[::-1].copy(), "mirrored")

    inputs = {
        "naca0012_65": naca4("0012"), "naca0012_97": naca4("0012"), "naca0012_129": naca4("0012"),
        "naca2412_65": naca4("2412"), "naca4415_97": naca4("4415", 60),
        "blunt0012_65": naca4("0012", 80, closed_te=False), "corners_49": diamond(),
        "halves2412_65": halves(), "mirrored2412_65": mirrored(), "viscous2412_65": naca4("2412"),
    }
    return {k: (inputs[k], REPANEL_KW[k]) for k in inputs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--converged", action="store_true")
    ap.add_argument("--polar", action="store_true")
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

    from aero2d.geometry import Airfoil, repanel   # noqa: E402  (reference)
    rep = {}
    for key, (af, kw) in repanel_inputs(naca4, Airfoil).items():
        out = repanel(af, **kw)
        rep[f"{key}_in_x"], rep[f"{key}_in_y"] = np.asarray(af.x, float), np.asarray(af.y, float)
        rep[f"{key}_out_x"], rep[f"{key}_out_y"] = out.x, out.y
    g = ogrid(repanel(naca4("0012"), 65), nj=49, ds0=2e-3, radius=40.0)
    rep["polar_coarse_0012_x"], rep["polar_coarse_0012_y"] = g.x, g.y
    np.savez_compressed(HERE / "ref_repanel.npz", **rep)

    if a.polar:
        sys.path.insert(0, str(ROOT))
        from oracle.euler_oracle import EulerModel
        from oracle.implicit_oracle import ImplicitModel
        im = ImplicitModel(EulerModel(g.x, g.y))          # g: the polar coarse grid above
        r = im.solve([0.5], [2.0], n_iter=80, tol=0.0)
        hist = np.asarray(r["res_hist"])[:, 0]
        json.dump({"grid": "ogrid(repanel(naca4('0012'), 65), nj=49, ds0=2e-3, radius=40)",
                   "mach": 0.5, "alpha": 2.0, "newton_steps": 80,
                   "log10_res_drop": float(np.log10(hist[-1] / hist[0])),
                   "cl_fp64": float(r["cl"][0]), "cd_fp64": float(r["cd"][0])},
                  open(HERE / "polar_known_answer.json", "w"), indent=1)
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
