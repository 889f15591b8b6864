"""Parity of converged solutions with the FP64 oracle on the benchmark
configurations, through the C ABI (aero2d_b200.plan.Plan / ImplicitEuler).

Known answers: tests/golden/oracle_configs.json, converged FP64 oracle
solutions written by tests/golden/make_configs.py (oracle/implicit_oracle.py,
the restatement of aero2d/implicit.py:169-253 with GMRES restart 30):
  c1      NACA 0012, 192 x 48, M 0.5, alpha 1.25 deg, drop 1e-10
  c2_k    8 cases of the 64-case NACA 2412 256 x 64 batch (seed 2412), drop 1e-10
  c3_k    transonic random NACA 4-digit sections on 384 x 96 grids, M 0.70-0.80
Gates: the all-FP64 path within 1e-8 of the oracle in Cl, Cd, Cm and every wall
Cp on cases the oracle converged to the tolerance; the mixed path within
|dCl| <= 1e-4 and |dCd| <= 2e-6 (its |dCm| and shock shift are printed); the
forces and the wall Cp of a given state within 1e-12 of the oracle's
(aero2d/euler.py:315-331)."""
import json

import numpy as np
import pytest
import torch

from aero2d_b200.core import shock_position
from aero2d_b200.euler import EulerSolver, compute_metrics
from aero2d_b200.geometry import naca4, naca4_params
from aero2d_b200.grid import ogrid
from aero2d_b200.implicit import ImplicitEuler
from aero2d_b200.plan import Plan
from oracle.euler_oracle import EulerModel, cons_to_prim
from tests.conftest import GOLDEN
from tests.helpers import grid, perturbed_state

pytestmark = pytest.mark.gpu

FIXTURES = GOLDEN / "oracle_configs.json"


def configs():
    return json.load(open(FIXTURES))["cases"]


def config_grid(g):
    af = naca4(g["code"], g["n_side"]) if "code" in g else naca4_params(g["m"], g["p"], g["t"], g["n_side"])
    return ogrid(af, nj=g["nj"], ds0=g["ds0"], radius=g["radius"])


def solve_cases(cases, dtype, device, gmres_restart=30):
    """One batch plan (ragged when the grids differ) solved to each case's
    tolerance; returns per-case (done, coef [3], cp [ni], nsteps)."""
    grids = [config_grid(c["grid"]) for c in cases]
    solvers = [EulerSolver(g, dtype=dtype, device=device) for g in grids]
    imp = ImplicitEuler(solvers[0], gmres_restart=gmres_restart)
    machs = np.array([c["mach"] for c in cases])
    alphas = np.array([c["alpha"] for c in cases])
    tol, n_iter = cases[0]["tol"], max(c["n_iter"] for c in cases)
    pl = Plan([s.dgrid for s in solvers], solvers[0].freestream(machs, alphas), imp.params(tol, n_iter), device)
    pl.init_freestream()
    pl.newton_run(n_iter)
    nsteps, done, frozen, lastrn, r0 = pl.status()
    coef, cps = pl.forces()
    out = dict(done=done & ~frozen, coef=coef.cpu().numpy(), cp=[c.cpu().numpy() for c in cps], nsteps=nsteps,
               grids=grids, saturations=pl.factor_saturations())
    pl.close()
    return out


def groups():
    cs = configs()
    return {"c1": [cs["c1"]], "c2": [cs[f"c2_{k}"] for k in range(8)],
            "c3": [cs[k] for k in sorted(cs) if k.startswith("c3_")]}


@pytest.mark.parametrize("key,name", [("U_m05_a2", 0), ("U_m08_a125", 1)])
def test_forces_and_cp_vs_oracle(cuda, converged_0012, known_answers, key, name):
    """Cl, Cd, Cm and the wall Cp of the converged golden states (and of a
    perturbed state) against the oracle's forces (aero2d/euler.py:315-331)."""
    g = grid("0012", 65, 49, 2e-3, 40.0)
    om = EulerModel(g.x, g.y)
    ref = known_answers["results_json"]["cases"][name]
    w = om.freestream(ref["mach"], ref["alpha"])
    s = EulerSolver(g, dtype=np.float64, device=cuda)
    for U in (converged_0012[key], perturbed_state(om, w, seed=5 + name)):
        cl, cd, cm, cp = om.forces(U, w)
        gl, gd, gm, gcp = s.forces(torch.as_tensor(U, device=cuda), w)
        assert abs(gl - cl) < 1e-12 and abs(gd - cd) < 1e-12 and abs(gm - cm) < 1e-12, ((gl, cl), (gd, cd), (gm, cm))
        assert np.max(np.abs(gcp.cpu().numpy() - cp)) < 1e-12


def test_local_dt_and_primitives_vs_oracle(cuda):
    """EulerSolver.local_dt (aero2d/euler.py:289-296) and the W that
    EulerSolver.residual returns (euler.py:260) against the oracle."""
    g = grid("2412", 65, 33)
    om = EulerModel(g.x, g.y)
    w = om.freestream(0.6, 3.0)
    U = perturbed_state(om, w, seed=11)
    W = cons_to_prim(U)
    s = EulerSolver(g, dtype=np.float64, device=cuda)
    dt = s.local_dt(torch.as_tensor(W, device=cuda)).cpu().numpy()
    dto = om.local_dt(W)
    assert dt.shape == dto.shape
    assert np.max(np.abs(dt - dto) / dto) < 1e-13
    _, Wg = s.residual(torch.as_tensor(U, device=cuda), w)
    assert np.max(np.abs(Wg.cpu().numpy() - W) / np.maximum(np.abs(W), 1.0)) < 1e-15


@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_fp64_converged_solutions_vs_oracle(cuda, name):
    """The all-FP64 path: converged Cl, Cd, Cm and wall Cp within 1e-8 of the
    oracle on every case the oracle took to the tolerance."""
    cases = groups()[name]
    r = solve_cases(cases, np.float64, cuda)
    compared = 0
    for k, c in enumerate(cases):
        oracle_done = c["log10_drop"] <= np.log10(c["tol"]) and not c["frozen"]
        if not oracle_done:
            continue
        assert r["done"][k], f"{c['name']}: the GPU did not reach the tolerance the oracle reached"
        coef = r["coef"][k]
        d = np.abs(coef - [c["cl"], c["cd"], c["cm"]])
        assert np.all(d <= 1e-8), (c["name"], d)
        assert np.max(np.abs(r["cp"][k] - np.asarray(c["cp"]))) <= 1e-8, c["name"]
        assert abs(int(r["nsteps"][k]) - c["newton_steps"]) <= 2, (c["name"], r["nsteps"][k], c["newton_steps"])
        compared += 1
    assert compared >= (1 if name == "c1" else 3), f"{name}: only {compared} cases compared"


@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_mixed_converged_solutions_vs_oracle(cuda, name):
    """The mixed-precision path (FP32 JVP, face Jacobians and sweeps around the
    FP64 residual, factorisation, Gram-Schmidt and update): |dCl| <= 1e-4,
    |dCd| <= 2e-6 against the FP64 oracle; |dCm| and, on the transonic cases,
    the upper-surface shock shift are reported."""
    cases = groups()[name]
    r = solve_cases(cases, np.float32, cuda)
    compared, dcm, shift = 0, [], []
    for k, c in enumerate(cases):
        oracle_done = c["log10_drop"] <= -8 and not c["frozen"]
        if not (oracle_done and r["done"][k]):
            continue
        coef = r["coef"][k]
        assert abs(coef[0] - c["cl"]) <= 1e-4, (c["name"], coef[0], c["cl"])
        assert abs(coef[1] - c["cd"]) <= 2e-6, (c["name"], coef[1], c["cd"])
        dcm.append(abs(coef[2] - c["cm"]))
        if "shock_x" in c:
            m = compute_metrics(r["grids"][k])
            xs = shock_position(m.xw, m.yw, r["cp"][k], c["mach"])
            assert np.isnan(xs) == np.isnan(c["shock_x"]), c["name"]
            if not np.isnan(xs):
                shift.append(abs(xs - c["shock_x"]))
                assert shift[-1] <= 2e-3, (c["name"], xs, c["shock_x"])
        compared += 1
    assert compared >= (1 if name == "c1" else 3), f"{name}: only {compared} cases compared"
    if name == "c3":
        # the stiffest configuration (384 x 96, first spacing 1e-3, CFL up to 300): no sweep
        # factor left the FP16 range in the whole solve
        assert r["saturations"] == 0, r["saturations"]
    print(f"{name}: {compared} cases, max |dCm| {max(dcm):.2e}, shock shifts {shift}, "
          f"FP16 factor saturations {r['saturations']}")
