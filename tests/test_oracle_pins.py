"""The oracle against the reference's own known answers and golden values
(no GPU).  These pins are what makes the oracle a trustworthy checker."""
import numpy as np
import pytest

from oracle.euler_oracle import (EulerModel, cons_to_prim, hllc_flux, prim_to_cons, vmax, vmin)
from oracle.implicit_oracle import ImplicitModel, hessenberg_lstsq
from tests.helpers import grid, perturbed_state


def test_hllc_consistency():
    """tests/test_euler.py:15-24."""
    W = np.array([[1.2], [0.3], [-0.1], [0.9]])
    S = np.array([[0.6], [0.8]])
    F = hllc_flux(W, W, S)
    r, u, v, p = W[:, 0]
    q = u * 0.6 + v * 0.8
    E = p / 0.4 + 0.5 * r * (u * u + v * v)
    ref = np.array([r * q, r * u * q + p * 0.6, r * v * q + p * 0.8, (E + p) * q])
    assert np.allclose(F[:, 0], ref, rtol=1e-6)


def test_prim_cons_roundtrip():
    """tests/test_euler.py:27-29."""
    W = np.array([1.1, 0.4, -0.2, 0.7])
    assert np.allclose(cons_to_prim(prim_to_cons(W)), W, rtol=1e-6)


def test_freestream_preserved():
    """tests/test_euler.py:32-40."""
    g = grid("0012", 33, 25)
    m = EulerModel(g.x, g.y, vortex_correction=False)
    w = m.freestream(0.5, 3.0)
    R, _ = m.residual(m.init_state(w), w, 0.0)
    assert np.max(np.abs(R[:, :, 3:]) / m.vol[None, :, 3:]) < 1e-3


@pytest.mark.parametrize("case,key", [(0, "U_m05_a2"), (1, "U_m08_a125")])
def test_converged_state_reproduces_published_cl(converged_0012, known_answers, case, key):
    """benchmarks/results.json FP64 lift and drag of the reference, reproduced
    from the oracle's converged state, whose residual is at the rounding floor."""
    g = grid("0012", 65, 49, 2e-3, 40.0)
    m = EulerModel(g.x, g.y)
    ref = known_answers["results_json"]["cases"][case]
    w = m.freestream(ref["mach"], ref["alpha"])
    U = converged_0012[key]
    cl, cd, cm, cp = m.forces(U, w)
    assert abs(cl - ref["cl_fp64"]) < 1e-12
    assert abs(cd - ref["cd_fp64"]) < 1e-12
    circ = m.circulation(U, w)
    R, _ = m.residual(U, w, circ)
    assert np.max(np.abs(R) / m.flux_scale(U, w, circ)) < 1e-11


def test_complex_step_jvp_matches_finite_difference():
    g = grid("0012", 33, 25)
    m = EulerModel(g.x, g.y)
    im = ImplicitModel(m)
    w = m.freestream(0.6, 2.0)
    U = perturbed_state(m, w, seed=3)
    v = np.random.default_rng(1).standard_normal(U.shape)
    jv = im.jvp(U, w, v)
    h = 1e-6
    fd = (im.res(U + h * v, w)[0] - im.res(U - h * v, w)[0]) / (2 * h)
    assert np.max(np.abs(jv - fd)) / np.max(np.abs(jv)) < 1e-6


def test_balanced_ties():
    a = np.array([1.0 + 2.0j])
    b = np.array([1.0 + 4.0j])
    assert vmax(a, b)[0] == 1.0 + 3.0j
    assert vmin(a, b)[0] == 1.0 + 3.0j


def test_block_thomas_is_exact():
    """The block-Thomas factorisation solves the block-tridiagonal line system
    exactly (the pattern of the reference's tests/test_rans.py:13-31)."""
    g = grid("0012", 33, 25)
    m = EulerModel(g.x, g.y)
    im = ImplicitModel(m, jacobi_sweeps=1)
    w = m.freestream(0.5, 1.0)
    U = perturbed_state(m, w, seed=5)
    circ = im.circ(U, w)
    R, W = m.residual(U, w, circ)
    dti = 1.0 / (m.local_dt(W) / m.cfl * 20.0)
    D, Bim, Bip, Bjm, Bjp = im.assemble(U, w, circ, dti)
    fac = im.factor_lines(D, Bjm, Bjp)
    r = np.random.default_rng(2).standard_normal(U.shape)
    x = im.solve_lines(fac, r)
    i = 7
    nc = m.nc
    A = np.zeros((4 * nc, 4 * nc))
    for j in range(nc):
        A[4 * j:4 * j + 4, 4 * j:4 * j + 4] = D[i, j]
        if j > 0:
            A[4 * j:4 * j + 4, 4 * (j - 1):4 * j] = Bjm[i, j]
        if j < nc - 1:
            A[4 * j:4 * j + 4, 4 * (j + 1):4 * (j + 2)] = Bjp[i, j]
    xd = np.linalg.solve(A, r[:, i, :].T.ravel())
    assert np.allclose(x[:, i, :].T.ravel(), xd, rtol=1e-10, atol=1e-12)


def test_hessenberg_lstsq_matches_numpy():
    rng = np.random.default_rng(0)
    k = 12
    H = np.triu(rng.standard_normal((k + 1, k)), -1)
    y = hessenberg_lstsq(H, 2.5)
    e = np.zeros(k + 1)
    e[0] = 2.5
    yn = np.linalg.lstsq(H, e, rcond=None)[0]
    assert np.allclose(y, yn, rtol=1e-10, atol=1e-12)


@pytest.mark.slow
def test_full_oracle_solve_reproduces_results_json(known_answers):
    """80 Newton steps (restart 50) on the results.json grid: the drop and the
    lift of the reference's FP64 run (minutes of CPU)."""
    g = grid("0012", 65, 49, 2e-3, 40.0)
    im = ImplicitModel(EulerModel(g.x, g.y))
    ref = known_answers["results_json"]
    r = im.solve([0.5], [2.0], n_iter=80, tol=0.0)
    assert abs(r["cl"][0] - ref["cases"][0]["cl_fp64"]) < 1e-10
    drop = np.log10(r["res_hist"][-1][0] / r["res_hist"][0][0])
    assert abs(drop - ref["log10_res_drop_fp64"][0]) < 0.2


def test_fas_cycle_fixed_point_at_converged_state(converged_0012, known_answers):
    """The FAS V-cycle (aero2d/euler.py:368-381) leaves a converged solution in
    place: the coarse forcing makes the coarse problem's solution the restricted
    state, so the prolonged correction vanishes to the residual level.  No test
    of the reference covers its multigrid; this pins the transfers' consistency
    (restriction, forcing and prolongation of the oracle's restatement)."""
    g = grid("0012", 65, 49, 2e-3, 40.0)
    ref = known_answers["results_json"]["cases"][0]
    U = converged_0012["U_m05_a2"]
    for levels in (2, 3):
        m = EulerModel(g.x, g.y, mg_levels=levels)
        w = m.freestream(ref["mach"], ref["alpha"])
        circ = m.circulation(U, w)
        U1, res = m.cycle(U, w, circ)
        assert np.max(np.abs(U1 - U)) < 1e-10 * np.max(np.abs(U))
        assert res < 1e-10


def test_fas_transfers():
    """Restriction preserves the volume integral; prolongation of a constant
    correction is that constant; odd grids are rejected (aero2d/euler.py:245-246)."""
    g = grid("2412", 33, 25)
    m = EulerModel(g.x, g.y, mg_levels=2)
    rng = np.random.default_rng(3)
    U = rng.standard_normal((4, m.ni, m.nc))
    Uc = m.sum4(U * m.vol[None]) / m.sum4(m.vol)[None]
    assert np.allclose((Uc * m.sum4(m.vol)[None]).sum(axis=(1, 2)), (U * m.vol[None]).sum(axis=(1, 2)))
    d = np.full((4, m.coarse.ni, m.coarse.nc), 0.37)
    assert np.array_equal(m.prolong(d), np.full((4, m.ni, m.nc), 0.37))
    g_odd = grid("0012", 33, 26)
    with pytest.raises(ValueError):
        EulerModel(g_odd.x, g_odd.y, mg_levels=2)
