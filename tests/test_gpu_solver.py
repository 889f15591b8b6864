"""The Newton-Krylov and explicit solvers on the GPU against the oracle and the
reference's published and known answers, through the reference-shaped API
(aero2d_b200.euler.EulerSolver, aero2d_b200.implicit.ImplicitEuler)."""
import numpy as np
import pytest
import torch

from aero2d_b200.euler import EulerSolver
from aero2d_b200.implicit import ImplicitEuler
from oracle.euler_oracle import EulerModel
from oracle.implicit_oracle import ImplicitModel
from tests.helpers import grid, perturbed_state

pytestmark = pytest.mark.gpu


def test_one_newton_step_vs_oracle(cuda):
    """One pseudo-transient Newton step from a perturbed state: the CUDA step
    and the oracle step build the same Krylov space; the updates agree to the
    rounding of a 30-vector GMRES cycle."""
    g = grid("0012", 33, 25)
    om = EulerModel(g.x, g.y)
    im = ImplicitModel(om, gmres_restart=30)
    w = om.freestream(0.5, 2.0)
    U = perturbed_state(om, w, seed=1, amp=0.01)
    Uo, rno, omo, _ = im.step(U, w, 10.0)
    s = ImplicitEuler(EulerSolver(g, dtype=np.float64, device=cuda), gmres_restart=30)
    Ug, rng, omg = s.step(torch.as_tensor(U), w, None, 10.0)
    Ug = Ug.cpu().numpy()
    assert abs(rng - rno) / rno < 1e-12
    assert abs(omg - omo) < 1e-8
    dUo = Uo - U
    assert np.max(np.abs((Ug - U) - dUo)) / np.max(np.abs(dUo)) < 1e-7


@pytest.mark.parametrize("case", [0, 1])
def test_solve_reproduces_published_fp64(cuda, known_answers, case):
    """benchmarks/results.json: NACA 0012 on ogrid(naca4("0012",65), nj=49,
    ds0=2e-3, radius=40), ImplicitEuler defaults (restart 50), FP64.  The
    converged lift must match the published FP64 value to 1e-8."""
    ref = known_answers["results_json"]["cases"][case]
    g = grid("0012", 65, 49, 2e-3, 40.0)
    s = ImplicitEuler(EulerSolver(g, dtype=np.float64, device=cuda))
    r = s.solve([ref["mach"]], [ref["alpha"]], n_iter=80, tol=1e-12, verbose=False)
    assert abs(r.cl[0] - ref["cl_fp64"]) < 1e-8, (r.cl[0], ref["cl_fp64"])
    assert abs(r.cd[0] - ref["cd_fp64"]) < 1e-8
    assert r.converged[0]


def test_mixed_precision_accuracy(cuda, known_answers):
    ref = known_answers["results_json"]["cases"][0]
    g = grid("0012", 65, 49, 2e-3, 40.0)
    s = ImplicitEuler(EulerSolver(g, dtype=np.float32, device=cuda))
    r = s.solve([ref["mach"]], [ref["alpha"]], n_iter=80, tol=1e-10, verbose=False)
    assert abs(r.cl[0] - ref["cl_fp64"]) <= 1e-4
    assert abs(r.cd[0] - ref["cd_fp64"]) <= 2e-6


def test_batch_invariance(cuda):
    """A case's FP64 result is bitwise the same alone and in a batch."""
    g = grid("0012", 33, 25)
    base = EulerSolver(g, dtype=np.float64, device=cuda)
    machs, alphas = [0.5, 0.6, 0.7], [1.0, -2.0, 3.0]
    rb = ImplicitEuler(base, gmres_restart=20).solve(machs, alphas, n_iter=12, tol=1e-9, verbose=False)
    for k in range(3):
        r1 = ImplicitEuler(base, gmres_restart=20).solve([machs[k]], [alphas[k]], n_iter=12, tol=1e-9,
                                                          verbose=False)
        assert torch.equal(r1.U[0], rb.U[k])
        assert r1.cl[0] == rb.cl[k]


def test_reference_subsonic_known_answers(cuda, known_answers):
    """tests/test_euler.py:43-65 of the reference: 96x40 grid, FP32 dtype,
    M 0.5, alpha 0 and 2 deg, 40 iterations, tol 1e-5."""
    g = grid("0012", 49, 41, 3e-3, 40.0)
    r = ImplicitEuler(EulerSolver(g, device=cuda)).solve([0.5, 0.5], [0.0, 2.0], n_iter=40, verbose=False,
                                                         tol=1e-5)
    assert abs(r.cl[0]) < 2e-3
    cl_pg = known_answers["panel_cl_0012_121_a2"] / np.sqrt(1 - 0.5 ** 2)
    assert abs(r.cl[1] / cl_pg - 1) < 0.04
    assert abs(r.cd[1]) < 3e-3
    drop = np.log10(r.res_hist[-1] / r.res_hist[0])
    assert np.all(drop < -3)


def test_freestream_preserved(cuda):
    """tests/test_euler.py:32-40: uniform flow is a discrete steady state away
    from the wall (no vortex correction)."""
    g = grid("0012", 33, 25)
    s = EulerSolver(g, vortex_correction=False, device=cuda)
    w = s.freestream(0.5, 3.0)
    U = s.init_state(w)
    R, _ = s.residual(U, w, 0.0)
    vol = torch.as_tensor(s.m_np.vol, device=cuda)
    assert float((R[:, :, 3:].abs() / vol[None, :, 3:]).max()) < 1e-3


def test_explicit_rk_vs_oracle(cuda):
    g = grid("0012", 33, 25)
    om = EulerModel(g.x, g.y)
    ro = om.solve([0.5], [2.0], n_iter=6, chunk=3, tol=0.0)
    s = EulerSolver(g, dtype=np.float64, device=cuda)
    rg = s.solve([0.5], [2.0], n_iter=6, chunk=3, tol=0.0, verbose=False)
    U = rg.U[0].cpu().numpy()
    dU = ro["U"][0] - om.init_state(om.freestream(0.5, 2.0))
    assert np.max(np.abs(U - ro["U"][0])) / np.max(np.abs(dU)) < 1e-9
    assert abs(rg.cl[0] - ro["cl"][0]) < 1e-10


def test_explicit_rk_fp32_vs_oracle(cuda):
    """dtype=float32: the explicit RK4 + IRS iteration runs in FP32 (residual,
    local time steps, smoothing and stage update, as the reference casts its
    explicit path to the solver dtype, aero2d/euler.py:222-234).  Against the
    FP64 oracle: FP32 rounding, not the FP64 path, and the state holds FP32
    values."""
    g = grid("0012", 33, 25)
    om = EulerModel(g.x, g.y)
    ro = om.solve([0.5], [2.0], n_iter=6, chunk=3, tol=0.0)
    s = EulerSolver(g, dtype=np.float32, device=cuda)
    rg = s.solve([0.5], [2.0], n_iter=6, chunk=3, tol=0.0, verbose=False)
    U = rg.U[0].cpu().numpy()
    dU = ro["U"][0] - om.init_state(om.freestream(0.5, 2.0))
    err = np.max(np.abs(U - ro["U"][0])) / np.max(np.abs(dU))
    assert 1e-9 < err < 1e-4, err
    assert abs(rg.cl[0] - ro["cl"][0]) < 1e-5
    assert np.array_equal(U.astype(np.float32).astype(np.float64), U)


def test_nan_case_is_isolated(cuda):
    """A case whose state is non-finite is rolled back, frozen after five
    failures and flagged non-converged; the other cases are unaffected."""
    g = grid("0012", 33, 25)
    base = EulerSolver(g, dtype=np.float64, device=cuda)
    w = base.freestream(np.array([0.5, 0.6]), np.array([1.0, 2.0]))
    U0 = base.init_state(w)
    U0[1, 0, 5, 3] = float("nan")
    s = ImplicitEuler(base, gmres_restart=20)
    r = s.solve([0.5, 0.6], [1.0, 2.0], n_iter=15, tol=1e-8, verbose=False, U0=U0)
    r_alone = ImplicitEuler(base, gmres_restart=20).solve([0.5], [1.0], n_iter=15, tol=1e-8, verbose=False)
    assert s.frozen[1] and not r.converged[1]
    assert torch.equal(r.U[0], r_alone.U[0])


@pytest.mark.parametrize("levels", [2, 3])
def test_fas_multigrid_vs_oracle(cuda, levels):
    """FAS V-cycles (aero2d/euler.py:349-381) through every level on the device
    against the oracle's cycles: state within 1e-9 of its change, Cl 1e-10."""
    g = grid("0012", 33, 25)
    om = EulerModel(g.x, g.y, mg_levels=levels)
    ro = om.solve([0.7], [1.5], n_iter=6, chunk=3, tol=0.0)
    s = EulerSolver(g, dtype=np.float64, device=cuda, mg_levels=levels)
    rg = s.solve([0.7], [1.5], n_iter=6, chunk=3, tol=0.0, verbose=False)
    U = rg.U[0].cpu().numpy()
    dU = ro["U"][0] - om.init_state(om.freestream(0.7, 1.5))
    assert np.max(np.abs(U - ro["U"][0])) / np.max(np.abs(dU)) < 1e-9
    assert abs(rg.cl[0] - ro["cl"][0]) < 1e-10
    assert np.allclose(rg.res_hist[:, 0], ro["res_hist"][:, 0], rtol=1e-9, atol=0)


def test_explicit_nan_raises(cuda):
    """A non-finite explicit run stops at the end of its chunk and raises
    FloatingPointError (aero2d/euler.py:423-432)."""
    g = grid("0012", 33, 25)
    s = EulerSolver(g, dtype=np.float64, device=cuda)
    w = s.freestream(np.array([0.5]), np.array([1.0]))
    U0 = s.init_state(w)
    U0[0, 0, 5, 3] = float("nan")
    with pytest.raises(FloatingPointError):
        s.solve([0.5], [1.0], n_iter=4, chunk=2, tol=0.0, verbose=False, U0=U0)
