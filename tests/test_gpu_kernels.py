"""Parity of the CUDA kernels with the FP64 oracle, operation by operation,
through the C ABI (aero2d_b200.plan.Plan wraps include/aero2d_b200.h).

Tolerances: FP64 residuals agree per cell to 1e-12 of the cell's summed face
flux magnitude (the residual is a difference of O(1) fluxes); derivatives to
1e-10 of the largest entry; mixed-precision JVP to 2e-5."""
import numpy as np
import pytest
import torch

from aero2d_b200 import _lib
from aero2d_b200.euler import EulerSolver, compute_metrics, hllc_flux
from aero2d_b200.plan import DeviceGrid, Plan
from oracle.euler_oracle import EulerModel, hllc_flux as hllc_oracle
from oracle.implicit_oracle import ImplicitModel
from tests.helpers import decode_metrics, grid, perturbed_state

pytestmark = pytest.mark.gpu


def _plan(g, winf_list, cuda, **over):
    dg = DeviceGrid(g, cuda)
    s = EulerSolver(g, dtype=np.float64, device=cuda)
    return Plan([dg] * len(winf_list), np.array(winf_list), s.params(**over), cuda), dg


@pytest.mark.parametrize("code,ns,nj", [("0012", 33, 25), ("2412", 65, 33)])
def test_metrics_bit_exact(cuda, code, ns, nj):
    g = grid(code, ns, nj)
    dg = DeviceGrid(g, cuda)
    torch.cuda.synchronize()
    vol, Si, Sj, xf, yf, xw, yw = decode_metrics(dg.metrics.cpu().numpy(), dg.ni, dg.nc)
    m = compute_metrics(g)
    assert np.array_equal(vol, m.vol)
    assert np.array_equal(Si, m.Si)
    assert np.array_equal(Sj, m.Sj)
    assert np.array_equal(xw, m.xw) and np.array_equal(yw, m.yw)
    assert np.array_equal(xf, 0.5 * (g.x[:, -1] + np.roll(g.x[:, -1], -1)))
    assert np.array_equal(yf, 0.5 * (g.y[:, -1] + np.roll(g.y[:, -1], -1)))


def test_point_flux_consistency(cuda):
    """F(W, W) is the physical flux (tests/test_euler.py:15-24)."""
    W = np.array([[1.2], [0.3], [-0.1], [0.9]])
    S = np.array([[0.6], [0.8]])
    F = hllc_flux(W, W, S)
    r, u, v, p = W[:, 0]
    q = u * 0.6 + v * 0.8
    E = p / 0.4 + 0.5 * r * (u * u + v * v)
    ref = np.array([r * q, r * u * q + p * 0.6, r * v * q + p * 0.8, (E + p) * q])
    assert np.allclose(F[:, 0], ref, rtol=1e-12)


def test_point_flux_vs_oracle(cuda):
    rng = np.random.default_rng(3)
    n = 4096
    WL = np.stack([rng.uniform(0.5, 1.5, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(0.3, 1.2, n)])
    WR = np.stack([rng.uniform(0.5, 1.5, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(0.3, 1.2, n)])
    S = rng.uniform(-1, 1, (2, n))
    F = hllc_flux(WL, WR, S)
    Fo = hllc_oracle(WL, WR, S)
    assert np.max(np.abs(F - Fo) / (np.abs(Fo) + 1.0)) < 1e-13


@pytest.mark.parametrize("code,ns,nj,mach,alpha", [("0012", 33, 25, 0.5, 3.0), ("2412", 65, 33, 0.75, -2.0),
                                                   ("0012", 33, 25, 1.3, 1.0)])
@pytest.mark.parametrize("circ_mode", ["from_U", "given"])
def test_residual_fp64_per_cell(cuda, code, ns, nj, mach, alpha, circ_mode):
    g = grid(code, ns, nj)
    om = EulerModel(g.x, g.y)
    w = om.freestream(mach, alpha)
    U = perturbed_state(om, w, seed=7)
    circ = om.circulation(U, w) if circ_mode == "from_U" else 0.137
    Ro, _ = om.residual(U, w, circ)
    scale = om.flux_scale(U, w, circ)
    pl, _ = _plan(g, [w], cuda)
    pl.set_vec(_lib.VEC_U, 0, torch.as_tensor(U))
    c = None if circ_mode == "from_U" else torch.full((1,), circ, dtype=torch.float64, device=cuda)
    pl.residual(c)
    R = pl.get_vec(_lib.VEC_R, 0).cpu().numpy()
    err = np.abs(R - Ro) / scale
    assert err.max() < 1e-12, err.max()


def test_residual_at_converged_state(cuda, converged_0012, known_answers):
    """At the oracle's converged FP64 state of the reference benchmark the CUDA
    residual is at the rounding floor and the forces reproduce the published Cl."""
    g = grid("0012", 65, 49, 2e-3, 40.0)
    om = EulerModel(g.x, g.y)
    w = om.freestream(0.5, 2.0)
    U = converged_0012["U_m05_a2"]
    pl, _ = _plan(g, [w], cuda)
    pl.set_vec(_lib.VEC_U, 0, torch.as_tensor(U))
    pl.residual(None)
    R = pl.get_vec(_lib.VEC_R, 0).cpu().numpy()
    circ = om.circulation(U, w)
    scale = om.flux_scale(U, w, circ)
    assert np.max(np.abs(R) / scale) < 1e-11
    coef, _ = pl.forces()
    cl = float(coef[0, 0])
    assert abs(cl - known_answers["results_json"]["cases"][0]["cl_fp64"]) < 1e-9


@pytest.mark.parametrize("prec,tol", [(_lib.A2D_FP64, 1e-10), (_lib.A2D_MIXED, 2e-5)])
def test_jvp_vs_complex_step(cuda, prec, tol):
    g = grid("2412", 65, 33)
    om = EulerModel(g.x, g.y)
    im = ImplicitModel(om)
    w = om.freestream(0.6, 2.5)
    U = perturbed_state(om, w, seed=11)
    v = np.random.default_rng(5).standard_normal(U.shape)
    Jv = im.jvp(U, w, v)
    pl, _ = _plan(g, [w], cuda, precision=prec)
    pl.set_vec(_lib.VEC_U, 0, torch.as_tensor(U))
    pl.set_vec(_lib.VEC_V, 0, torch.as_tensor(v))
    pl.jvp()
    J = pl.get_vec(_lib.VEC_JV, 0).cpu().numpy()
    for k in range(4):
        err = np.max(np.abs(J[k] - Jv[k])) / np.max(np.abs(Jv[k]))
        assert err < tol, (k, err)


# ni = 64 fills two 32-line groups; ni = 80 leaves a partial third group.
# Tolerances: FP64 factors 1e-10 relative; mixed path (FP32 pivot inverses,
# FP16 sweep factors) 5e-3.
@pytest.mark.parametrize("ns,nj,sweeps,mixed", [(33, 25, 4, False), (41, 17, 1, False), (41, 17, 2, False),
                                                (41, 17, 4, False), (41, 17, 4, True), (33, 25, 3, True)])
def test_precond_vs_oracle(cuda, ns, nj, sweeps, mixed):
    g = grid("0012", ns, nj)
    om = EulerModel(g.x, g.y)
    im = ImplicitModel(om, jacobi_sweeps=sweeps)
    w = om.freestream(0.55, 1.0)
    U = perturbed_state(om, w, seed=2, amp=0.01)
    cfl = 37.0
    circ = im.circ(U, w)
    R, W = om.residual(U, w, circ)
    dtau_inv = 1.0 / (om.local_dt(W) / om.cfl * cfl)
    D, Bim, Bip, Bjm, Bjp = im.assemble(U, w, circ, dtau_inv)
    fac = im.factor_lines(D, Bjm, Bjp)
    r = np.random.default_rng(9).standard_normal(U.shape)
    xo = im.precond(fac, Bim, Bip, r)
    over = {"jacobi_sweeps": sweeps}
    if mixed:
        over["precision"] = _lib.A2D_MIXED
    pl, _ = _plan(g, [w], cuda, **over)
    pl.set_vec(_lib.VEC_U, 0, torch.as_tensor(U))
    pl.set_cfl([cfl])
    pl.precond_setup()
    pl.set_vec(_lib.VEC_V, 0, torch.as_tensor(r))
    pl.precond_apply()
    x = pl.get_vec(_lib.VEC_JV, 0).cpu().numpy()
    assert np.max(np.abs(x - xo)) / np.max(np.abs(xo)) < (5e-3 if mixed else 1e-10)


def test_smoothing_vs_fft(cuda):
    g = grid("0012", 33, 25)
    om = EulerModel(g.x, g.y)
    s = EulerSolver(g, dtype=np.float64, device=cuda)
    R = np.random.default_rng(4).standard_normal((4, om.ni, om.nc))
    Ro = om.smooth(R)
    Rs = s.smooth(torch.as_tensor(R)).cpu().numpy()
    assert np.max(np.abs(Rs - Ro)) / np.max(np.abs(Ro)) < 1e-12


@pytest.mark.parametrize("mixed", [False, True])
def test_precond_and_step_repeatable(cuda, mixed):
    """The line preconditioner and a whole Newton step are pure functions of
    their inputs: on the 256 x 64 benchmark grid with 16 cases and 4 sweeps,
    two inputs applied alternately give bitwise the same output every time, and
    a Newton step repeated from the same state gives the same update.  (Large
    enough that the sweep kernels fill the GPU; small grids hide scheduling
    effects.)"""
    from aero2d_b200.geometry import naca4
    from aero2d_b200.grid import ogrid
    g = ogrid(naca4("2412", 129), nj=65, ds0=2e-3, radius=20.0)
    rng = np.random.default_rng(5)
    B = 16
    base = EulerSolver(g, dtype=np.float32 if mixed else np.float64, device=cuda)
    w = base.freestream(rng.uniform(0.3, 0.75, B), rng.uniform(-4, 8, B))
    pl = Plan([base.dgrid] * B, w, base.params(gmres_restart=30, jacobi_sweeps=4), cuda)
    pl.init_freestream()
    for _ in range(3):
        pl.newton_step()
    shape = (B, 4, g.shape[0], g.shape[1] - 1)
    Va = torch.as_tensor(rng.standard_normal(shape), device=cuda)
    Vb = torch.as_tensor(rng.standard_normal(shape), device=cuda)
    pl.precond_setup()
    outs = {0: [], 1: []}
    for r in range(12):
        pl.set_batch(_lib.VEC_V, Va if r % 2 == 0 else Vb)
        pl.precond_apply()
        outs[r % 2].append(pl.get_batch(_lib.VEC_JV))
    for o in outs.values():
        assert all(torch.equal(x, o[0]) for x in o[1:])
    U = pl.get_batch(_lib.VEC_U).clone()
    dus = []
    for _ in range(4):
        pl.set_batch(_lib.VEC_U, U)
        pl.reset()
        pl.newton_step()
        dus.append(pl.get_batch(_lib.VEC_DU))
    assert all(torch.equal(d, dus[0]) for d in dus[1:])
    pl.close()
