"""CPU FP64 oracle for the pseudo-transient Newton-Krylov solver of aero2d
(reference: aero2d/implicit.py).

TEST INFRASTRUCTURE ONLY (see oracle/euler_oracle.py): what the CUDA path is
compared against, never part of the product.

Derivatives that the reference takes with jax.jvp / jax.jacfwd are taken here
by the complex step on the oracle residual, which is exact to rounding.
The linear solver restates jax.scipy.sparse.linalg.gmres(..., restart=m,
maxiter=1, solve_method="batched") as called at aero2d/implicit.py:184-185
(jax >= 0.4.30, unpinned in the reference's pyproject.toml:6): left
preconditioning, a skip test against ptol = tol * ||M b||, one cycle of m
Arnoldi steps with classical Gram-Schmidt run twice, breakdown when the new
vector's norm falls to eps times its norm before orthogonalisation, then
x = x0 + V y.  The small least-squares problem min ||beta e1 - H y|| is solved
by Givens rotations (as aero2d/krylov.py:54-85 does) instead of JAX's normal
equations; the two agree in exact arithmetic.  Intermediate Krylov iterates of
the reference are pinned by no test ("parity unpinned" at the GMRES / 4x4
inverse boundary); converged states do not depend on them.
"""
from __future__ import annotations

import numpy as np

from .euler_oracle import (EulerModel, GAMMA, cons_to_prim, farfield_ghost, hllc_flux)

CSTEP = 1e-30        # complex-step size; J v = Im f(U + i h v) / h


def flux_c(UL, UR, S):
    """aero2d/implicit.py:32-33: first-order HLLC from conserved states."""
    return hllc_flux(cons_to_prim(UL), cons_to_prim(UR), S)


def _jac4(f, U):
    """d f / d U for f: (4, n) -> (4, n); returns (n, 4, 4) [out, in]."""
    n = U.shape[1]
    J = np.empty((n, 4, 4))
    for k in range(4):
        d = np.zeros((4, 1), complex)
        d[k] = 1j * CSTEP
        J[:, :, k] = (np.imag(f(U + d)) / CSTEP).T
    return J


def face_jac(UL, UR, S):
    """aero2d/implicit.py:36-41."""
    AL = _jac4(lambda u: flux_c(u, UR, S), UL)
    AR = _jac4(lambda u: flux_c(UL, u, S), UR)
    return AL, AR


def wall_jac(U0, S):
    """aero2d/implicit.py:44-51: mirrored ghost on the left of the wall face."""
    area = np.sqrt(S[0] ** 2 + S[1] ** 2)
    nx, ny = S[0] / area, S[1] / area

    def f(u):
        w = cons_to_prim(u)
        vn = w[1] * nx + w[2] * ny
        g = np.stack([w[0], w[1] - 2 * vn * nx, w[2] - 2 * vn * ny, w[3]])
        return hllc_flux(g, w, S)
    return _jac4(f, U0)


def far_jac(Ui, S, winf, xf, yf, circ):
    """aero2d/implicit.py:54-59 (circulation held fixed)."""
    def f(u):
        w = cons_to_prim(u)
        wb = farfield_ghost(w, S, winf, xf, yf, circ)
        return hllc_flux(w, wb, S)
    return _jac4(f, Ui)


def bmv(A, x):
    return np.einsum("...ab,...b->...a", A, x)


def _norm(x):
    return float(np.sqrt(np.sum(x * x)))


def _safe_normalize(x, thresh=None):
    """Zero vector and zero norm when the norm is at or below thresh (default eps)."""
    n = _norm(x)
    if thresh is None:
        thresh = np.finfo(np.float64).eps
    if n > thresh:
        return x / n, n
    return np.zeros_like(x), 0.0


def gmres_batched(A, M, b, x0, tol, restart):
    """One restart cycle of left-preconditioned GMRES with the semantics of
    jax.scipy.sparse.linalg.gmres(maxiter=1, solve_method="batched", atol=0).
    Returns (x, k) with k the number of Arnoldi vectors used."""
    eps = np.finfo(np.float64).eps
    b_norm = _norm(b)
    if not b_norm > 0:
        return x0, 0
    atol = max(tol * b_norm, 0.0)
    Mb_norm = _norm(M(b))
    ptol = Mb_norm * min(1.0, atol / b_norm)
    r = M(b - A(x0))
    unit, beta = _safe_normalize(r)
    if not beta > ptol:
        return x0, 0
    n = b.size
    V = np.zeros((restart + 1, n))
    V[0] = unit.ravel()
    H = np.zeros((restart + 1, restart))       # column k = Arnoldi step k
    k_used = 0
    for k in range(restart):
        w = M(A(V[k].reshape(b.shape))).ravel()
        w_norm0 = _norm(w)
        h = V[:k + 1] @ w
        w = w - h @ V[:k + 1]
        h2 = V[:k + 1] @ w
        w = w - h2 @ V[:k + 1]
        h = h + h2
        unit_w, wn = _safe_normalize(w, eps * w_norm0)
        V[k + 1] = unit_w
        H[:k + 1, k] = h
        H[k + 1, k] = wn
        k_used = k + 1
        if wn == 0.0:
            break
    y = hessenberg_lstsq(H[:k_used + 1, :k_used], beta)
    x = x0 + (y @ V[:k_used]).reshape(b.shape)
    return x, k_used


def hessenberg_lstsq(H, beta):
    """min || beta e1 - H y || for an upper Hessenberg (k+1, k) H, by Givens rotations."""
    H = np.array(H, dtype=np.float64)
    k = H.shape[1]
    g = np.zeros(k + 1)
    g[0] = beta
    for j in range(k):
        a, c = H[j, j], H[j + 1, j]
        d = np.hypot(a, c)
        if d == 0.0:
            cs, sn = 1.0, 0.0
        else:
            cs, sn = a / d, c / d
        # rotate rows j, j+1 of columns j..k-1 and of g
        hj = H[j, j:].copy()
        hj1 = H[j + 1, j:].copy()
        H[j, j:] = cs * hj + sn * hj1
        H[j + 1, j:] = -sn * hj + cs * hj1
        gj, gj1 = g[j], g[j + 1]
        g[j] = cs * gj + sn * gj1
        g[j + 1] = -sn * gj + cs * gj1
    y = np.zeros(k)
    for i in range(k - 1, -1, -1):
        s = g[i] - H[i, i + 1:k] @ y[i + 1:k]
        y[i] = s / H[i, i] if H[i, i] != 0.0 else 0.0
    return y


class ImplicitModel:
    """Oracle of ImplicitEuler (aero2d/implicit.py:67-253), one case at a time."""

    def __init__(self, base: EulerModel, cfl0=10.0, cfl_max=300.0, gmres_restart=50,
                 gmres_tol=0.01, jacobi_sweeps=4, max_update=0.2):
        self.b = base
        self.cfl0, self.cfl_max = cfl0, cfl_max
        self.restart, self.gtol = gmres_restart, gmres_tol
        self.sweeps = jacobi_sweeps
        self.max_update = max_update

    # -- first-order Jacobian blocks (aero2d/implicit.py:81-110) ------------
    def assemble(self, U, winf, circ, dtau_inv):
        b = self.b
        ni, nc = b.ni, b.nc
        UL = np.roll(U, 1, axis=1).reshape(4, -1)
        UR = U.reshape(4, -1)
        AL, AR = face_jac(UL, UR, b.Si.reshape(2, -1))
        AL, AR = AL.reshape(ni, nc, 4, 4), AR.reshape(ni, nc, 4, 4)
        D = np.roll(AL, -1, axis=0) - AR
        Bip = np.roll(AR, -1, axis=0)
        Bim = -AL
        UL = U[:, :, :-1].reshape(4, -1)
        UR = U[:, :, 1:].reshape(4, -1)
        AL, AR = face_jac(UL, UR, b.Sj[:, :, 1:-1].reshape(2, -1))
        AL, AR = AL.reshape(ni, nc - 1, 4, 4), AR.reshape(ni, nc - 1, 4, 4)
        z = np.zeros((ni, 1, 4, 4))
        D = D + np.concatenate([AL, z], 1) - np.concatenate([z, AR], 1)
        Bjp = np.concatenate([AR, z], 1)
        Bjm = np.concatenate([z, -AL], 1)
        Aw = wall_jac(U[:, :, 0], b.Sj[:, :, 0])
        Af = far_jac(U[:, :, -1], b.Sj[:, :, -1], winf, b.xf, b.yf, circ * b.vortex)
        D[:, 0] += -Aw
        D[:, -1] += Af
        D = D + (b.vol * dtau_inv)[:, :, None, None] * np.eye(4)
        return D, Bim, Bip, Bjm, Bjp

    @staticmethod
    def factor_lines(D, Bjm, Bjp):
        """Block Thomas forward elimination along j (aero2d/implicit.py:112-128)."""
        Dt = np.moveaxis(D, 1, 0)
        Am = np.moveaxis(Bjm, 1, 0)
        Cp = np.moveaxis(Bjp, 1, 0)
        nc = Dt.shape[0]
        inv = np.empty_like(Dt)
        c = np.empty_like(Dt)
        cprev = np.zeros_like(Dt[0])
        for j in range(nc):
            den = Dt[j] - Am[j] @ cprev
            inv[j] = np.linalg.inv(den)
            c[j] = inv[j] @ Cp[j]
            cprev = c[j]
        return inv, c, Am

    @staticmethod
    def solve_lines(fac, r):
        """aero2d/implicit.py:130-148."""
        inv, c, Am = fac
        rt = np.transpose(r, (2, 1, 0))
        nc = rt.shape[0]
        d = np.empty_like(rt)
        dprev = np.zeros_like(rt[0])
        for j in range(nc):
            dprev = bmv(inv[j], rt[j] - bmv(Am[j], dprev))
            d[j] = dprev
        xs = np.empty_like(rt)
        xn = np.zeros_like(rt[0])
        for j in range(nc - 1, -1, -1):
            xn = d[j] - bmv(c[j], xn)
            xs[j] = xn
        return np.transpose(xs, (2, 1, 0))

    def precond(self, fac, Bim, Bip, r):
        """Line Jacobi in i around the j-line solves (aero2d/implicit.py:150-157)."""
        x = self.solve_lines(fac, r)
        for _ in range(self.sweeps - 1):
            xb = np.transpose(x, (1, 2, 0))
            off = bmv(Bim, np.roll(xb, 1, 0)) + bmv(Bip, np.roll(xb, -1, 0))
            x = self.solve_lines(fac, r - np.transpose(off, (2, 0, 1)))
        return x

    # -- residual with the lift-dependent circulation (aero2d/implicit.py:160-167)
    def circ(self, U, winf):
        return self.b.circulation(U, winf)

    def res(self, U, winf):
        return self.b.residual(U, winf, self.circ(U, winf))

    def jvp(self, U, winf, v):
        """d/dU [residual(U, winf, Gamma(U))] . v by complex step."""
        R, _ = self.res(U + 1j * CSTEP * v, winf)
        return np.imag(R) / CSTEP

    def step(self, U, winf, cfl):
        """One pseudo-transient Newton step (aero2d/implicit.py:169-192).
        Returns (U_new, rnorm, omega, info) with info the GMRES vector count."""
        b = self.b
        circ = self.circ(U, winf)
        R, W = self.b.residual(U, winf, circ)
        dt_loc = b.local_dt(W) / b.cfl * cfl
        dtau_inv = 1.0 / dt_loc
        D, Bim, Bip, Bjm, Bjp = self.assemble(U, winf, circ, dtau_inv)
        fac = self.factor_lines(D, Bjm, Bjp)
        diag = (b.vol * dtau_inv)[None]

        def matvec(v):
            return diag * v + self.jvp(U, winf, v)

        def M(r):
            return self.precond(fac, Bim, Bip, r)

        x0 = M(-R)
        dU, k = gmres_batched(matvec, M, -R, x0, self.gtol, self.restart)
        Wn = cons_to_prim(U + dU)
        with np.errstate(invalid="ignore", divide="ignore"):
            rel = max(np.max(np.abs(Wn[0] - W[0]) / W[0]), np.max(np.abs(Wn[3] - W[3]) / W[3]))
            omega = min(1.0, self.max_update / (rel + 1e-30))
            if not np.isfinite(rel):
                omega = np.nan
            Unew = U + omega * dU
        rnorm = np.sqrt(np.mean((R[0] / b.vol) ** 2))
        return Unew, rnorm, omega, k

    def solve(self, machs, alphas, n_iter=200, tol=1e-8, U0=None, callback=None,
              retire=False, verbose=False):
        """Batch solve with the reference's host loop (aero2d/implicit.py:194-253):
        per-case rollback of non-finite steps, freeze after 5 failures, SER CFL.
        retire=True stops stepping each case once it is done (the reference keeps
        stepping every case until all are done)."""
        b = self.b
        machs = np.asarray(machs, np.float64)
        alphas = np.asarray(alphas, np.float64)
        nb = len(machs)
        winf = [b.freestream(machs[k], alphas[k]) for k in range(nb)]
        U = [b.init_state(w) for w in winf] if U0 is None else [np.array(u, np.float64) for u in U0]
        cfl = np.full(nb, self.cfl0)
        hist, clh = [], []
        r0 = None
        fails = np.zeros(nb, int)
        frozen = np.zeros(nb, bool)
        done = np.zeros(nb, bool)
        steps_taken = np.zeros(nb, int)
        self.iterations = 0
        for it in range(n_iter):
            rn = np.full(nb, np.nan)
            om = np.full(nb, np.nan)
            finite = np.zeros(nb, bool)
            Unew = [None] * nb
            for k in range(nb):
                if retire and done[k]:
                    rn[k] = hist[-1][k]
                    om[k] = 1.0
                    finite[k] = np.isfinite(rn[k])
                    Unew[k] = U[k]
                    continue
                Unew[k], rn[k], om[k], _ = self.step(U[k], winf[k], cfl[k])
                steps_taken[k] += 1
                finite[k] = np.isfinite(rn[k]) and np.all(np.isfinite(Unew[k]))
            bad = ~finite | frozen
            fails += ~finite
            frozen |= fails >= 5
            for k in range(nb):
                if not bad[k]:
                    U[k] = Unew[k]
            rn = np.where(finite, rn, np.nan)
            if r0 is None:
                r0 = np.where(np.isfinite(rn), np.maximum(rn, 1e-30), 1.0)
            cl = np.array([b.forces(U[k], winf[k])[0] for k in range(nb)])
            ser = self.cfl0 * (r0 / np.where(np.isfinite(rn), np.maximum(rn, 1e-30), r0))
            cfl_new = np.clip(ser, self.cfl0, self.cfl_max)
            with np.errstate(invalid="ignore"):
                cfl_new = np.where(om < 1.0, np.maximum(cfl_new * 0.5, 1.0), cfl_new)
            cfl_new = np.where(~finite, 1.0, cfl_new)
            if retire:
                cfl = np.where(done, cfl, cfl_new)
            else:
                cfl = cfl_new
            hist.append(rn)
            clh.append(cl)
            self.iterations = it + 1
            if verbose:
                print(f"  it {it + 1:4d} log10(res/res0) {np.log10(rn / r0)}")
            done = done | (rn / r0 < tol) | frozen
            if callback is not None and callback(it + 1, n_iter, np.log10(rn / r0), cl):
                break
            if np.all(done):
                break
        self.cl_history = np.array(clh)
        self.frozen = frozen
        self.steps_taken = steps_taken
        hist = np.array(hist)
        f = [b.forces(U[k], winf[k]) for k in range(nb)]
        last = np.array([h[np.isfinite(h)][-1] if np.any(np.isfinite(h)) else np.nan
                         for h in hist.T])
        converged = (~frozen) & (np.log10(last / r0) < -3)
        return dict(mach=machs, alpha=alphas, cl=np.array([x[0] for x in f]),
                    cd=np.array([x[1] for x in f]), cm=np.array([x[2] for x in f]),
                    cp=np.array([x[3] for x in f]), res_hist=hist, U=np.array(U),
                    converged=converged, r0=r0)
