"""Pseudo-transient Newton-Krylov Euler solver, B200 implementation.

Drop-in for aero2d/implicit.py: ImplicitEuler(base, cfl0, cfl_max,
gmres_restart, gmres_tol, jacobi_sweeps, max_update) with step() and the
batched solve(machs, alphas, n_iter, tol, verbose, U0, callback).  Each Newton
step solves (V/dtau + dR/dU) dU = -R(U) by one restarted-GMRES cycle,
left-preconditioned by the first-order block-tridiagonal line solver with
line-Jacobi coupling in i; the Jacobian-vector product is the hand-written
linearisation of the second-order residual, including the derivative of the
far-field vortex through the circulation.  The whole step, and the per-case
rollback / freeze / SER-CFL logic of the reference's host loop, run on the
device; one CUDA graph replays a step.

Differences from the reference that a caller can observe:
  * cases retire individually once their residual has dropped by `tol`
    (the reference keeps stepping every case until all are done); set
    retire=False to step them in lockstep as the reference does;
  * dtype=float32 selects the mixed-precision mode: the JVP, the face
    Jacobians and the Krylov basis are FP32 while the residual, the line
    factorisation, Gram-Schmidt, norms and the state update stay FP64, so the
    converged answer is the FP64 one (the reference's all-FP32 mode stalls
    near a 1e-6 residual drop).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .euler import EulerResult, EulerSolver, cons_to_prim
from .plan import Plan


class ImplicitEuler:
    def __init__(self, base: EulerSolver, cfl0: float = 10.0, cfl_max: float = 300.0,
                 gmres_restart: int = 50, gmres_tol: float = 0.01, jacobi_sweeps: int = 4,
                 max_update: float = 0.2, retire: bool = True, use_graph: bool = True):
        self.b = base
        self.cfl0, self.cfl_max = cfl0, cfl_max
        self.restart, self.gtol = gmres_restart, gmres_tol
        self.sweeps = jacobi_sweeps
        self.max_update = max_update
        self.retire = retire
        self.use_graph = use_graph
        self.plan = None

    def params(self, tol: float, n_iter: int) -> _lib.Params:
        return self.b.params(gmres_restart=int(self.restart), jacobi_sweeps=int(self.sweeps),
                             gmres_tol=float(self.gtol), cfl0=float(self.cfl0),
                             cfl_max=float(self.cfl_max), max_update=float(self.max_update),
                             tol=float(tol), retire=int(bool(self.retire)),
                             max_iter=int(max(1, n_iter)), use_graph=int(bool(self.use_graph)))

    # ------------------------------------------------------------------
    def step(self, U, winf, circ=None, cfl=None):
        """One Newton step of one case (aero2d/implicit.py:169-192).
        Returns (U_new, rnorm, omega); circ is recomputed from U as the
        reference does, so the argument is accepted and ignored."""
        b = self.b
        cfl = self.cfl0 if cfl is None else float(cfl)
        pl = Plan([b.dgrid], np.asarray(winf, np.float64).reshape(1, 4), self.params(0.0, 2), b.device)
        pl.set_vec(_lib.VEC_U, 0, U)
        pl.reset()
        pl.set_cfl([cfl])
        pl.newton_step()
        sc = pl.scalars()[0]
        rn, omega, committed = float(sc[0]), float(sc[1]), bool(sc[7])
        if committed:
            Unew = pl.get_vec(_lib.VEC_U, 0)
        else:   # a failed step: the device kept U; hand back the non-finite candidate as the reference does
            dU = pl.get_vec(_lib.VEC_DU, 0)
            Unew = torch.as_tensor(U, dtype=torch.float64, device=b.device) + omega * dU
        return Unew, rn, omega

    def solve(self, machs, alphas, n_iter=200, tol=1e-8, verbose=True, U0=None, callback=None):
        """Batch solve (aero2d/implicit.py:194-253).  A case that fails a step
        is rolled back and retried with CFL 1; after 5 failures it is frozen and
        flagged non-converged without affecting the others.

        callback(it, n_iter, log10_res, cl) is called after every step; if it
        returns True the run stops with the current state."""
        b = self.b
        machs = np.atleast_1d(np.asarray(machs, np.float64))
        alphas = np.atleast_1d(np.asarray(alphas, np.float64))
        if machs.shape != alphas.shape:
            raise ValueError("machs and alphas must have the same length")
        B = len(machs)
        winf = b.freestream(machs, alphas)
        pl = Plan([b.dgrid] * B, winf, self.params(tol, n_iter), b.device)
        self.plan = pl
        if U0 is None:
            pl.init_freestream()
        else:
            pl.set_batch(_lib.VEC_U, torch.as_tensor(U0, dtype=torch.float64, device=b.device))
            pl.reset()
        self.iterations = 0
        if callback is None and not verbose:
            self.iterations = pl.newton_run(n_iter)
        else:
            for it in range(n_iter):
                pl.newton_step()
                self.iterations = it + 1
                nsteps, done, frozen, lastrn, r0 = pl.status()
                rn_h, cl_h = pl.history(max(1, int(nsteps.max())))
                rn = np.array([rn_h[nsteps[k] - 1, k] if nsteps[k] else np.nan for k in range(B)])
                cl = np.array([cl_h[nsteps[k] - 1, k] if nsteps[k] else np.nan for k in range(B)])
                with np.errstate(divide="ignore", invalid="ignore"):
                    lr = np.log10(rn / r0)
                if verbose and (it % 5 == 0 or it == n_iter - 1):
                    print(f"  it {it + 1:4d}  log10(res/res0) {np.array2string(lr, precision=2)}"
                          f"  Cl {np.array2string(cl, precision=4)}")
                if callback is not None and callback(it + 1, n_iter, lr, cl):
                    break
                if self.retire:
                    if np.all(done | frozen):
                        break
                elif np.all(done):
                    break
        return self._result(pl, machs, alphas)

    def _result(self, pl: Plan, machs, alphas) -> EulerResult:
        B = pl.B
        nsteps, done, frozen, lastrn, r0 = pl.status()
        steps = int(nsteps.max()) if B else 0
        rn_h, cl_h = pl.history(steps)
        # rows past a retired case's last step repeat its last value
        for k in range(B):
            if 0 < nsteps[k] < steps:
                rn_h[nsteps[k]:, k] = rn_h[nsteps[k] - 1, k]
                cl_h[nsteps[k]:, k] = cl_h[nsteps[k] - 1, k]
        self.cl_history = cl_h
        self.frozen = frozen
        self.done = done
        self.steps_taken = nsteps
        coef, cps = pl.forces()
        c = coef.cpu().numpy()
        U = pl.get_batch(_lib.VEC_U)
        res = EulerResult(machs, alphas, c[:, 0], c[:, 1], c[:, 2], torch.stack(cps).cpu().numpy(),
                          rn_h, U)
        with np.errstate(divide="ignore", invalid="ignore"):
            res.converged = (~frozen) & (np.log10(lastrn / r0) < -3)
        return res
