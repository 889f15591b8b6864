"""CPU FP64 oracle for the Euler residual path of aero2d (reference: aero2d/euler.py).

TEST INFRASTRUCTURE ONLY.  The CUDA path is compared against this module; only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg may import it.  The product (aero2d_b200) never calls it.

It restates, in NumPy, the arithmetic of aero2d/euler.py step by step, keeping
the reference's operation order so that FP64 results agree to rounding.  Every
function accepts complex arrays so that derivatives can be taken by the
complex-step method (d/dh Im f(x + i h v) = J v, exact to rounding): every
comparison therefore looks at the real part only, and jnp.maximum/minimum are
restated with JAX's balanced derivative at ties (0.5/0.5).

Parity status: pinned.  The converged FP64 lift of the reference's own
benchmark (benchmarks/results.json, NACA 0012 128x48, M 0.5 a 2 deg,
Cl = 0.28162520444340794) and the known answers of tests/test_euler.py are
reproduced by tests/test_oracle_pins.py.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GAMMA = 1.4
GM1 = GAMMA - 1.0          # evaluates to 0.3999999999999999, exactly as the reference's GAMMA - 1


def _re(x):
    return np.real(x)


def vmax(a, b):
    """jnp.maximum (aero2d/euler.py:99,178, implicit via JAX): real-part compare,
    balanced tangent at an exact tie."""
    a = np.asarray(a)
    b = np.asarray(b)
    ra, rb = _re(a), _re(b)
    return np.where(ra > rb, a, np.where(ra < rb, b, 0.5 * (a + b)))


def vmin(a, b):
    """jnp.minimum with the same tie rule (aero2d/euler.py:100)."""
    a = np.asarray(a)
    b = np.asarray(b)
    ra, rb = _re(a), _re(b)
    return np.where(ra < rb, a, np.where(ra > rb, b, 0.5 * (a + b)))


# ---------------------------------------------------------------------------
# metrics (aero2d/euler.py:33-60, aero2d/grid.py:24-31)
# ---------------------------------------------------------------------------
@dataclass
class Metrics:
    vol: np.ndarray
    Si: np.ndarray
    Sj: np.ndarray
    xc: np.ndarray
    yc: np.ndarray
    xw: np.ndarray
    yw: np.ndarray


def cell_areas(x, y):
    """aero2d/grid.py:24-31."""
    x1, y1 = np.roll(x, -1, 0), np.roll(y, -1, 0)
    d1x, d1y = x1[:, 1:] - x[:, :-1], y1[:, 1:] - y[:, :-1]
    d2x, d2y = x[:, 1:] - x1[:, :-1], y[:, 1:] - y1[:, :-1]
    return -0.5 * (d1x * d2y - d1y * d2x)


def compute_metrics(x, y) -> Metrics:
    """aero2d/euler.py:44-60."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    vol = cell_areas(x, y)
    dx = x[:, 1:] - x[:, :-1]
    dy = y[:, 1:] - y[:, :-1]
    Si = np.stack([-dy, dx])
    x1, y1 = np.roll(x, -1, 0), np.roll(y, -1, 0)
    dx = x1 - x
    dy = y1 - y
    Sj = np.stack([dy, -dx])
    xc = 0.25 * (x[:, :-1] + x[:, 1:] + x1[:, :-1] + x1[:, 1:])
    yc = 0.25 * (y[:, :-1] + y[:, 1:] + y1[:, :-1] + y1[:, 1:])
    xw = 0.5 * (x[:, 0] + x1[:, 0])
    yw = 0.5 * (y[:, 0] + y1[:, 0])
    return Metrics(vol, Si, Sj, xc, yc, xw, yw)


# ---------------------------------------------------------------------------
# thermodynamics and HLLC (aero2d/euler.py:66-121)
# ---------------------------------------------------------------------------
def cons_to_prim(U):
    rho = U[0]
    u = U[1] / rho
    v = U[2] / rho
    p = GM1 * (U[3] - 0.5 * rho * (u * u + v * v))
    return np.stack([rho, u, v, p])


def prim_to_cons(W):
    rho, u, v, p = W
    return np.stack([rho, rho * u, rho * v, p / GM1 + 0.5 * rho * (u * u + v * v)])


def hllc_flux(WL, WR, S):
    """aero2d/euler.py:79-121: HLLC with Einfeldt/Roe wave speeds, times face area."""
    area = np.sqrt(S[0] ** 2 + S[1] ** 2)
    nx, ny = S[0] / area, S[1] / area
    rL, uL, vL, pL = WL
    rR, uR, vR, pR = WR
    qL = uL * nx + vL * ny
    qR = uR * nx + vR * ny
    cL = np.sqrt(GAMMA * pL / rL)
    cR = np.sqrt(GAMMA * pR / rR)
    EL = pL / GM1 + 0.5 * rL * (uL * uL + vL * vL)
    ER = pR / GM1 + 0.5 * rR * (uR * uR + vR * vR)
    sl, sr = np.sqrt(rL), np.sqrt(rR)
    qt = (sl * qL + sr * qR) / (sl + sr)
    HL = (EL + pL) / rL
    HR = (ER + pR) / rR
    Ht = (sl * HL + sr * HR) / (sl + sr)
    ut = (sl * uL + sr * uR) / (sl + sr)
    vt = (sl * vL + sr * vR) / (sl + sr)
    ct = np.sqrt(vmax(GM1 * (Ht - 0.5 * (ut * ut + vt * vt)), 1e-12))
    SL = vmin(qL - cL, qt - ct)
    SR = vmax(qR + cR, qt + ct)
    SM = (pR - pL + rL * qL * (SL - qL) - rR * qR * (SR - qR)) / (rL * (SL - qL) - rR * (SR - qR))

    def F(r, u, v, p, E, q):
        return np.stack([r * q, r * u * q + p * nx, r * v * q + p * ny, (E + p) * q])

    def Ustar(r, u, v, p, E, q, Sk):
        f = r * (Sk - q) / (Sk - SM)
        return np.stack([f,
                         f * (u + (SM - q) * nx),
                         f * (v + (SM - q) * ny),
                         f * (E / r + (SM - q) * (SM + p / (r * (Sk - q))))])

    with np.errstate(divide="ignore", invalid="ignore"):
        FL = F(rL, uL, vL, pL, EL, qL)
        FR = F(rR, uR, vR, pR, ER, qR)
        UL = np.stack([rL, rL * uL, rL * vL, EL])
        UR = np.stack([rR, rR * uR, rR * vR, ER])
        FsL = FL + SL * (Ustar(rL, uL, vL, pL, EL, qL, SL) - UL)
        FsR = FR + SR * (Ustar(rR, uR, vR, pR, ER, qR, SR) - UR)
    flux = np.where(_re(SL) >= 0, FL,
                    np.where(_re(SM) >= 0, FsL, np.where(_re(SR) > 0, FsR, FR)))
    return flux * area


def van_albada(a, b, eps):
    """Smooth van Albada limiter, the reference default LIMITER="smooth"
    (aero2d/euler.py:124-136)."""
    eps = eps + 1e-20
    return ((b * b + eps) * a + (a * a + eps) * b) / (a * a + b * b + 2 * eps)


# ---------------------------------------------------------------------------
# boundary states (aero2d/euler.py:143-205)
# ---------------------------------------------------------------------------
def wall_ghost(W, Sj0):
    area = np.sqrt(Sj0[0] ** 2 + Sj0[1] ** 2)
    nx, ny = Sj0[0] / area, Sj0[1] / area

    def mirror(Wc):
        r, u, v, p = Wc
        vn = u * nx + v * ny
        return np.stack([r, u - 2 * vn * nx, v - 2 * vn * ny, p])

    return mirror(W[:, :, 1]), mirror(W[:, :, 0])


def farfield_ghost(Wi, Sjf, winf, xf, yf, circ):
    """Riemann-invariant far field with the compressible point-vortex correction
    (aero2d/euler.py:156-205)."""
    area = np.sqrt(Sjf[0] ** 2 + Sjf[1] ** 2)
    nx, ny = Sjf[0] / area, Sjf[1] / area
    rinf, uinf, vinf, pinf = winf
    minf2 = (uinf * uinf + vinf * vinf) / (GAMMA * pinf / rinf)
    dxv, dyv = xf - 0.25, yf
    alpha = np.arctan2(vinf, uinf)
    phi = np.arctan2(dyv, dxv)
    rr = np.sqrt(dxv * dxv + dyv * dyv)
    beta = np.sqrt(max(1 - minf2, 1e-6))
    if minf2 < 1:
        sn = np.sin(phi - alpha)
        fac = circ * beta / (2 * np.pi * rr * (1 - minf2 * (sn * sn)))
    else:
        fac = 0.0 * rr + 0.0 * circ
    ub = uinf + fac * np.sin(phi)
    vb = vinf - fac * np.cos(phi)
    q2inf = uinf * uinf + vinf * vinf
    q2b = ub * ub + vb * vb
    cinf2 = GAMMA * pinf / rinf
    cb2 = vmax(cinf2 + 0.5 * GM1 * (q2inf - q2b), 1e-6)
    pb = pinf * (cb2 / cinf2) ** (GAMMA / GM1)
    rb = rinf * (cb2 / cinf2) ** (1 / GM1)
    r, u, v, p = Wi
    ci = np.sqrt(GAMMA * p / r)
    cb = np.sqrt(GAMMA * pb / rb)
    qni = u * nx + v * ny
    qnb = ub * nx + vb * ny
    Rp = qni + 2 * ci / GM1
    Rm = qnb - 2 * cb / GM1
    qn = 0.5 * (Rp + Rm)
    c = 0.25 * GM1 * (Rp - Rm)
    outflow = _re(qn) > 0
    ut = np.where(outflow, u - qni * nx, ub - qnb * nx)
    vt = np.where(outflow, v - qni * ny, vb - qnb * ny)
    s = np.where(outflow, p / r ** GAMMA, pb / rb ** GAMMA)
    rho = (c * c / (GAMMA * s)) ** (1 / GM1)
    pres = rho * c * c / GAMMA
    Wb = np.stack([rho, ut + qn * nx, vt + qn * ny, pres])
    qnorm_inf = uinf * nx + vinf * ny
    sup_in = (qnorm_inf < 0) & (np.abs(qnorm_inf) > np.sqrt(cinf2))
    sup_out = (_re(qni) > 0) & (_re(qni) > _re(ci))
    ext = np.stack(np.broadcast_arrays(rb, ub, vb, pb))
    Wb = np.where(sup_in, ext, Wb)
    Wb = np.where(sup_out, Wi, Wb)
    return Wb


def _recon(Wm, W0, Wp, Wpp, eps):
    """MUSCL left/right states on the face between W0 and Wp (aero2d/euler.py:211-215)."""
    sL = van_albada(W0 - Wm, Wp - W0, eps)
    sR = van_albada(Wp - W0, Wpp - Wp, eps)
    return W0 + 0.5 * sL, Wp - 0.5 * sR


def _clamp_pos(W):
    """Positivity clamp of face density and pressure at 1e-6 (aero2d/euler.py:274-275)."""
    return np.stack([vmax(W[0], 1e-6), W[1], W[2], vmax(W[3], 1e-6)])


def freestream(mach, alpha_deg):
    """aero2d/euler.py:253-256."""
    a = np.deg2rad(alpha_deg)
    return np.array([1.0, mach * np.cos(a), mach * np.sin(a), 1.0 / GAMMA])


# ---------------------------------------------------------------------------
# the solver model (aero2d/euler.py:218-435), one case at a time
# ---------------------------------------------------------------------------
class EulerModel:
    """Oracle of EulerSolver.  Grid nodes (x, y) of shape (ni, nj); cells (ni, nc)."""

    def __init__(self, x, y, cfl=2.5, irs_eps=0.6, order=2, vortex_correction=True,
                 lim_k=0.02, mg_levels=1):
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        m = compute_metrics(x, y)
        self.m = m
        self.vol, self.Si, self.Sj = m.vol, m.Si, m.Sj
        self.xf = 0.5 * (x[:, -1] + np.roll(x[:, -1], -1))
        self.yf = 0.5 * (y[:, -1] + np.roll(y[:, -1], -1))
        self.xw, self.yw = m.xw, m.yw
        self.cfl, self.irs_eps, self.order, self.lim_k = cfl, irs_eps, order, lim_k
        self.vortex = vortex_correction
        self.ni, self.nc = m.vol.shape
        k = np.arange(self.ni)
        self.irs_den_i = 1 + 2 * irs_eps * (1 - np.cos(2 * np.pi * k / self.ni))
        # FAS multigrid (aero2d/euler.py:241-250): every other node in i and j,
        # first order, the reference's default lim_k
        self.coarse = None
        if mg_levels > 1:
            if self.ni % 2 or self.nc % 2:
                raise ValueError("multigrid needs an even number of cells in i and j")
            self.coarse = EulerModel(x[::2, ::2], y[::2, ::2], cfl, irs_eps, order=1,
                                     vortex_correction=vortex_correction, mg_levels=mg_levels - 1)

    def freestream(self, mach, alpha_deg):
        return freestream(mach, alpha_deg)

    def init_state(self, winf):
        return np.broadcast_to(prim_to_cons(np.asarray(winf)[:, None, None]),
                               (4, self.ni, self.nc)).astype(np.float64)

    def residual(self, U, winf, circ):
        """aero2d/euler.py:259-287 (R is not divided by the cell area)."""
        R, W, _, _ = self.residual_faces(U, winf, circ)
        return R, W

    def flux_scale(self, U, winf, circ):
        """Per-cell sum of |face flux| over the four faces, per component: the
        scale against which a residual's rounding is judged."""
        _, _, Fi, Fj = self.residual_faces(U, winf, circ)
        Fi, Fj = np.abs(np.real(Fi)), np.abs(np.real(Fj))
        return Fi + np.roll(Fi, -1, 1) + Fj[:, :, 1:] + Fj[:, :, :-1]

    def residual_faces(self, U, winf, circ):
        """Residual plus the i-face and j-face fluxes it is formed from."""
        W = cons_to_prim(U)
        mach = np.sqrt(winf[1] ** 2 + winf[2] ** 2)
        scale = np.array([winf[0], mach, mach, winf[3]])
        ls = self.lim_k * scale
        eps = (ls * ls)[:, None, None]
        g2, g1 = wall_ghost(W, self.Sj[:, :, 0])
        Wf = farfield_ghost(W[:, :, -1], self.Sj[:, :, -1], winf, self.xf, self.yf,
                            circ * self.vortex)
        We = np.concatenate([g2[:, :, None], g1[:, :, None], W, Wf[:, :, None], Wf[:, :, None]],
                            axis=2)
        if self.order == 2:
            WL, WR = _recon(We[:, :, 0:-3], We[:, :, 1:-2], We[:, :, 2:-1], We[:, :, 3:], eps)
        else:
            WL, WR = We[:, :, 1:-2], We[:, :, 2:-1]
        Fj = hllc_flux(_clamp_pos(WL), _clamp_pos(WR), self.Sj)
        Wm2, Wm1, Wp1 = np.roll(W, 2, 1), np.roll(W, 1, 1), np.roll(W, -1, 1)
        if self.order == 2:
            WL, WR = _recon(Wm2, Wm1, W, Wp1, eps)
        else:
            WL, WR = Wm1, W
        Fi = hllc_flux(_clamp_pos(WL), _clamp_pos(WR), self.Si)
        R = (np.roll(Fi, -1, 1) - Fi) + (Fj[:, :, 1:] - Fj[:, :, :-1])
        return R, W, Fi, Fj

    def local_dt(self, W):
        """aero2d/euler.py:289-296."""
        r, u, v, p = W
        c = np.sqrt(GAMMA * p / r)
        Si_c = 0.5 * (self.Si + np.roll(self.Si, -1, 1))
        Sj_c = 0.5 * (self.Sj[:, :, 1:] + self.Sj[:, :, :-1])
        li = np.abs(u * Si_c[0] + v * Si_c[1]) + c * np.sqrt(Si_c[0] ** 2 + Si_c[1] ** 2)
        lj = np.abs(u * Sj_c[0] + v * Sj_c[1]) + c * np.sqrt(Sj_c[0] ** 2 + Sj_c[1] ** 2)
        return self.cfl * self.vol / (li + lj)

    def smooth(self, R):
        """Implicit residual smoothing (aero2d/euler.py:298-312): periodic constant
        tridiagonal along i by FFT, then the (-e, 1+2e, -e) system along j."""
        if self.irs_eps <= 0:
            return R
        Rh = np.fft.fft(R, axis=1)
        R = np.real(np.fft.ifft(Rh / self.irs_den_i[None, :, None], axis=1))
        e = self.irs_eps
        n = self.nc
        dl = np.full(n, -e)
        dl[0] = 0.0
        du = np.full(n, -e)
        du[-1] = 0.0
        d = np.full(n, 1 + 2 * e)
        d[0] = d[-1] = 1 + e
        return thomas(dl, d, du, R)

    def wall_pressure(self, W):
        return 1.5 * W[3, :, 0] - 0.5 * W[3, :, 1]

    def forces(self, U, winf):
        """aero2d/euler.py:318-331."""
        W = cons_to_prim(U)
        pw = self.wall_pressure(W)
        S = self.Sj[:, :, 0]
        q = 0.5 * (winf[1] ** 2 + winf[2] ** 2)
        cp = (pw - winf[3]) / q
        fx = -np.sum(cp * S[0])
        fy = -np.sum(cp * S[1])
        mach = np.sqrt(2 * q)
        ca, sa = winf[1] / mach, winf[2] / mach
        cl = fy * ca - fx * sa
        cd = fx * ca + fy * sa
        cm = np.sum(cp * ((self.xw - 0.25) * S[1] - self.yw * S[0]))
        return cl, cd, cm, cp

    def circulation(self, U, winf):
        """Gamma = 1/2 Cl M (aero2d/euler.py:401-403, aero2d/implicit.py:160-164)."""
        cl = self.forces(U, winf)[0]
        return 0.5 * cl * np.sqrt(winf[1] ** 2 + winf[2] ** 2)

    def iterate(self, U, winf, circ, P=None):
        """One 4-stage RK iteration with local time step and IRS, P the FAS
        forcing term (aero2d/euler.py:334-346)."""
        U0 = U
        W = cons_to_prim(U)
        dt = self.local_dt(W)
        for a in (0.25, 1 / 3, 0.5, 1.0):
            R, _ = self.residual(U, winf, circ)
            if P is not None:
                R = R + P
            R = self.smooth(R)
            U = U0 - a * (dt / self.vol)[None] * R
        res = np.sqrt(np.mean(((U[0] - U0[0]) / dt) ** 2))
        return U, res

    @staticmethod
    def sum4(a):
        """Sum over the four fine cells of each coarse cell (aero2d/euler.py:350-352)."""
        return a[..., 0::2, 0::2] + a[..., 1::2, 0::2] + a[..., 0::2, 1::2] + a[..., 1::2, 1::2]

    @staticmethod
    def prolong(d):
        """Bilinear correction, weights 3/4 and 1/4, periodic in i and held at
        the ends in j (aero2d/euler.py:354-366)."""
        e = 0.75 * d + 0.25 * np.roll(d, 1, axis=1)
        o = 0.75 * d + 0.25 * np.roll(d, -1, axis=1)
        d = np.stack([e, o], axis=2).reshape(d.shape[0], -1, d.shape[2])
        dm = np.concatenate([d[:, :, :1], d[:, :, :-1]], axis=2)
        dp = np.concatenate([d[:, :, 1:], d[:, :, -1:]], axis=2)
        e = 0.75 * d + 0.25 * dm
        o = 0.75 * d + 0.25 * dp
        return np.stack([e, o], axis=3).reshape(d.shape[0], d.shape[1], -1)

    def cycle(self, U, winf, circ, P=None):
        """One FAS V-cycle (aero2d/euler.py:368-381); without a coarse level, one iteration."""
        U, res = self.iterate(U, winf, circ, P)
        if self.coarse is not None:
            cs = self.coarse
            R, _ = self.residual(U, winf, circ)
            if P is not None:
                R = R + P
            Uc0 = self.sum4(U * self.vol[None]) / self.sum4(self.vol)[None]
            Rc, _ = cs.residual(Uc0, winf, circ)
            Pc = self.sum4(R) - Rc
            Uc, _ = cs.cycle(Uc0, winf, circ, Pc)
            U = U + self.prolong(Uc - Uc0)
            U, _ = self.iterate(U, winf, circ, P)
        return U, res

    def solve(self, machs, alphas, n_iter=4000, chunk=200, tol=1e-7, U0=None,
              tol_cl=2e-5, tol_cd=2e-6):
        """Explicit batch solve with the reference's chunked stop tests
        (aero2d/euler.py:386-435).  Returns a dict of per-case arrays."""
        machs = np.asarray(machs, np.float64)
        alphas = np.asarray(alphas, np.float64)
        B = len(machs)
        winf = [self.freestream(machs[b], alphas[b]) for b in range(B)]
        U = [self.init_state(w) for w in winf] if U0 is None else [np.array(u) for u in U0]
        circ = [0.0] * B
        hist, clh, cdh = [], [], []
        res0 = None
        iterations = 0
        for it in range(0, n_iter, chunk):
            res = np.zeros(B)
            for b in range(B):
                for _ in range(chunk):
                    U[b], r = self.cycle(U[b], winf[b], circ[b])
                    circ[b] = self.circulation(U[b], winf[b])
                res[b] = r
            iterations = it + chunk
            if res0 is None:
                res0 = res
            f = [self.forces(U[b], winf[b]) for b in range(B)]
            cl = np.array([x[0] for x in f])
            cd = np.array([x[1] for x in f])
            hist.append(res)
            clh.append(cl)
            cdh.append(cd)
            if not np.all(np.isfinite(res)):
                break
            if np.all(res / res0 < tol):
                break
            if len(clh) > 2 and np.all(np.abs(clh[-1] - clh[-2]) < tol_cl) \
                    and np.all(np.abs(cdh[-1] - cdh[-2]) < tol_cd):
                break
        if not all(np.all(np.isfinite(u)) for u in U):
            raise FloatingPointError("diverged (NaN)")
        f = [self.forces(U[b], winf[b]) for b in range(B)]
        return dict(mach=machs, alpha=alphas, cl=np.array([x[0] for x in f]),
                    cd=np.array([x[1] for x in f]), cm=np.array([x[2] for x in f]),
                    cp=np.array([x[3] for x in f]), res_hist=np.array(hist), U=np.array(U),
                    iterations=iterations, cl_history=np.array(clh))


def thomas(dl, d, du, R):
    """Solve the constant tridiagonal system along the last axis of R
    (jax.lax.linalg.tridiagonal_solve semantics: dl[0] = du[-1] = 0)."""
    n = len(d)
    cp = np.empty(n)
    dp = np.empty(R.shape)
    cp[0] = du[0] / d[0]
    dp[..., 0] = R[..., 0] / d[0]
    for k in range(1, n):
        den = d[k] - dl[k] * cp[k - 1]
        cp[k] = du[k] / den
        dp[..., k] = (R[..., k] - dl[k] * dp[..., k - 1]) / den
    x = np.empty(R.shape)
    x[..., -1] = dp[..., -1]
    for k in range(n - 2, -1, -1):
        x[..., k] = dp[..., k] - cp[k] * x[..., k + 1]
    return x
