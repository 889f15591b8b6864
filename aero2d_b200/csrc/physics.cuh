// Point-wise physics of the finite-volume Euler residual: thermodynamics, the
// HLLC face flux, the smooth van Albada MUSCL reconstruction and the wall and
// far-field ghost states.  Written once over a scalar type S that is either a
// plain real (double / float) or a dual number, so that the residual, its
// Jacobian-vector product and the 4x4 face Jacobians share one arithmetic.
//
// Operation order follows aero2d/euler.py so that FP64 values agree with the
// reference to rounding.  Constants that the reference spells as GAMMA - 1 are
// the double 1.4 - 1.0 = 0.3999999999999999, as Python evaluates them.
#pragma once
#include "dual.cuh"

namespace a2d {

constexpr double kGamma = 1.4;
constexpr double kGm1 = kGamma - 1.0;
constexpr double kGammaOverGm1 = kGamma / kGm1;   // pressure exponent of the isentrope
constexpr double kInvGm1 = 1.0 / kGm1;             // density exponent of the isentrope
constexpr double kHalfGm1 = 0.5 * kGm1;
constexpr double kQuarterGm1 = 0.25 * kGm1;
constexpr double kPi = 3.141592653589793;

template <typename S>
struct State4 {
  S c[4];
};

// conserved (rho, rho u, rho v, E) -> primitive (rho, u, v, p)   [euler.py:66-71]
template <typename S, typename T>
__device__ __forceinline__ State4<S> cons_to_prim(const State4<S>& U) {
  State4<S> W;
  const S rho = U.c[0];
  const S u = U.c[1] / rho;
  const S v = U.c[2] / rho;
  W.c[0] = rho;
  W.c[1] = u;
  W.c[2] = v;
  W.c[3] = T(kGm1) * (U.c[3] - T(0.5) * rho * (u * u + v * v));
  return W;
}

// HLLC flux through a face with area vector (sx, sy), already times length [euler.py:79-121]
template <typename S, typename T>
__device__ __forceinline__ State4<S> hllc(const State4<S>& WL, const State4<S>& WR, T sx, T sy) {
  const T area = dsqrt(sx * sx + sy * sy);
  const T nx = sx / area, ny = sy / area;
  const S rL = WL.c[0], uL = WL.c[1], vL = WL.c[2], pL = WL.c[3];
  const S rR = WR.c[0], uR = WR.c[1], vR = WR.c[2], pR = WR.c[3];
  const S qL = uL * nx + vL * ny;
  const S qR = uR * nx + vR * ny;
  const S cL = dsqrt(T(kGamma) * pL / rL);
  const S cR = dsqrt(T(kGamma) * pR / rR);
  const S EL = pL / T(kGm1) + T(0.5) * rL * (uL * uL + vL * vL);
  const S ER = pR / T(kGm1) + T(0.5) * rR * (uR * uR + vR * vR);
  const S sl = dsqrt(rL), sr = dsqrt(rR);
  const S ssum = sl + sr;
  const S qt = (sl * qL + sr * qR) / ssum;
  const S HL = (EL + pL) / rL;
  const S HR = (ER + pR) / rR;
  const S Ht = (sl * HL + sr * HR) / ssum;
  const S ut = (sl * uL + sr * uR) / ssum;
  const S vt = (sl * vL + sr * vR) / ssum;
  const S ct = dsqrt(vmax(T(kGm1) * (Ht - T(0.5) * (ut * ut + vt * vt)), T(1e-12)));
  const S SL = vmin(qL - cL, qt - ct);
  const S SR = vmax(qR + cR, qt + ct);
  const S SM = (pR - pL + rL * qL * (SL - qL) - rR * qR * (SR - qR)) /
               (rL * (SL - qL) - rR * (SR - qR));
  State4<S> F;
  const T sLv = val(SL), sMv = val(SM), sRv = val(SR);
  if (sLv >= T(0) || !(sMv >= T(0) || sRv > T(0))) {
    // supersonic to either side: the one-sided physical flux
    const bool left = sLv >= T(0);
    const S r = left ? rL : rR, u = left ? uL : uR, v = left ? vL : vR;
    const S p = left ? pL : pR, E = left ? EL : ER, q = left ? qL : qR;
    F.c[0] = r * q;
    F.c[1] = r * u * q + p * nx;
    F.c[2] = r * v * q + p * ny;
    F.c[3] = (E + p) * q;
  } else {
    // star region on the side of the contact
    const bool left = sMv >= T(0);
    const S r = left ? rL : rR, u = left ? uL : uR, v = left ? vL : vR;
    const S p = left ? pL : pR, E = left ? EL : ER, q = left ? qL : qR;
    const S Sk = left ? SL : SR;
    const S f = r * (Sk - q) / (Sk - SM);
    const S dq = SM - q;
    const S us0 = f;
    const S us1 = f * (u + dq * nx);
    const S us2 = f * (v + dq * ny);
    const S us3 = f * (E / r + dq * (SM + p / (r * (Sk - q))));
    const S f0 = r * q;
    const S f1 = r * u * q + p * nx;
    const S f2 = r * v * q + p * ny;
    const S f3 = (E + p) * q;
    F.c[0] = f0 + Sk * (us0 - r);
    F.c[1] = f1 + Sk * (us1 - r * u);
    F.c[2] = f2 + Sk * (us2 - r * v);
    F.c[3] = f3 + Sk * (us3 - E);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) F.c[k] = F.c[k] * area;
  return F;
}

// smooth van Albada limiter (LIMITER = "smooth", euler.py:127-136)
template <typename S, typename T>
__device__ __forceinline__ S van_albada(const S& a, const S& b, T eps) {
  const T e = eps + T(1e-20);
  return ((b * b + e) * a + (a * a + e) * b) / (a * a + b * b + T(2) * e);
}

// MUSCL: left/right states on the face between W0 and Wp (euler.py:211-215),
// followed by the positivity clamp of density and pressure (euler.py:274-275)
template <typename S, typename T>
__device__ __forceinline__ void recon(const State4<S>& Wm, const State4<S>& W0, const State4<S>& Wp,
                                      const State4<S>& Wpp, const T eps[4], bool second_order,
                                      State4<S>& WL, State4<S>& WR) {
  if (second_order) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const S sLk = van_albada(W0.c[k] - Wm.c[k], Wp.c[k] - W0.c[k], eps[k]);
      const S sRk = van_albada(Wp.c[k] - W0.c[k], Wpp.c[k] - Wp.c[k], eps[k]);
      WL.c[k] = W0.c[k] + T(0.5) * sLk;
      WR.c[k] = Wp.c[k] - T(0.5) * sRk;
    }
  } else {
    WL = W0;
    WR = Wp;
  }
  WL.c[0] = vmax(WL.c[0], T(1e-6));
  WL.c[3] = vmax(WL.c[3], T(1e-6));
  WR.c[0] = vmax(WR.c[0], T(1e-6));
  WR.c[3] = vmax(WR.c[3], T(1e-6));
}

// mirrored wall ghost of one cell state (euler.py:143-153)
template <typename S, typename T>
__device__ __forceinline__ State4<S> wall_mirror(const State4<S>& W, T sx, T sy) {
  const T area = dsqrt(sx * sx + sy * sy);
  const T nx = sx / area, ny = sy / area;
  const S vn = W.c[1] * nx + W.c[2] * ny;
  State4<S> G;
  G.c[0] = W.c[0];
  G.c[1] = W.c[1] - T(2) * vn * nx;
  G.c[2] = W.c[2] - T(2) * vn * ny;
  G.c[3] = W.c[3];
  return G;
}

// Freestream primitives of one case (euler.py:253-256): rho=1, |V|=M, p=1/gamma.
struct Freestream {
  double r, u, v, p;
};

// Riemann-invariant far-field ghost with the compressible point-vortex
// correction about (0.25, 0) (euler.py:156-205).  Circ is the circulation
// Gamma; it is a dual number when its derivative is carried.
template <typename S, typename T>
__device__ __forceinline__ State4<S> farfield_ghost(const State4<S>& Wi, T sx, T sy, T rinf, T uinf,
                                                    T vinf, T pinf, T xf, T yf, const S& circ) {
  const T area = dsqrt(sx * sx + sy * sy);
  const T nx = sx / area, ny = sy / area;
  const T minf2 = (uinf * uinf + vinf * vinf) / (T(kGamma) * pinf / rinf);
  const T dxv = xf - T(0.25), dyv = yf;
  const T alpha = atan2(vinf, uinf);
  const T phi = atan2(dyv, dxv);
  const T rr = dsqrt(dxv * dxv + dyv * dyv);
  const T beta = dsqrt(vmax(T(1) - minf2, T(1e-6)));
  const T sphi = sin(phi), cphi = cos(phi);
  S fac;
  if (minf2 < T(1)) {
    const T s = sin(phi - alpha);
    fac = circ * beta / (T(2) * T(kPi) * rr * (T(1) - minf2 * (s * s)));
  } else {
    fac = circ * T(0);
  }
  const S ub = uinf + fac * sphi;
  const S vb = vinf - fac * cphi;
  const T q2inf = uinf * uinf + vinf * vinf;
  const S q2b = ub * ub + vb * vb;
  const T cinf2 = T(kGamma) * pinf / rinf;
  const S cb2 = vmax(cinf2 + T(kHalfGm1) * (q2inf - q2b), T(1e-6));
  const S ratio = cb2 / cinf2;
  const S pb = pinf * dpow(ratio, T(kGammaOverGm1));
  const S rb = rinf * dpow(ratio, T(kInvGm1));
  const S r = Wi.c[0], u = Wi.c[1], v = Wi.c[2], p = Wi.c[3];
  const S ci = dsqrt(T(kGamma) * p / r);
  const S cb = dsqrt(T(kGamma) * pb / rb);
  const S qni = u * nx + v * ny;
  const S qnb = ub * nx + vb * ny;
  const S Rp = qni + T(2) * ci / T(kGm1);
  const S Rm = qnb - T(2) * cb / T(kGm1);
  const S qn = T(0.5) * (Rp + Rm);
  const S c = T(kQuarterGm1) * (Rp - Rm);
  const bool outflow = val(qn) > T(0);
  const S ut = outflow ? u - qni * nx : ub - qnb * nx;
  const S vt = outflow ? v - qni * ny : vb - qnb * ny;
  const S s = outflow ? p / dpow(r, T(kGamma)) : pb / dpow(rb, T(kGamma));
  const S rho = dpow(c * c / (T(kGamma) * s), T(kInvGm1));
  const S pres = rho * c * c / T(kGamma);
  State4<S> Wb;
  Wb.c[0] = rho;
  Wb.c[1] = ut + qn * nx;
  Wb.c[2] = vt + qn * ny;
  Wb.c[3] = pres;
  const T qnorm_inf = uinf * nx + vinf * ny;
  const bool sup_in = (qnorm_inf < T(0)) && (fabs(qnorm_inf) > dsqrt(cinf2));
  const bool sup_out = (val(qni) > T(0)) && (val(qni) > val(ci));
  if (sup_in) {
    Wb.c[0] = rb;
    Wb.c[1] = ub;
    Wb.c[2] = vb;
    Wb.c[3] = pb;
  }
  if (sup_out) Wb = Wi;
  return Wb;
}

}  // namespace a2d
