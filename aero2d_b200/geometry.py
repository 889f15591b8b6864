"""NACA 4-digit airfoil contours, the geometry input of the Euler path.

Follows aero2d/geometry.py:15-87 (Airfoil, _cosine_spacing, naca4): chord 1,
leading edge at (0, 0), contour ordered trailing edge -> upper surface ->
leading edge -> lower surface -> trailing edge with cosine point spacing,
2*n_side - 1 points.  The arithmetic is kept in the reference's order so that
a contour, and the O-grid marched from it, are bit-identical to the
reference's.  `naca4_params` takes the camber, camber position and thickness as
floats, which the random-airfoil workloads need and a 4-digit code string
cannot express.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# x of zero half-thickness of the original (a4 = -0.1015) NACA formula,
# used by the scaled trailing-edge closure (aero2d/geometry.py:46)
NACA_TMR_X0 = 1.008930411365


@dataclass
class Airfoil:
    x: np.ndarray
    y: np.ndarray
    name: str = "airfoil"

    @property
    def n(self) -> int:
        return len(self.x)

    def coords(self) -> np.ndarray:
        return np.column_stack([self.x, self.y])


def cosine_spacing(n: int) -> np.ndarray:
    """Points on [0, 1] clustered at both ends (aero2d/geometry.py:41-43)."""
    return 0.5 * (1.0 - np.cos(np.linspace(0.0, np.pi, n)))


def _half_thickness(xc, t, a4):
    poly = 0.2969 * np.sqrt(xc) - 0.1260 * xc - 0.3516 * xc**2 + 0.2843 * xc**3 + a4 * xc**4
    return 5 * t * poly


def naca4_params(m: float, p: float, t: float, n_side: int = 100, closed_te: bool = True,
                 scaled_te: bool = False, name: str | None = None) -> Airfoil:
    """NACA 4-digit section from float parameters: maximum camber m (chord
    fraction), its position p, thickness t (aero2d/geometry.py:49-87)."""
    xc = cosine_spacing(n_side)
    if scaled_te:
        xs = xc * NACA_TMR_X0
        yt = _half_thickness(xs, t, -0.1015) / NACA_TMR_X0
        yt[-1] = 0.0
        closed_te = True
    else:
        yt = _half_thickness(xc, t, -0.1036 if closed_te else -0.1015)
    yc = np.zeros_like(xc)
    slope = np.zeros_like(xc)
    if m > 0 and p > 0:
        fore = xc < p
        aft = ~fore
        yc[fore] = m / p**2 * (2 * p * xc[fore] - xc[fore] ** 2)
        slope[fore] = 2 * m / p**2 * (p - xc[fore])
        yc[aft] = m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * xc[aft] - xc[aft] ** 2)
        slope[aft] = 2 * m / (1 - p) ** 2 * (p - xc[aft])
    th = np.arctan(slope)
    s, c = np.sin(th), np.cos(th)
    xu, yu = xc - yt * s, yc + yt * c
    xl, yl = xc + yt * s, yc - yt * c
    x = np.concatenate([xu[::-1], xl[1:]])
    y = np.concatenate([yu[::-1], yl[1:]])
    if closed_te:
        y[0] = y[-1] = 0.5 * (y[0] + y[-1])
    if name is None:
        name = f"NACA m={m:.4f} p={p:.3f} t={t:.4f}"
    return Airfoil(x, y, name)


def naca4(code: str, n_side: int = 100, closed_te: bool = True, scaled_te: bool = False) -> Airfoil:
    """NACA 4-digit section from its code string, e.g. "2412"."""
    m = int(code[0]) / 100.0
    p = int(code[1]) / 10.0
    t = int(code[2:]) / 100.0
    return naca4_params(m, p, t, n_side, closed_te, scaled_te, name=f"NACA {code}")
