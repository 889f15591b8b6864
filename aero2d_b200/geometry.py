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


# ---------------------------------------------------------------------------
# Re-panelling of an arbitrary contour (aero2d/geometry.py:244-391), the step the
# reference's polar scenario applies to every input before marching its grid
# (aero2d/core.py:236).  The floating-point steps are the reference's, in its
# order and through the same SciPy spline constructors, so the re-panelled
# contour, and the grid marched from it, match the reference's.
# ---------------------------------------------------------------------------
def _chord_frame(x, y):
    """Chord from the trailing-edge midpoint to the farthest contour point:
    translated to put that point at the origin, scaled to unit chord and rotated
    onto the x axis (aero2d/geometry.py:268-279)."""
    te = 0.5 * np.array([x[0] + x[-1], y[0] + y[-1]])
    far = int(np.argmax(np.hypot(x - te[0], y - te[1])))
    le = np.array([x[far], y[far]])
    chord = te - le
    length = np.hypot(*chord)
    rot = np.arctan2(chord[1], chord[0])
    cr, sr = np.cos(-rot), np.sin(-rot)
    xs, ys = (x - le[0]) / length, (y - le[1]) / length
    return xs * cr - ys * sr, xs * sr + ys * cr


def normalize(af: Airfoil) -> Airfoil:
    """The package's contour convention (aero2d/geometry.py:244-265): trailing
    edge -> upper -> leading edge -> lower -> trailing edge, counter-clockwise,
    chord 1 from (0, 0).  Two-halves (Lednicer) input is joined; contours that
    already span [0, 1] with the trailing edge on y = 0 keep their frame."""
    x, y = np.asarray(af.x, float), np.asarray(af.y, float)
    if x[0] < 0.5 and np.any(np.diff(x) < -0.5):
        k = int(np.argmax(np.diff(x) < -0.5)) + 1
        dup = np.isclose(x[k:][0], x[:k][0])
        yk0 = np.isclose(af.x[k:][0], af.x[:k][0])
        x = np.concatenate([x[:k][::-1], x[k:][1:] if dup else x[k:]])
        y = np.concatenate([af.y[:k][::-1], af.y[k:][1:] if yk0 else af.y[k:]])
    framed = abs(x.min()) < 2e-3 and abs(x.max() - 1) < 2e-3 and abs(0.5 * (y[0] + y[-1])) < 2e-3
    if not framed:
        x, y = _chord_frame(x, y)
    if 0.5 * np.sum(x[:-1] * y[1:] - x[1:] * y[:-1]) < 0:
        x, y = x[::-1], y[::-1]
    return Airfoil(x, y, af.name)


def corner_indices(x, y, angle: float = 30.0) -> np.ndarray:
    """Interior points where the contour direction turns by more than `angle`
    degrees (aero2d/geometry.py:282-288)."""
    d = np.column_stack([np.diff(x), np.diff(y)])
    d /= np.maximum(np.linalg.norm(d, axis=1), 1e-300)[:, None]
    cosang = np.clip(np.sum(d[:-1] * d[1:], 1), -1.0, 1.0)
    return np.where(np.degrees(np.arccos(cosang)) > angle)[0] + 1


class ContourSpline:
    """x(s), y(s) by arc length, one cubic spline per smooth piece between
    corners (not-a-knot; pieces of fewer than four points interpolated at the
    highest degree they allow), as aero2d/geometry.py:291-317 builds it."""

    def __init__(self, s, x, y, cuts):
        from scipy.interpolate import CubicSpline, make_interp_spline
        self.bounds = np.concatenate([[0], np.asarray(cuts, int), [len(s) - 1]])
        self.sb = s[self.bounds]
        self.pieces = []
        for lo, hi in zip(self.bounds[:-1], self.bounds[1:]):
            sp, xp, yp = s[lo:hi + 1], x[lo:hi + 1], y[lo:hi + 1]
            if len(sp) >= 4:
                self.pieces.append((CubicSpline(sp, xp), CubicSpline(sp, yp)))
            else:
                deg = len(sp) - 1
                self.pieces.append((make_interp_spline(sp, xp, k=deg), make_interp_spline(sp, yp, k=deg)))

    def __call__(self, st):
        st = np.asarray(st, float)
        piece = np.clip(np.searchsorted(self.sb, st, side="right") - 1, 0, len(self.pieces) - 1)
        xo, yo = np.empty_like(st), np.empty_like(st)
        for k, (fx, fy) in enumerate(self.pieces):
            sel = piece == k
            if sel.any():
                xo[sel], yo[sel] = fx(st[sel]), fy(st[sel])
        return xo, yo


def repanel(af: Airfoil, n_side: int = 100, spacing: str = "cosine", keep_frame: bool = False,
            corner_angle: float = 30.0, te_merge: float = 2e-3) -> Airfoil:
    """n_side points per side along an arc-length spline of the contour
    (aero2d/geometry.py:320-391): cosine clustering to both edges, or "viscous"
    (strong at the leading edge, mild at the trailing edge); corners sharper than
    corner_angle stay nodes (the nearest node moves onto the corner, its six
    neighbours on each side follow with a linear fall-off), except the two corners
    of a blunt trailing-edge base; the result is normalised (or, with keep_frame,
    only made counter-clockwise), a trailing-edge gap below te_merge chords is
    closed at its midpoint and a larger one closed by a segment."""
    x, y = np.asarray(af.x, float), np.asarray(af.y, float)
    keep = np.concatenate([[True], np.hypot(np.diff(x), np.diff(y)) > 1e-10])
    x, y = x[keep], y[keep]
    s = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(x), np.diff(y)))])
    cuts = corner_indices(x, y, corner_angle) if corner_angle else np.array([], int)
    # corners within 0.5 % chord of both contour ends are a blunt base: spline through it
    near_end = 0.005 * max(float(np.ptp(x)), 1e-12)
    at_start = (np.hypot(x[cuts] - x[0], y[cuts] - y[0]) <= near_end) & (s[cuts] < 0.5 * s[-1])
    at_end = (np.hypot(x[cuts] - x[-1], y[cuts] - y[-1]) <= near_end) & (s[cuts] > 0.5 * s[-1])
    if at_start.any() and at_end.any():
        cuts = cuts[~(at_start | at_end)]
    spline = ContourSpline(s, x, y, cuts)
    probe = np.linspace(0, s[-1], 20001)
    s_le = probe[np.argmin(spline(probe)[0])]
    if spacing == "viscous":
        u = np.linspace(0, 1, n_side)
        wgt = 0.55
        g = wgt * (1 - np.cos(0.5 * np.pi * u)) + (1 - wgt) * 0.5 * (1 - np.cos(np.pi * u))
        first = s_le * (1 - g[::-1])
        second = s_le + (s[-1] - s_le) * g
    else:
        b = np.linspace(0, np.pi, n_side)
        first = s_le * 0.5 * (1 - np.cos(b))
        second = s_le + (s[-1] - s_le) * 0.5 * (1 - np.cos(b))
    st = np.concatenate([first, second[1:]])
    spread = 6
    fixed = set()
    for sc in s[cuts]:
        k = int(np.argmin(np.abs(st[1:-1] - sc))) + 1
        shift = sc - st[k]
        for j in range(-spread, spread + 1):
            i = k + j
            if 0 < i < len(st) - 1 and i not in fixed:
                st[i] += shift * (1.0 - abs(j) / (spread + 1))
        st[k] = sc
        fixed.add(k)
    st = np.sort(st)
    xo, yo = spline(st)
    out = Airfoil(xo, yo, af.name)
    if keep_frame:
        if 0.5 * np.sum(out.x[:-1] * out.y[1:] - out.x[1:] * out.y[:-1]) < 0:
            out = Airfoil(out.x[::-1].copy(), out.y[::-1].copy(), af.name)
    else:
        out = normalize(out)
    gap = np.hypot(out.x[0] - out.x[-1], out.y[0] - out.y[-1])
    if gap <= te_merge * max(float(np.ptp(out.x)), 1e-12):
        out.x[0] = out.x[-1] = 0.5 * (out.x[0] + out.x[-1])
        out.y[0] = out.y[-1] = 0.5 * (out.y[0] + out.y[-1])
    else:
        out = Airfoil(np.r_[out.x, out.x[0]], np.r_[out.y, out.y[0]], out.name)
    return out
