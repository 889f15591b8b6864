"""Structured O-grid around an airfoil, the mesh input of the Euler path.

Follows aero2d/grid.py:15-81: layers are marched outward along smoothed
normals with geometric spacing growth, each layer is smoothed along itself,
and the last layer is snapped to a circle about (0.5, 0).  Index i runs
counter-clockwise along the contour (periodic), j from the wall outward.  The
steps and their floating-point order are the reference's, so grids are
bit-identical to the reference's for the same airfoil.  Grids are produced on
the host once per airfoil and uploaded to the device once.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geometry import Airfoil


class GridError(RuntimeError):
    """Raised for a grid with a non-positive cell area (aero2d/grid.py:78-80)."""


@dataclass
class OGrid:
    x: np.ndarray   # (ni, nj) node coordinates
    y: np.ndarray

    @property
    def shape(self):
        return self.x.shape

    def cell_areas(self) -> np.ndarray:
        """Cell areas from the two diagonals (aero2d/grid.py:24-31); the node
        loop (i,j)->(i+1,j)->(i+1,j+1)->(i,j+1) runs clockwise."""
        x, y = self.x, self.y
        x1, y1 = np.roll(x, -1, 0), np.roll(y, -1, 0)
        d1x, d1y = x1[:, 1:] - x[:, :-1], y1[:, 1:] - y[:, :-1]
        d2x, d2y = x[:, 1:] - x1[:, :-1], y[:, 1:] - y1[:, :-1]
        return -0.5 * (d1x * d2y - d1y * d2x)


def growth_ratio(ds0: float, total: float, n: int) -> float:
    """r with ds0 * (r**n - 1) / (r - 1) = total, by 200 bisection steps on
    [1 + 1e-9, 2] (aero2d/grid.py:34-41)."""
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if ds0 * (r**n - 1) / (r - 1) < total:
            lo = r
        else:
            hi = r
    return 0.5 * (lo + hi)


def _smooth_ring(a, eps, passes):
    """Periodic Laplacian smoothing along a layer (aero2d/grid.py:44-47)."""
    for _ in range(passes):
        a = a + eps * (np.roll(a, 1, 0) + np.roll(a, -1, 0) - 2 * a)
    return a


def _unit_rows(v):
    return v / np.sqrt(np.sum(v * v, axis=1, keepdims=True))


def ogrid(af: Airfoil, nj: int = 64, ds0: float = 2e-3, radius: float = 40.0,
          normal_smoothing: int = 20) -> OGrid:
    """Hyperbolic-marching O-grid with nj node layers (nc = nj - 1 cells)."""
    ring = af.coords()[:-1].astype(float)       # trailing-edge point once
    ni = len(ring)
    r = growth_ratio(ds0, radius, nj - 1)
    spacing = ds0 * r ** np.arange(nj - 1)
    nodes = np.zeros((ni, nj, 2))
    nodes[:, 0] = ring
    for j in range(1, nj):
        cur = nodes[:, j - 1]
        tangent = _unit_rows(np.roll(cur, -1, 0) - np.roll(cur, 1, 0))
        normal = np.column_stack([tangent[:, 1], -tangent[:, 0]])
        normal = _smooth_ring(normal, 0.25, normal_smoothing if j > 1 else 2)
        normal = _unit_rows(normal)
        frac = j / (nj - 1)
        nodes[:, j] = _smooth_ring(cur + spacing[j - 1] * normal, 0.1 + 0.3 * frac,
                                   2 + int(8 * frac))
    center = np.array([0.5, 0.0])
    rel = nodes[:, -1] - center
    ang = np.arctan2(rel[:, 1], rel[:, 0])
    rmean = np.mean(np.linalg.norm(rel, axis=1))
    nodes[:, -1] = center + rmean * np.column_stack([np.cos(ang), np.sin(ang)])
    g = OGrid(nodes[..., 0], nodes[..., 1])
    a = g.cell_areas()
    if a.min() <= 0:
        raise GridError(f"grid with inverted cells: min area {a.min():.3e}")
    return g
