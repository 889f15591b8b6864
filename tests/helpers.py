"""Shared builders for the parity tests: grids, seeded perturbed states and
decoding of the device metrics blob."""
from __future__ import annotations

import numpy as np

from aero2d_b200.geometry import naca4, naca4_params
from aero2d_b200.grid import ogrid
from oracle.euler_oracle import EulerModel, prim_to_cons


def grid(code="0012", n_side=33, nj=25, ds0=2e-3, radius=40.0):
    return ogrid(naca4(code, n_side), nj=nj, ds0=ds0, radius=radius)


def perturbed_state(model: EulerModel, winf, seed=0, amp=0.02):
    """Freestream plus a smooth seeded perturbation of every primitive
    (positive density and pressure), a state far from any fixed point."""
    rng = np.random.default_rng(seed)
    ni, nc = model.ni, model.nc
    ii = np.arange(ni)[:, None] / ni
    jj = np.arange(nc)[None, :] / nc
    W = np.empty((4, ni, nc))
    base = np.asarray(winf, float)
    for k in range(4):
        a, b, c = rng.uniform(-1, 1, 3)
        f = a * np.sin(2 * np.pi * (ii + c)) * np.cos(np.pi * jj * (1 + b)) + 0.3 * rng.standard_normal((ni, nc))
        scale = max(abs(base[k]), 0.3)
        W[k] = base[k] + amp * scale * f
    return prim_to_cons(W)


def transonic_draw(n=8, seed=2025):
    """The transonic cases: random NACA 4-digit sections (m ~ U[0, 0.06],
    p ~ U[0.2, 0.6], t ~ U[0.08, 0.16], 193 points per side), each on its own
    384 x 96 O-grid (ds0 1e-3, radius 20; sections whose grid folds are redrawn),
    then M ~ U[0.70, 0.80] and alpha ~ U[0, 3] deg, from default_rng(seed).
    Returns (params [(m, p, t)], grids, machs, alphas, redrawn)."""
    from aero2d_b200.grid import GridError
    rng = np.random.default_rng(seed)
    params, grids, rejected = [], [], 0
    while len(grids) < n:
        m, p, t = rng.uniform(0, 0.06), rng.uniform(0.2, 0.6), rng.uniform(0.08, 0.16)
        try:
            grids.append(ogrid(naca4_params(m, p, t, 193), nj=97, ds0=1e-3, radius=20.0))
            params.append((float(m), float(p), float(t)))
        except GridError:
            rejected += 1
    machs, alphas = rng.uniform(0.70, 0.80, n), rng.uniform(0.0, 3.0, n)
    return params, grids, machs, alphas, rejected


def decode_metrics(blob: np.ndarray, ni: int, nc: int):
    """Split the device metrics blob (uint8) into its FP64 arrays in the
    reference layout: vol (ni, nc), Si (2, ni, nc), Sj (2, ni, nc+1), xf, yf, xw, yw."""
    N = ni * nc
    nd = 5 * N + 6 * ni
    d = blob[: nd * 8].view(np.float64)
    vol = d[:N].reshape(nc, ni).T
    Si = d[N:3 * N].reshape(2, nc, ni).transpose(0, 2, 1)
    Sj = d[3 * N:3 * N + 2 * (N + ni)].reshape(2, nc + 1, ni).transpose(0, 2, 1)
    o = 3 * N + 2 * (N + ni)
    xf, yf, xw, yw = (d[o + q * ni: o + (q + 1) * ni] for q in range(4))
    return vol, Si, Sj, xf, yf, xw, yw


__all__ = ["grid", "perturbed_state", "transonic_draw", "decode_metrics", "naca4", "naca4_params", "ogrid"]
