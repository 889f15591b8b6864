"""O-grids generated on the device, many airfoils at once.

The same hyperbolic marching as `grid.ogrid` (aero2d/grid.py:50-81) runs in
`a2d_grid_build`, one CTA per airfoil, and the metrics follow on the device,
so a request for a new airfoil never waits for the host generator (36-77 ms
per grid in NumPy).  Layers 0 .. nj-2 are bitwise the host generator's; the
outer layer, snapped to a circle with the device's atan2/cos/sin, agrees to a
few units in the last place.  The layer spacings are computed on the host with
the host generator's own `growth_ratio`, so they are the same numbers.
"""
from __future__ import annotations

import ctypes as C
from collections import defaultdict

import numpy as np
import torch

from . import _lib
from .geometry import Airfoil
from .grid import GridError, growth_ratio
from .plan import DeviceGrid, _ptr, device_of, stream_handle


def layer_spacing(nj: int, ds0: float, radius: float) -> np.ndarray:
    """ds0 * r**k for k < nj - 1 with the marching's growth ratio (aero2d/grid.py:52-53)."""
    r = growth_ratio(ds0, radius, nj - 1)
    return ds0 * r ** np.arange(nj - 1)


def ogrid_batch(airfoils: list[Airfoil], nj: int = 64, ds0: float = 2e-3, radius: float = 40.0,
                normal_smoothing: int = 20, device=None) -> list[DeviceGrid]:
    """Device grids (with metrics) for every airfoil; airfoils with the same
    number of contour points share one launch.  Raises GridError naming the
    airfoils whose grid has an inverted cell (aero2d/grid.py:78-80)."""
    dev = device_of(device)
    lib = _lib.load()
    sp = layer_spacing(nj, ds0, radius)
    by_ni: dict[int, list[int]] = defaultdict(list)
    rings = []
    for k, af in enumerate(airfoils):
        ring = np.ascontiguousarray(af.coords()[:-1], np.float64)
        rings.append(ring)
        by_ni[len(ring)].append(k)
    out: list[DeviceGrid | None] = [None] * len(airfoils)
    bad = []
    with torch.cuda.device(dev):
        s = stream_handle(dev)
        for ni, ks in by_ni.items():
            n = len(ks)
            ring_d = torch.as_tensor(np.stack([rings[k] for k in ks]), device=dev)
            sp_d = torch.as_tensor(np.broadcast_to(sp, (n, nj - 1)).copy(), device=dev)
            x = torch.empty((n, ni, nj), dtype=torch.float64, device=dev)
            y = torch.empty_like(x)
            amin = torch.empty(n, dtype=torch.float64, device=dev)
            _lib.check(lib.a2d_grid_build(n, ni, nj, C.c_void_p(_ptr(ring_d)), C.c_void_p(_ptr(sp_d)),
                                          int(normal_smoothing), C.c_void_p(_ptr(x)), C.c_void_p(_ptr(y)),
                                          C.c_void_p(_ptr(amin)), C.c_void_p(s)))
            am = amin.cpu().numpy()
            for q, k in enumerate(ks):
                if not am[q] > 0:
                    bad.append((k, float(am[q])))
                    continue
                out[k] = DeviceGrid(nodes=(x[q], y[q]))
    if bad:
        raise GridError("grids with inverted cells: " + ", ".join(f"airfoil {k} (min area {a:.3e})" for k, a in bad))
    return out
