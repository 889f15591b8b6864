"""aero2d_b200: the batched 2-D Euler solver path of aero2d on B200 GPUs.

Modules mirror the reference package layout for this path:
  geometry  NACA 4-digit contours          (aero2d/geometry.py)
  grid      structured O-grid generator    (aero2d/grid.py)
  euler     residual, forces, RK4 + IRS    (aero2d/euler.py)
  implicit  Newton-Krylov solver           (aero2d/implicit.py)
  replicas  one process per GPU: case shards, job time, result gathering
The numerics run in libaero2d_b200.so (hand-written sm_100a CUDA) through the
C ABI of include/aero2d_b200.h.
"""
from .geometry import Airfoil, naca4, naca4_params  # noqa: F401
from .grid import GridError, OGrid, ogrid  # noqa: F401

__version__ = "0.1.0"
