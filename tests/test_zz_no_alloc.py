"""The allocation-free residual entry point (a2d_residual_norms_static).

Callers that cannot call cudaMalloc -- a host application whose memory manager
owns all device memory and does not let a plugin allocate, or a loop that must
not allocate while it runs -- use this entry point instead of a plan.  It
keeps its scratch in a file-scope device array, so this test checks it
against the plan-based a2d_residual on the same inputs, twice in a row (the
second call runs on the array the first one left behind).  The file sorts last
so that a run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from aero2d_b200 import _lib
from aero2d_b200.euler import EulerSolver
from aero2d_b200.plan import DeviceGrid, Plan
from oracle.euler_oracle import EulerModel
from tests.helpers import grid, perturbed_state

pytestmark = pytest.mark.gpu


def test_static_entry_matches_plan_residual_twice(cuda):
    lib = _lib.load()
    g = grid("2412", 65, 33)
    om = EulerModel(g.x, g.y)
    machs, alphas = [0.5, 0.72, 0.35], [2.0, -1.0, 6.0]
    winf = np.stack([om.freestream(m, a) for m, a in zip(machs, alphas)])
    U = np.stack([perturbed_state(om, w, seed=21 + k) for k, w in enumerate(winf)])
    B, ni, nc = U.shape[0], om.ni, om.nc

    # the existing entry point: a plan, reference layout in and out
    dg = DeviceGrid(g, cuda)
    s = EulerSolver(g, dtype=np.float64, device=cuda)
    pl = Plan([dg] * B, winf, s.params(), cuda)
    Ut = torch.as_tensor(U, device=cuda)
    for k in range(B):
        pl.set_vec(_lib.VEC_U, k, Ut[k])
    pl.residual(None)
    R_plan = torch.stack([pl.get_vec(_lib.VEC_R, k) for k in range(B)]).cpu().numpy()

    # the static entry point: the library's internal layout [case][4][nc][ni]
    U_int = Ut.permute(0, 1, 3, 2).contiguous()
    w_dev = torch.as_tensor(winf, device=cuda)
    vol = om.vol
    for call in range(2):
        R_int = torch.full_like(U_int, float("nan"))
        rn = torch.full((B,), float("nan"), dtype=torch.float64, device=cuda)
        stream = torch.cuda.current_stream(cuda).cuda_stream
        _lib.check(lib.a2d_residual_norms_static(dg.ptr, ni, nc + 1, B, U_int.data_ptr(), w_dev.data_ptr(),
                                                 None, None, R_int.data_ptr(), rn.data_ptr(), stream))
        torch.cuda.synchronize()
        R = R_int.permute(0, 1, 3, 2).cpu().numpy()
        for k in range(B):
            circ = om.circulation(U[k], winf[k])
            scale = om.flux_scale(U[k], winf[k], circ)
            assert np.max(np.abs(R[k] - R_plan[k]) / scale) < 1e-12, (call, k)
            rn_ref = np.sqrt(np.mean((R_plan[k][0] / vol) ** 2))
            assert abs(rn.cpu().numpy()[k] - rn_ref) <= 1e-12 * rn_ref, (call, k)


def test_static_entry_rejects_sizes_beyond_its_scratch(cuda):
    lib = _lib.load()
    rc = lib.a2d_residual_norms_static(C.c_void_p(4096), 1024, 65, 1, C.c_void_p(4096), C.c_void_p(4096), None,
                                       None, C.c_void_p(4096), C.c_void_p(4096), None)
    assert rc == _lib.A2D_ERR_ARG
    assert b"static scratch" in lib.a2d_last_error()
    rc = lib.a2d_residual_norms_static(C.c_void_p(4096), 256, 65, 65, C.c_void_p(4096), C.c_void_p(4096), None,
                                       None, C.c_void_p(4096), C.c_void_p(4096), None)
    assert rc == _lib.A2D_ERR_ARG
