"""ctypes binding of the C ABI in include/aero2d_b200.h.

The library is the in-tree build aero2d_b200/libaero2d_b200.so.  There is no
fallback: if the library is missing or cannot be loaded, every solver call
raises ExtensionMissing.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libaero2d_b200.so"

A2D_OK = 0
A2D_ERR_ARG = 1
A2D_ERR_CUDA = 2
A2D_ERR_STATE = 3

A2D_FP64 = 0
A2D_MIXED = 1

# tuning knobs (a2d_plan_set_tuning)
JVP_TILES = {"32x8": 0, "32x16": 1, "64x4": 2, "16x16": 3}
SWEEP_VARIANTS = {"lanes": 0, "rows": 1, "pairs": 2, "halves": 3}

VEC_U, VEC_R, VEC_V, VEC_JV, VEC_DU = 0, 1, 2, 3, 4

# kernels that a2d_time_kernel can time
K_JVP, K_SWEEP, K_SWEEP_FIRST, K_DOTS, K_UPDATE, K_RESIDUAL, K_FACEJAC, K_FACTOR, K_PROJECT = range(9)


class ExtensionMissing(RuntimeError):
    """The CUDA library libaero2d_b200.so is not built or cannot be loaded."""


class A2DError(RuntimeError):
    """A call into libaero2d_b200 returned an error status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"aero2d_b200 status {status}: {message}")
        self.status = status


class Params(C.Structure):
    """Mirror of struct a2d_params."""
    _fields_ = [
        ("gmres_restart", C.c_int),
        ("jacobi_sweeps", C.c_int),
        ("gmres_tol", C.c_double),
        ("cfl0", C.c_double),
        ("cfl_max", C.c_double),
        ("max_update", C.c_double),
        ("tol", C.c_double),
        ("cfl", C.c_double),
        ("irs_eps", C.c_double),
        ("lim_k", C.c_double),
        ("order", C.c_int),
        ("vortex_correction", C.c_int),
        ("precision", C.c_int),
        ("retire", C.c_int),
        ("max_iter", C.c_int),
        ("use_graph", C.c_int),
    ]


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_SZ = C.c_size_t

# name -> (restype, argtypes)
SIGNATURES = {
    "a2d_version": (_I, []),
    "a2d_last_error": (C.c_char_p, []),
    "a2d_default_params": (None, [C.POINTER(Params)]),
    "a2d_metrics_bytes": (_I, [_I, _I, C.POINTER(_SZ)]),
    "a2d_metrics_build": (_I, [_I, _I, _P, _P, _P, _P]),
    "a2d_plan_create": (_I, [_I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_P), C.POINTER(_D),
                             C.POINTER(Params), C.POINTER(_P)]),
    "a2d_plan_workspace_bytes": (_I, [_P, C.POINTER(_SZ)]),
    "a2d_plan_bind": (_I, [_P, _P, _SZ, _P]),
    "a2d_plan_destroy": (_I, [_P]),
    "a2d_plan_ncases": (_I, [_P]),
    "a2d_plan_set_tuning": (_I, [_P, _I, _I, _P]),
    "a2d_plan_get_tuning": (_I, [_P, C.POINTER(_I), C.POINTER(_I)]),
    "a2d_vec_set": (_I, [_P, _I, _I, _P, _P]),
    "a2d_vec_get": (_I, [_P, _I, _I, _P, _P]),
    "a2d_vec_get_prim": (_I, [_P, _I, _I, _P, _P]),
    "a2d_local_dt": (_I, [_P, _I, _P, _P, _P]),
    "a2d_init_freestream": (_I, [_P, _P]),
    "a2d_reset": (_I, [_P, _P]),
    "a2d_residual": (_I, [_P, _P, _P]),
    "a2d_jvp": (_I, [_P, _P]),
    "a2d_forces": (_I, [_P, _P, _P, _P]),
    "a2d_precond_setup": (_I, [_P, _P]),
    "a2d_precond_apply": (_I, [_P, _P]),
    "a2d_set_cfl": (_I, [_P, C.POINTER(_D), _P]),
    "a2d_newton_step": (_I, [_P, _P]),
    "a2d_newton_run": (_I, [_P, _I, C.POINTER(_I), _P]),
    "a2d_case_status": (_I, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_D),
                             C.POINTER(_D), _P]),
    "a2d_case_scalars": (_I, [_P, C.POINTER(_D), _P]),
    "a2d_history": (_I, [_P, _I, C.POINTER(_D), C.POINTER(_D), _P]),
    "a2d_live_count": (_I, [_P, C.POINTER(_I), _P]),
    "a2d_factor_saturations": (_I, [_P, C.POINTER(C.c_ulonglong), _I, _P]),
    "a2d_plan_stats": (_I, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_SZ)]),
    "a2d_time_kernel": (_I, [_P, _I, _I, C.POINTER(C.c_float), _P]),
    "a2d_rk_iterate": (_I, [_P, _I, _P, _P]),
    "a2d_smooth": (_I, [_P, _P]),
    "a2d_set_circulation": (_I, [_P, C.POINTER(_D), _P]),
    "a2d_hllc_flux": (_I, [_I, _P, _P, _P, _P, _P]),
    "a2d_residual_norms_static": (_I, [_P, _I, _I, _I, _P, _P, _P, C.POINTER(Params), _P, _P, _P]),
    "a2d_case_forces": (_I, [_P, C.POINTER(_D), C.POINTER(_D), _P]),
    "a2d_case_restart": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_D), _I, _P]),
    "a2d_case_retire": (_I, [_P, _I, C.POINTER(_I), _P]),
    "a2d_service_create": (_I, [_I, _I, _P, _I, C.POINTER(Params), C.POINTER(_P)]),
    "a2d_service_workspace_bytes": (_I, [_P, C.POINTER(_SZ)]),
    "a2d_service_bind": (_I, [_P, _P, _SZ, _P]),
    "a2d_service_submit": (_I, [_P, _I, C.POINTER(_D), _I, C.POINTER(C.c_longlong)]),
    "a2d_service_step": (_I, [_P, C.POINTER(_I), _P]),
    "a2d_service_poll": (_I, [_P, C.POINTER(C.c_longlong), _I, C.POINTER(_I)]),
    "a2d_service_result": (_I, [_P, C.c_longlong, C.POINTER(_D), C.POINTER(_D), C.POINTER(_I), C.POINTER(_I)]),
    "a2d_service_pending": (_I, [_P, C.POINTER(_I), C.POINTER(_I)]),
    "a2d_service_result_drop": (_I, [_P, C.c_longlong, C.POINTER(_D)]),
    "a2d_service_destroy": (_I, [_P]),
    "a2d_service_stats": (_I, [_P, C.POINTER(_I), C.POINTER(C.c_longlong)]),
    "a2d_service_plan": (_I, [_P, C.POINTER(_P)]),
    "a2d_service_lanes": (_I, [_P, C.POINTER(_I)]),
    "a2d_service_lane": (_I, [_P, _I, C.POINTER(_P), C.POINTER(_I), C.POINTER(_I)]),
    "a2d_service_create_lanes": (_I, [_I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_P), C.POINTER(_I), _I,
                                      C.POINTER(Params), C.POINTER(_P)]),
    "a2d_plan_set_coarse": (_I, [_P, _P]),
    "a2d_case_set_grid": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_P), _P]),
    "a2d_service_create_ragged": (_I, [_I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_P), C.POINTER(_I),
                                       C.POINTER(Params), C.POINTER(_P)]),
    "a2d_service_submit_grid": (_I, [_P, _I, _I, _P, _I, C.POINTER(_D), _I, C.POINTER(C.c_longlong)]),
    "a2d_grid_spacing": (_I, [_I, _D, _D, C.POINTER(_D)]),
    "a2d_grid_build": (_I, [_I, _I, _I, _P, _P, _I, _P, _P, _P, _P]),
}

_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load (once) and return the library; raises ExtensionMissing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise ExtensionMissing(
                f"{LIB_PATH} is not built; run `python -m aero2d_b200.build` (needs nvcc)")
        try:
            lib = C.CDLL(str(LIB_PATH))
        except OSError as e:
            raise ExtensionMissing(f"cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int) -> None:
    if status != A2D_OK:
        msg = load().a2d_last_error()
        raise A2DError(status, msg.decode() if msg else "unknown error")


def default_params() -> Params:
    p = Params()
    load().a2d_default_params(C.byref(p))
    return p
