"""Host-side checks without a GPU: the grid generator against the reference's
grids, and the C ABI library (loads, exports every declared symbol, plans are
laid out on the host)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from aero2d_b200 import _lib
from aero2d_b200.geometry import naca4, naca4_params
from aero2d_b200.grid import GridError, ogrid
from tests.conftest import ROOT
from tests.golden.make_golden import GRIDS


@pytest.mark.parametrize("key", list(GRIDS))
def test_grid_bit_identical_to_reference(ref_grids, key):
    code, ns, nj, ds0, rad = GRIDS[key]
    g = ogrid(naca4(code, ns), nj=nj, ds0=ds0, radius=rad)
    assert np.array_equal(g.x, ref_grids[f"{key}_x"])
    assert np.array_equal(g.y, ref_grids[f"{key}_y"])


def test_float_naca_params_match_code():
    a = naca4("2412", 65)
    b = naca4_params(0.02, 0.4, 0.12, 65)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


def test_inverted_grid_raises():
    with pytest.raises(GridError):
        ogrid(naca4("6412", 193), nj=97, ds0=1e-3, radius=20.0)


def _declared_symbols():
    hdr = (ROOT / "include" / "aero2d_b200.h").read_text()
    return sorted(set(re.findall(r"\b(a2d_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared_symbols()
    assert len(names) > 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_params_struct_matches_header():
    hdr = (ROOT / "include" / "aero2d_b200.h").read_text()
    body = hdr[hdr.index("typedef struct a2d_params"):hdr.index("} a2d_params;")]
    fields = re.findall(r"^\s*(?:int|double)\s+(\w+);", body, re.M)
    assert fields == [f for f, _ in _lib.Params._fields_]


def test_plan_layout_on_host():
    """Plans are created and sized on the host; no device call is made."""
    lib = _lib.load()
    n = C.c_size_t()
    _lib.check(lib.a2d_metrics_bytes(256, 65, C.byref(n)))
    assert n.value > 0
    B = 3
    ni = (C.c_int * B)(256, 192, 128)
    nc = (C.c_int * B)(64, 48, 32)
    fake = (C.c_void_p * B)(4096, 8192, 16384)     # never dereferenced before bind
    winf = (C.c_double * (4 * B))(*([1.0, 0.5, 0.0, 1 / 1.4] * B))
    p = _lib.default_params()
    h = C.c_void_p()
    _lib.check(lib.a2d_plan_create(B, ni, nc, fake, winf, C.byref(p), C.byref(h)))
    _lib.check(lib.a2d_plan_workspace_bytes(h, C.byref(n)))
    cells = 256 * 64 + 192 * 48 + 128 * 32
    assert n.value > 8 * 4 * cells * (p.gmres_restart + 1)
    assert lib.a2d_plan_ncases(h) == B
    assert lib.a2d_residual(h, None, None) == _lib.A2D_ERR_STATE     # unbound plan
    _lib.check(lib.a2d_plan_destroy(h))


def test_plan_rejects_bad_params():
    lib = _lib.load()
    p = _lib.default_params()
    p.gmres_restart = 100
    h = C.c_void_p()
    ni = (C.c_int * 1)(64)
    nc = (C.c_int * 1)(24)
    m = (C.c_void_p * 1)(4096)
    w = (C.c_double * 4)(1.0, 0.5, 0.0, 1 / 1.4)
    assert lib.a2d_plan_create(1, ni, nc, m, w, C.byref(p), C.byref(h)) == _lib.A2D_ERR_ARG
    assert b"gmres_restart" in lib.a2d_last_error()


@pytest.mark.parametrize("nj,ds0,radius", [(25, 2e-3, 40.0), (49, 2e-3, 40.0), (65, 2e-3, 20.0), (97, 1e-3, 20.0)])
def test_device_grid_spacing_matches_host(nj, ds0, radius):
    """The C ABI's layer spacings (host C++) against the host generator's."""
    from aero2d_b200.gridgen import layer_spacing
    out = np.empty(nj - 1)
    _lib.check(_lib.load().a2d_grid_spacing(nj, ds0, radius, out.ctypes.data_as(C.POINTER(C.c_double))))
    ref = layer_spacing(nj, ds0, radius)
    assert np.max(np.abs(out - ref) / ref) <= 2.3e-16


def test_repanel_matches_reference():
    """Arc-length spline re-panelling (aero2d/geometry.py:320-391), bitwise the
    reference's own output on the same contours (tests/golden/ref_repanel.npz):
    NACA sections at the polar levels' resolutions, a blunt trailing edge, a
    contour with corners, two-halves input, a mirrored unnormalised contour and
    the viscous spacing."""
    from aero2d_b200.geometry import Airfoil, repanel
    from tests.golden.make_golden import REPANEL_KW
    d = np.load(ROOT / "tests" / "golden" / "ref_repanel.npz")
    for key, kw in REPANEL_KW.items():
        out = repanel(Airfoil(d[f"{key}_in_x"], d[f"{key}_in_y"]), **kw)
        assert np.array_equal(out.x, d[f"{key}_out_x"]) and np.array_equal(out.y, d[f"{key}_out_y"]), key


def _fake_plan(lib, precision, B=2):
    ni = (C.c_int * B)(*([64] * B))
    nc = (C.c_int * B)(*([24] * B))
    fake = (C.c_void_p * B)(*([4096] * B))     # never dereferenced before bind
    winf = (C.c_double * (4 * B))(*([1.0, 0.5, 0.0, 1 / 1.4] * B))
    p = _lib.default_params()
    p.precision = precision
    h = C.c_void_p()
    _lib.check(lib.a2d_plan_create(B, ni, nc, fake, winf, C.byref(p), C.byref(h)))
    return h


def test_plan_starting_configuration_on_host():
    """A new mixed plan starts with 32x16 JVP tiles and the halves sweep; an FP64 plan
    starts on the lanes sweep and refuses rows and halves (host-only: nothing is bound)."""
    lib = _lib.load()
    t, v = C.c_int(), C.c_int()
    hm = _fake_plan(lib, _lib.A2D_MIXED)
    _lib.check(lib.a2d_plan_get_tuning(hm, C.byref(t), C.byref(v)))
    assert (t.value, v.value) == (_lib.JVP_TILES["32x16"], _lib.SWEEP_VARIANTS["halves"])
    h64 = _fake_plan(lib, _lib.A2D_FP64)
    _lib.check(lib.a2d_plan_get_tuning(h64, C.byref(t), C.byref(v)))
    assert v.value == _lib.SWEEP_VARIANTS["lanes"]
    for v in ("rows", "halves"):
        assert lib.a2d_plan_set_tuning(h64, 0, _lib.SWEEP_VARIANTS[v], None) == _lib.A2D_ERR_ARG
        assert b"mixed-precision plans only" in lib.a2d_last_error()
    _lib.check(lib.a2d_plan_set_tuning(h64, 0, _lib.SWEEP_VARIANTS["pairs"], None))
    for h in (hm, h64):
        _lib.check(lib.a2d_plan_destroy(h))


def test_service_lanes_layout_on_host():
    """Slot q of each class goes to lane q mod lanes; the lane count is capped by the
    largest class; the workspace holds every lane's plan (host-only)."""
    from aero2d_b200.service import default_lanes
    lib = _lib.load()
    ni = (C.c_int * 2)(64, 96)
    nc = (C.c_int * 2)(24, 32)
    fake = (C.c_void_p * 2)(4096, 8192)
    slots = (C.c_int * 2)(5, 2)
    p = _lib.default_params()
    p.precision = _lib.A2D_MIXED
    h = C.c_void_p()
    _lib.check(lib.a2d_service_create_lanes(2, ni, nc, fake, slots, 3, C.byref(p), C.byref(h)))
    nl = C.c_int()
    _lib.check(lib.a2d_service_lanes(h, C.byref(nl)))
    assert nl.value == 3
    lanes, total = [], 0
    for lane in range(3):
        n = C.c_int()
        _lib.check(lib.a2d_service_lane(h, lane, None, C.byref(n), None))
        ids = (C.c_int * n.value)()
        _lib.check(lib.a2d_service_lane(h, lane, None, None, ids))
        lanes.append(list(ids))
    # class 0 owns slots 0..4, class 1 slots 5..6
    assert lanes == [[0, 3, 5], [1, 4, 6], [2]]
    ws = C.c_size_t()
    _lib.check(lib.a2d_service_workspace_bytes(h, C.byref(ws)))
    assert ws.value > 0
    _lib.check(lib.a2d_service_destroy(h))
    h2 = C.c_void_p()
    _lib.check(lib.a2d_service_create_lanes(2, ni, nc, fake, slots, 8, C.byref(p), C.byref(h2)))
    _lib.check(lib.a2d_service_lanes(h2, C.byref(nl)))
    assert nl.value == 5          # at most the largest class's slot count
    _lib.check(lib.a2d_service_destroy(h2))
    assert [default_lanes(c) for c in ([64], [16], [8], [32], [394, 176, 99, 44])] == [4, 1, 1, 2, 4]
