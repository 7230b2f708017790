"""The C-ABI library without a GPU: it loads, exports every symbol include/v3dba.h declares, and
its host-side argument validation rejects bad problems before touching the device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from v3dsfmtoolkit_b200 import capi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    syms = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            syms |= set(re.findall(r"\b(v3dba_\w+)\s*\(", txt))
    return syms


def test_library_exports_every_declared_symbol():
    lib = capi.library()
    declared = _declared_symbols()
    assert declared, "no declarations found"
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(capi.EXPORTS) <= declared


def test_dims_and_defaults():
    assert capi.dims(0, 0) == (6, 0)
    assert capi.dims(1, 4) == (6, 7)
    assert capi.dims(1, 3) == (6, 5)
    assert capi.dims(1, -1) == (6, 0)
    assert capi.dims(2, 4) == (13, 0)
    assert capi.dims(2, 1) == (7, 0)
    o = capi.default_options()
    assert o.tau == 1e-3 and o.max_iterations == 50
    assert o.gradient_threshold == 1e-10 and o.update_threshold == 1e-10
    assert capi.dims(capi.MODEL_STEREO, 0) == (6, 0)
    with pytest.raises(capi.V3dbaError):
        capi.dims(4, 0)
    with pytest.raises(capi.V3dbaError):
        capi.dims(1, 5)


def _problem(sc, **over):
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (sc.K, sc.R, sc.T, sc.X, sc.meas)]
    view = np.ascontiguousarray(sc.view, dtype=np.int32)
    point = np.ascontiguousarray(sc.point, dtype=np.int32)
    d = np.zeros(4)
    p = capi.Problem(sc.model, sc.mode, sc.n_cams, sc.n_points, sc.n_obs, sc.inlier_threshold,
                     capi._d(arrs[0]), capi._d(arrs[1]), capi._d(arrs[2]), capi._d(d), capi._d(arrs[3]),
                     capi._d(arrs[4]), view.ctypes.data_as(capi._ip), point.ctypes.data_as(capi._ip))
    for k, v in over.items():
        setattr(p, k, v)
    return p, (arrs, view, point, d)


def test_create_rejects_bad_arguments_before_device_use():
    lib = capi.library()
    h = C.c_void_p()
    assert lib.v3dba_create(None, C.byref(h)) == capi.ERR_INVALID_ARGUMENT
    sc = scenes.circle_scene(n_cams=4, n_points=30, seed=1)
    p, keep = _problem(sc, model=7)
    assert lib.v3dba_create(C.byref(p), C.byref(h)) == capi.ERR_INVALID_ARGUMENT
    p, keep = _problem(sc, n_cameras=-1)
    assert lib.v3dba_create(C.byref(p), C.byref(h)) == capi.ERR_INVALID_ARGUMENT
    # a view index out of range is an input error
    bad = sc.copy()
    bad.view[3] = sc.n_cams
    p, keep = _problem(bad)
    assert lib.v3dba_create(C.byref(p), C.byref(h)) == capi.ERR_INVALID_INPUT
    # NaN in the parameters is an input error
    bad = sc.copy()
    bad.X[2, 1] = np.nan
    p, keep = _problem(bad)
    assert lib.v3dba_create(C.byref(p), C.byref(h)) == capi.ERR_INVALID_INPUT
    bad = sc.copy()
    bad.meas[0, 0] = np.inf
    p, keep = _problem(bad)
    assert lib.v3dba_create(C.byref(p), C.byref(h)) == capi.ERR_INVALID_INPUT
    p, keep = _problem(sc, inlier_threshold=0.0)
    assert lib.v3dba_create(C.byref(p), C.byref(h)) == capi.ERR_INVALID_INPUT
    assert not h.value


def test_error_strings():
    lib = capi.library()
    for code in range(0, 8):
        assert lib.v3dba_error_string(code)
