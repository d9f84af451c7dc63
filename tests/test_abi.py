"""The C ABI library loads, exports every function include/femorax_b200.h declares, and reports
argument errors with status codes (no device work: runs without a GPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import _lib as L

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "femorax_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fx_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(L.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared()) <= set(L.PROTOTYPES), sorted(set(declared()) - set(L.PROTOTYPES))


def test_version_and_errors():
    lib = L.lib()
    assert b"sm_100a" in lib.fx_version()
    h = C.c_void_p()
    assert lib.fx_model_create(-1, None, None, C.byref(h)) == L.FX_E_INVALID
    assert b"bad arguments" in lib.fx_last_error()
    tags = np.arange(1, 9, dtype=np.int32)
    coords = np.zeros(24)
    assert lib.fx_model_create(8, tags.ctypes.data_as(L.p_i32), coords.ctypes.data_as(L.p_f64), C.byref(h)) == 0
    mat = L.fx_material(kind=0, E=-1.0, nu=0.3, rho=1.0)
    b = np.zeros(3)
    et = np.array([1], np.int32)
    rc = lib.fx_model_add_group(h, C.byref(mat), b.ctypes.data_as(L.p_f64), 0, 1, et.ctypes.data_as(L.p_i32),
                                tags.ctypes.data_as(L.p_i32))
    assert rc == L.FX_E_INVALID
    lib.fx_model_destroy(h)
    assert lib.fx_force_create(None, 0, C.byref(h)) == L.FX_E_INVALID
    assert lib.fx_vops_create(-5, 32, 0, C.byref(h)) == L.FX_E_INVALID


def test_host_api_mirrors_reference_names():
    for name in ("InternalForce", "MatrixFreeOperator", "ConjugateGradient", "Gmres", "KrylovSolver",
                 "OperatorCoefficients", "SolveOptions", "SolveResult", "VectorOps"):
        assert hasattr(fx, name)
