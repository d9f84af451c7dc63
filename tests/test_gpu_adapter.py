"""The reference-side binding (tests/integration/b200_operator.hpp, a solvers::LinearOperator over
this library's operator) drives the reference's own ConjugateGradient and Jacobi
(oracle/_ref/libfxadapter.so: the binding compiled against the reference's headers, the solvers
from the reference's sources) on a B200: the solution equals, within 1e-10 of its largest entry,
what the same reference solver gives on the reference's own InternalForce operator, in an
iteration count within 2 % of it; the host views of the reference's host build go through the
host-buffer calls fx_apply_operator_host and fx_operator_diagonal_host."""
import ctypes as C
import os

import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes
from tests.models_for_tests import soil_column, two_region_block

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

ADAPTER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libfxadapter.so")
CASES = {
    "static_cube": (lambda: meshes.static_cube(10), (1.0, 0.0, 0.0)),
    "block_damped": (two_region_block, (1.0, 40.0, 400.0)),
    "column_ties": (soil_column, (1.0, 0.0, 0.0)),
}


def adapter():
    if not os.path.exists(ADAPTER):
        pytest.skip("adapter library not built (needs the reference checkout at build time)")
    lib = C.CDLL(ADAPTER)
    lib.fxadapt_cg_solve.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                     C.c_void_p]
    lib.fxadapt_last_error.restype = C.c_char_p
    return lib


@pytest.mark.parametrize("name", list(CASES))
def test_reference_cg_through_b200_operator(name, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    lib = adapter()
    build, k = CASES[name]
    spec = build()
    mesh = fx.Model(spec).compile().mesh()
    force = fx.InternalForce(mesh)
    n = mesh.num_equations
    b = np.random.default_rng(7).standard_normal(n)
    x = np.zeros(n)
    kk = np.array(k, np.float64)
    out = np.zeros(6)
    rc = lib.fxadapt_cg_solve(force._h, n, kk.ctypes.data, b.ctypes.data, x.ctypes.data, 1e-10, 5000, out.ctypes.data)
    assert rc == 0, lib.fxadapt_last_error()
    assert out[0] == 1 and out[5] == 0
    rf = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile(), cache=True)
    x_ref, info = rf.solve(b, k=k, method="cg", rtol=1e-10, lanes=1)
    assert np.max(np.abs(x - x_ref)) <= 1e-10 * np.max(np.abs(x_ref))
    assert abs(int(out[1]) - info["iterations"]) <= max(2, info["iterations"] // 50)
