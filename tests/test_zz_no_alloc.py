"""fx_dot_noalloc against fx_vops_dot through the C ABI, on a B200.

fx_dot_noalloc keeps its partial sums in a fixed device array of the library instead of memory
allocated by a handle; the reduction order is the same, so the results must be the same bits
(the tolerance the dot tests use). Two calls in a row of different lengths check that the
shared array's leftover partials from one call never leak into the next.
"""
import ctypes as C

import numpy as np
import pytest

from femorax_b200 import _lib as L

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda:0")
MAX_N = 1 << 27


def _vops_dot(x, y, lanes):
    lib = L.lib()
    h = C.c_void_p()
    L.check(lib.fx_vops_create(x.numel(), lanes, 0, C.byref(h)))
    try:
        out = C.c_double()
        L.check(lib.fx_vops_dot(h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.numel(), None,
                                C.byref(out), None))
        return out.value
    finally:
        lib.fx_vops_destroy(h)


def _noalloc_dot(x, y, lanes, result_dev=None):
    lib = L.lib()
    out = C.c_double()
    rd = C.c_void_p(result_dev.data_ptr()) if result_dev is not None else None
    L.check(lib.fx_dot_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.numel(), lanes, rd,
                               C.byref(out), None))
    return out.value


@pytest.mark.parametrize("lanes", [32, 1])
def test_noalloc_dot_matches_vops_two_calls(lanes):
    rng = np.random.default_rng(1234 + lanes)
    # three levels of partials first (2049 chunks), then a single chunk, then two levels
    for n in (2048 * 2048 + 5, 1500, 3_000_001):
        x = torch.as_tensor(rng.standard_normal(n), device=DEV)
        y = torch.as_tensor(rng.standard_normal(n), device=DEV)
        want = _vops_dot(x, y, lanes)
        first = _noalloc_dot(x, y, lanes)
        r = torch.full((1,), float("nan"), dtype=torch.float64, device=DEV)
        second = _noalloc_dot(x, y, lanes, result_dev=r)
        torch.cuda.synchronize()
        assert first == want, (n, first, want)
        assert second == want, (n, second, want)
        assert r.item() == want
        exact = float(np.dot(x.cpu().numpy(), y.cpu().numpy()))
        assert abs(want - exact) <= 1e-12 * np.sqrt(n) * float(torch.linalg.vector_norm(x) * torch.linalg.vector_norm(y))


def test_noalloc_dot_empty_and_limit():
    x = torch.ones(4, dtype=torch.float64, device=DEV)
    assert _noalloc_dot(x[:0], x[:0], 32) == 0.0
    lib = L.lib()
    out = C.c_double()
    # rejected on the host before any device work: the length is checked first
    rc = lib.fx_dot_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), MAX_N + 1, 32, None, C.byref(out),
                            None)
    assert rc == L.FX_E_INVALID
    assert "scratch limit" in lib.fx_last_error().decode()
