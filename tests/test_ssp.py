"""SSPbrick's per-element data and compile maps on the CPU, against the reference (oracle/_ref):
the geometry record (Bnot's rows, the volume, each node's volume weight) and the stabilization
constants (hourglass vectors and the 12 x 12 interior matrix of GetStab) of fx_ssp_element_constants
bit for bit the reference's SSPbrick::point_store_geometry and element_constants on regular,
stretched, rotated and distorted elements; the compile step's arrays (including the SSPbrick
lumped masses: density times each node's volume weight) bit for bit compile_model's."""
import numpy as np
import pytest

import femorax_b200 as fx
from tests.models_for_tests import as_ssp, soil_column, ssp_block

BASE = np.array([[0, 1, 1, 0, 0, 1, 1, 0], [0, 0, 1, 1, 0, 0, 1, 1], [0, 0, 0, 0, 1, 1, 1, 1]], float)


def shapes(n=120, seed=0):
    rng = np.random.default_rng(seed)
    yield BASE
    yield BASE * np.array([[2.5], [0.4], [1.1]])
    for t in range(n):
        xl = BASE * rng.uniform(0.3, 3.0, (3, 1)) + 0.2 * rng.uniform(-1, 1, (3, 8))
        th = rng.uniform(0, 2 * np.pi)
        R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
        yield R @ xl if t % 2 else xl


def test_element_constants_bitwise(oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    for nu in (0.3, 0.49):
        for xl in shapes():
            g, c = fx.ssp_element_constants(xl, 3e7, nu)
            gr, cr = oracle_mod.ref_ssp_constants(xl, 3e7, nu)
            assert np.array_equal(g, gr) and np.array_equal(c, cr)


def test_stabilization_properties():
    """Kstab = Mben^T interior Mben annihilates rigid motions and linear fields (Bnot integrates
    them exactly): the interior matrix is symmetric positive semi-definite on the hourglass modes,
    the node volume weights sum to the volume, and Bnot reproduces a linear field's gradient."""
    xl = BASE * np.array([[1.3], [0.8], [2.0]]) + 0.1 * np.random.default_rng(1).uniform(-1, 1, (3, 8))
    g, c = fx.ssp_element_constants(xl, 3e7, 0.3)
    vol, nv = g[24], g[25:33]
    assert abs(nv.sum() - vol) <= 1e-12 * vol
    dN = g[:24].reshape(8, 3)
    grad = np.array([[0.3, -0.1, 0.2], [0.05, 0.4, -0.3], [0.1, 0.2, 0.7]])
    u = (grad @ xl).T  # u_i = grad x_i
    assert np.allclose(dN.T @ u, grad.T, rtol=0, atol=1e-12)
    gamma = c[:32].reshape(4, 8)
    assert np.allclose(gamma @ xl.T, 0.0, atol=1e-12)  # hourglass vectors orthogonal to linear fields
    K = np.zeros((12, 12))
    k = 32
    for r in range(12):
        for q in range(r, 12):
            K[r, q] = K[q, r] = c[k]
            k += 1
    assert np.min(np.linalg.eigvalsh(K)) >= -1e-9 * np.max(np.abs(K))


@pytest.mark.parametrize("name", ["block", "distorted", "column"])
def test_compile_maps_bitwise(name, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    spec = {"block": ssp_block(), "distorted": ssp_block(distort=0.2), "column": as_ssp(soil_column())}[name]
    mine = fx.Model(spec).compile()
    theirs = oracle_mod.RefModel(spec).compile()
    for a in fx.Compiled.I32 + fx.Compiled.F64:
        assert np.array_equal(mine.array(a), theirs.array(a)), a
    assert (fx.params_table(mine.params())[:, 15] == 1).all()
