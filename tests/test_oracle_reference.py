"""The C restatement (oracle/port) against the reference built here (oracle/_ref/libfxref.so):
bit for bit on the operator, its diagonal, the force, M r, CG, GMRES and the dot order."""
import numpy as np
import pytest

import femorax_b200 as fx
from tests.models_for_tests import soil_column, two_region_block


@pytest.fixture(scope="module", params=["block", "column"])
def pair(request, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    spec = two_region_block() if request.param == "block" else soil_column()
    c = oracle_mod.RefModel(spec).compile(renumbering="rcm", simd_width=32)
    mesh = fx.MeshArrays(**c.mesh_fields())
    return oracle_mod.PortMesh(mesh), oracle_mod.RefForce(c), c.num_equations


@pytest.mark.parametrize("k", [(1, 0, 0), (1, 0.3, 2.0), (0, 0, 1), (0.5, 1.5, 0)])
def test_operator_and_diagonal(pair, k):
    port, ref, n = pair
    x = np.random.default_rng(1).standard_normal(n)
    assert np.array_equal(port.apply_operator(k, x), ref.apply_operator(k, x))
    assert np.array_equal(port.operator_diagonal(k), ref.operator_diagonal(k))


def test_force_and_ground(pair):
    port, ref, n = pair
    rng = np.random.default_rng(2)
    u, v = rng.standard_normal(n) * 1e-3, rng.standard_normal(n) * 1e-2
    assert np.array_equal(port.force(u, v), ref.force(u, v))
    for d in range(3):
        assert np.array_equal(port.mass_times_ground(d), ref.mass_times_ground(d))


def test_solvers(pair):
    port, ref, n = pair
    b = np.random.default_rng(3).standard_normal(n)
    xr, rr = ref.solve(b, method="cg", lanes=1)
    xp, rp = port.cg(b, lanes=1)
    assert rr["iterations"] == rp["iterations"] and np.array_equal(xr, xp)
    xr, rr = ref.solve(b, method="gmres", lanes=1, restart=20)
    xp, rp = port.gmres(b, lanes=1, restart=20)
    assert rr["iterations"] == rp["iterations"] and np.array_equal(xr, xp)


@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 100000, 5000000])
@pytest.mark.parametrize("lanes", [1, 32])
def test_dot_order(oracle_mod, ref_available, n, lanes):
    if not ref_available:
        pytest.skip("reference library not built")
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    assert oracle_mod.ref_host_dot(x, y, lanes) == oracle_mod.port_dot(x, y, lanes, 0)
