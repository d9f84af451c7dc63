"""The C restatement (oracle/port) against the reference built here (oracle/_ref/libfxref.so):
bit for bit on the operator, its diagonal, the force, M r, CG, GMRES and the dot order."""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes
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


def motion_patterns(seed=0):
    """Three UniformExcitation patterns: a uniform series with a leading zero, a time-array
    series, and a short uniform series that holds its last value."""
    rng = np.random.default_rng(seed)
    return [dict(dof=0, fact=9.81, values=rng.standard_normal(50), dt=0.01, factor=1.5, prepend_zero=True),
            dict(dof=2, fact=-1.0, values=rng.standard_normal(40), times=np.cumsum(rng.uniform(0.005, 0.02, 40)),
                 factor=0.7),
            dict(dof=0, fact=2.0, values=rng.standard_normal(10), dt=0.03, use_last=True)]


def test_ground_motions_match_reference(oracle_mod, ref_available):
    """The port's PathSeries / PathTimeSeries restatement against the reference's own
    exec::GroundMotions, bit for bit, with times before the start, past the end and walking
    backwards through the time array."""
    if not ref_available:
        pytest.skip("reference library not built")
    pats = motion_patterns()
    port, ref = oracle_mod.PortMotions(pats), oracle_mod.RefMotions(pats)
    times = list(np.arange(-0.02, 0.7, 0.0037)) + [0.3, 0.1, 0.05, 0.6, 0.0, 0.35]
    for t in times:
        assert np.array_equal(port.evaluate(t), ref.evaluate(t)), t


def test_central_and_explicit_difference_agree_without_damping(oracle_mod):
    """Without damping both schemes are the central-difference recurrence
    u(n+1) = 2 u(n) - u(n-1) + dt^2 M^-1 (F(t_n) - K u(n)): from rest under a motion that starts at
    zero (no body force), the oracle's two stage restatements give the same displacements up to
    rounding."""
    spec = meshes.box_model(3, 2, 6, (1.0, 1.0, 3.0), E=2.0e5, nu=0.3, rho=2.0, lumped=True)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    port = oracle_mod.PortMesh(mesh)
    eq_dof = comp.array("eq_dof").astype(np.int8)
    cm = comp.array("lumped_alpha_mass")
    pats = [dict(dof=0, fact=1.0, values=np.sin(np.linspace(0, 6, 200)) ** 2, dt=0.002)]
    dt = 2e-4
    ue, _, _, te, _ = port.stage(1, mesh.lumped_mass, cm, eq_dof, pats, dt, 300)
    uc, _, _, tc, _ = port.stage(0, mesh.lumped_mass, cm, eq_dof, pats, dt, 300)
    scale = np.max(np.abs(ue))
    assert scale > 0
    assert np.max(np.abs(ue - uc)) <= 1e-9 * scale
    assert te == tc
