"""Solvers, reductions and time stepping on a B200 against the oracle, through the C ABI.

- dot: the documented order (chunks of 2048, 32 lanes, fused products) bit for bit;
- CG / GMRES / Krylov: the solution of the oracle's solver within 1e-8 relative (iterates differ by
  rounding: the GPU vector kernels fuse multiply-adds), and the true FP64 residual, computed by
  the oracle's operator, below the requested tolerance;
- FP32 CG in FP64 iterative refinement: true FP64 residual <= 1e-8 relative; below the FP64
  floor it stops when a round no longer halves the residual;
- ExplicitDifference: displacements after 200 steps within 1e-10 relative of the oracle's; the
  FP32 run's recorded acceleration within 2e-3 of the largest FP64 value.
"""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes
from tests.models_for_tests import soil_column, two_region_block

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")


def t(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=DEV).contiguous()


def build(spec):
    c = fx.Model(spec).compile()
    mesh = c.mesh()
    return mesh, fx.InternalForce(mesh), c


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 65536 + 7, 3_000_001])
def test_dot_bitwise(n, oracle_mod):
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    for lanes in (32, 1):
        ops = fx.VectorOps(n, lanes)
        assert ops.dot(t(x), t(y)) == oracle_mod.port_dot(x, y, lanes, 1)


SOLVE_CASES = {
    "static_cube": (meshes.static_cube(8), (1.0, 0.0, 0.0)),
    "newmark_hetero": (meshes.heterogeneous_cube(7, seed=2), (1.0, 0.5 / (0.25 * 1e-3), 1.0 / (0.25 * 1e-6))),
    "block_damped": (two_region_block(), (1.0, 40.0, 400.0)),
    "column_ties": (soil_column(), (1.0, 0.0, 0.0)),
}


@pytest.mark.parametrize("name", list(SOLVE_CASES))
@pytest.mark.parametrize("solver", ["cg", "gmres", "krylov"])
def test_solvers_match_oracle(name, solver, oracle_mod):
    spec, k = SOLVE_CASES[name]
    mesh, force, _ = build(spec)
    port = oracle_mod.PortMesh(mesh)
    rng = np.random.default_rng(21)
    b = rng.standard_normal(mesh.num_equations)
    cls = {"cg": fx.ConjugateGradient, "gmres": fx.Gmres, "krylov": fx.KrylovSolver}[solver]
    s = cls(fx.SolveOptions(relative_tolerance=1e-10, max_iterations=5000))
    s.setup(fx.MatrixFreeOperator(force, fx.OperatorCoefficients(*k)))
    x = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
    r = s.solve(t(b), x)
    assert r.converged, r
    xo, ro = port.cg(b, k=k, rtol=1e-10, lanes=32) if solver != "gmres" else port.gmres(b, k=k, rtol=1e-10, lanes=32)
    xg = x.cpu().numpy()
    assert np.max(np.abs(xg - xo)) <= 1e-8 * np.max(np.abs(xo))
    res = b - port.apply_operator(k, xg)
    assert np.linalg.norm(res) <= 1.0001e-10 * np.linalg.norm(b)
    assert abs(r.iterations - ro["iterations"]) <= max(2, ro["iterations"] // 50)


def test_cg_warm_start_and_repeatability():
    mesh, force, _ = build(meshes.static_cube(6))
    b = t(np.random.default_rng(3).standard_normal(mesh.num_equations))
    s = fx.ConjugateGradient(fx.SolveOptions(relative_tolerance=1e-10))
    s.setup(fx.MatrixFreeOperator(force))
    x1 = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
    r1 = s.solve(b, x1)
    x2 = torch.zeros_like(x1)
    r2 = s.solve(b, x2)
    assert torch.equal(x1, x2) and r1.iterations == r2.iterations
    r3 = s.solve(b, x1)  # warm start from the solution: converged at iteration 0
    assert r3.converged and r3.iterations == 0


@pytest.mark.parametrize("name", ["per_set", "layered"])
def test_cg_graph_kept_between_solves(name):
    """A solver keeps its iteration graph for the next solve: the same vectors (graph reused),
    other vectors (captured again), a setup with other coefficients (graph dropped), and an apply
    with other coefficients between two solves (the coefficient tables rebuilt under it) all give
    the bits of a fresh solver."""
    spec = two_region_block(6, 5, 7) if name == "per_set" else meshes.layered_box(9, 8, 24, layers=3, seed=2)[0]
    mesh, force, _ = build(spec)
    n = mesh.num_equations
    b = t(np.random.default_rng(4).standard_normal(n))
    k1, k2 = fx.OperatorCoefficients(1.0, 0.2, 3.0), fx.OperatorCoefficients(1.0, 0.0, 50.0)
    opts = fx.SolveOptions(relative_tolerance=1e-11)

    def fresh(k):
        s = fx.ConjugateGradient(opts)
        s.setup(fx.MatrixFreeOperator(force, k))
        x = torch.zeros(n, dtype=torch.float64, device=DEV)
        r = s.solve(b, x)
        assert r.iterations > 16  # past the eager block: the graph ran
        return x, r.iterations

    x_ref1, it1 = fresh(k1)
    x_ref2, it2 = fresh(k2)
    s = fx.ConjugateGradient(opts)
    s.setup(fx.MatrixFreeOperator(force, k1))
    xa = torch.zeros(n, dtype=torch.float64, device=DEV)
    xb = torch.zeros(n, dtype=torch.float64, device=DEV)
    for x in (xa, xa, xb):
        x.zero_()
        assert s.solve(b, x).iterations == it1
        assert torch.equal(x, x_ref1)
    y = torch.zeros_like(b)
    force.apply_operator(k2, b, y)  # rebuilds the operator's coefficient tables for k2
    xa.zero_()
    s.solve(b, xa)
    assert torch.equal(xa, x_ref1)
    s.setup(fx.MatrixFreeOperator(force, k2))
    xa.zero_()
    assert s.solve(b, xa).iterations == it2
    assert torch.equal(xa, x_ref2)


def test_cg_indefinite_detection():
    """A negative stiffness coefficient makes p.Ap <= 0: CG reports indefinite, Krylov falls back."""
    mesh, force, _ = build(meshes.static_cube(4))
    b = t(np.ones(mesh.num_equations))
    s = fx.ConjugateGradient()
    # Jacobi needs a nonzero diagonal: -K has one; the operator is negative definite
    s.setup(fx.MatrixFreeOperator(force, fx.OperatorCoefficients(-1.0, 0.0, 0.0)))
    x = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
    r = s.solve(b, x)
    assert r.indefinite and not r.converged and r.iterations == 0


@pytest.mark.parametrize("name", ["static_cube", "newmark_hetero"])
def test_mixed_precision_refinement(name, oracle_mod):
    spec, k = SOLVE_CASES[name]
    mesh, force, _ = build(spec)
    port = oracle_mod.PortMesh(mesh)
    b = np.random.default_rng(5).standard_normal(mesh.num_equations)
    s = fx.MixedPrecisionSolver(fx.SolveOptions(relative_tolerance=1e-8, max_iterations=20000), inner_tolerance=1e-4)
    s.setup(fx.MatrixFreeOperator(force, fx.OperatorCoefficients(*k)))
    x = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
    r = s.solve(t(b), x)
    assert r.converged and r.refinements >= 1
    res = b - port.apply_operator(k, x.cpu().numpy())
    assert np.linalg.norm(res) <= 1.0001e-8 * np.linalg.norm(b)


def test_refinement_stops_at_the_fp64_floor():
    """A tolerance below what FP64 resolves (1e-20 relative): refinement stops at the first round
    that does not halve the FP64 residual, well before the 50-round limit, unconverged, with a
    residual at the FP64 level; the engine's slots stop by the same test."""
    spec, k = SOLVE_CASES["static_cube"]
    mesh, force, _ = build(spec)
    b = np.random.default_rng(6).standard_normal(mesh.num_equations)
    s = fx.MixedPrecisionSolver(fx.SolveOptions(relative_tolerance=1e-20, max_iterations=200000),
                                inner_tolerance=1e-4)
    s.setup(fx.MatrixFreeOperator(force, fx.OperatorCoefficients(*k)))
    x = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
    r = s.solve(t(b), x)
    assert not r.converged
    assert 2 <= r.refinements < 15, r.refinements
    assert r.final_residual <= 1e-12 * r.rhs_norm
    e = fx.BatchEngine(1 << 20, 2, k=fx.OperatorCoefficients(*k),
                       options=fx.SolveOptions(relative_tolerance=1e-20, max_iterations=200000))
    slot = e.admit(force, b)
    for _ in range(60):
        e.round()
        if e.finished(slot):
            break
    xe, re = e.retire(slot)
    assert not re.converged and re.refinements == r.refinements
    assert np.array_equal(xe, x.cpu().numpy())


def test_explicit_difference_matches_oracle(oracle_mod):
    spec, _ = meshes.layered_box(6, 5, 8, layers=4, seed=6, h=1.0)
    mesh, force, c = build(spec)
    port = oracle_mod.PortMesh(mesh)
    eq_dof = c.array("eq_dof").astype(np.int8)
    dt = 0.5 * force.min_critical_dt("ExplicitDifference")
    steps = 200
    ag = meshes.ricker(np.arange(steps) * dt + dt, f0=5.0, amplitude=1.0)
    n = mesh.num_equations
    rec = n - 1
    u, vh, a, v = (torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(4))
    hist = force.explicit_run(t(mesh.lumped_mass), u, vh, a, v, dt, steps, ag=ag, direction=0, record_eq=rec)
    uo, vho, ao, vo, ho = port.ed_steps(mesh.lumped_mass, eq_dof, dt, steps, ag=ag, direction=0, record_eq=rec)
    scale = np.max(np.abs(uo))
    assert scale > 0
    assert np.max(np.abs(u.cpu().numpy() - uo)) <= 1e-10 * scale
    assert np.max(np.abs(hist - ho)) <= 1e-10 * np.max(np.abs(ho))
    # FP32: the same steps in single precision
    u32, vh32, a32, v32 = (torch.zeros(n, dtype=torch.float32, device=DEV) for _ in range(4))
    h32 = force.explicit_run(t(mesh.lumped_mass, torch.float32), u32, vh32, a32, v32, dt, steps, ag=ag, direction=0,
                             record_eq=rec)
    assert np.max(np.abs(h32 - ho)) <= 2e-3 * np.max(np.abs(ho))


def test_critical_dt_matches_reference(oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    for spec in (meshes.layered_box(4, 3, 8, layers=4, seed=1)[0], two_region_block()):
        mesh, force, _ = build(spec)
        rf = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile())
        for scheme in ("ExplicitDifference", "CentralDifference"):
            assert abs(force.min_critical_dt(scheme) - rf.min_critical_dt(scheme)) <= 1e-10 * rf.min_critical_dt(scheme)
