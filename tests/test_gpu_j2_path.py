"""Quasi-static cyclic load paths on J2 meshes (Newton with the device CG per iteration,
fx_solver_newton) against a dense Newton on the oracle's J2 restatement (tests/j2_newton_ref.py),
on a B200. Both use the stage's NormUnbalance test ||f_ext - f_int|| <= 1e-6 N; the linear solves
differ (CG to 1e-12 against direct), so the monitored displacement histories agree to 1e-7 of
their largest value, and the plastic point counts agree step by step.
"""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import serving, stages
from tests.j2_newton_ref import dense_newton_path, top_shear_load
from tests.models_for_tests import j2_column

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda:0")


@pytest.mark.parametrize("total,hk", [(20e3, 0.5), (40e3, 0.0), (40e3, 1.0)])
def test_cyclic_path_matches_dense_newton(oracle_mod, total, hk):
    spec = j2_column(nx=2, ny=2, nz=4, hk=hk)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    F, mon = top_shear_load(spec, serving.equation_map(comp), total)
    factors = stages.cyclic_factors(1, 8)
    want, plastic = dense_newton_path(oracle_mod.PortMesh(mesh), F, factors, mon, tol=1e-6)
    force = fx.InternalForce(mesh)
    got = stages.load_path(force, torch.as_tensor(F, device=DEV), factors, mon, tol=1e-6)
    assert got.converged
    assert np.max(np.abs(got.monitor - want)) <= 1e-7 * np.max(np.abs(want))
    assert np.array_equal(got.plastic, plastic)
    assert plastic.max() > 0 and abs(want[-1]) > 1e-3 * np.max(np.abs(want))  # yielding; a residual offset


def test_disp_incr_test_and_elastic_box(oracle_mod):
    """NormDispIncr, and Newton on an elastic box mesh (the box force form): one linear step."""
    spec = fx.meshes.box_model(4, 3, 5, lumped=True)
    comp = fx.Model(spec).compile()
    force = fx.InternalForce(comp.mesh())
    assert force.info()["box_force"] == 1
    F, mon = top_shear_load(spec, serving.equation_map(comp), 1e5)
    got = stages.load_path(force, torch.as_tensor(F, device=DEV), [1.0], mon, tol=1e-9, test="NormDispIncr")
    assert got.converged and got.newton[0] <= 2
    x = torch.zeros(comp.num_equations, dtype=torch.float64, device=DEV)
    cg = fx.ConjugateGradient(fx.SolveOptions(relative_tolerance=1e-12))
    cg.setup(fx.MatrixFreeOperator(force, fx.OperatorCoefficients()))
    cg.solve(torch.as_tensor(F, device=DEV), x)
    assert got.monitor[0] == pytest.approx(float(x[mon].item()), rel=1e-9)


def test_fp32_gauss_point_operator(oracle_mod):
    """The FP32 Gauss-point operator (fx_apply_operator_f32 off the box path) against the FP64 one:
    an elastic distorted mesh with consistent mass and damping factors, and a J2 column after a
    force evaluation that leaves plastic points (their tangents), within 2e-5 of the largest entry."""
    spec = fx.meshes.distort(fx.meshes.box_model(5, 4, 6, lumped=False), 0.2, seed=7)
    cases = [(spec, fx.OperatorCoefficients(1.0, 0.3, 2.5)), (j2_column(nx=2, ny=2, nz=6), fx.OperatorCoefficients())]
    for sp, k in cases:
        comp = fx.Model(sp).compile()
        mesh = comp.mesh()
        force = fx.InternalForce(mesh)
        assert force.info()["path"] == "general"
        n = mesh.num_equations
        rng = np.random.default_rng(3)
        if sp is not spec:  # J2: strain the column past yield, keeping the trial tangents
            F, mon = top_shear_load(sp, serving.equation_map(comp), 60e3)
            u = torch.zeros(n, dtype=torch.float64, device=DEV)
            s = fx.ConjugateGradient(fx.SolveOptions(relative_tolerance=1e-12))
            s.setup(fx.MatrixFreeOperator(force, fx.OperatorCoefficients()))
            s.newton(torch.as_tensor(F, device=DEV), u, tol=1e-6)
            assert force.plastic_points() > 0
        x = rng.standard_normal(n)
        y64 = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.apply_operator(k, torch.as_tensor(x, device=DEV), y64)
        y32 = torch.zeros(n, dtype=torch.float32, device=DEV)
        force.apply_operator(k, torch.as_tensor(x, dtype=torch.float32, device=DEV), y32)
        ref = y64.cpu().numpy()
        assert np.max(np.abs(y32.cpu().numpy() - ref)) <= 2e-5 * np.max(np.abs(ref))


def test_mixed_precision_newton_on_j2(oracle_mod):
    """A cyclic J2 path with FP32 CG inside FP64 refinement for the Newton steps (FP32 operator on
    the point tangents, FP64 return map and residuals): the same plastic points step by step and
    the displacement history within 1e-6 of the plain FP64 path's largest value."""
    spec = j2_column(nx=2, ny=2, nz=6, hk=0.5)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    F, mon = top_shear_load(spec, serving.equation_map(comp), 30e3)
    factors = stages.cyclic_factors(1, 8)
    Ft = torch.as_tensor(F, device=DEV)
    plain = stages.load_path(fx.InternalForce(mesh), Ft, factors, mon, tol=1e-6)
    ir = fx.MixedPrecisionSolver(fx.SolveOptions(relative_tolerance=1e-12, max_iterations=20000), inner_tolerance=1e-4)
    mixed = stages.load_path(fx.InternalForce(mesh), Ft, factors, mon, tol=1e-6, solver=ir)
    assert plain.converged and mixed.converged
    assert plain.plastic.max() > 0
    assert np.array_equal(mixed.plastic, plain.plastic)
    assert np.max(np.abs(mixed.monitor - plain.monitor)) <= 1e-6 * np.max(np.abs(plain.monitor))
