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
