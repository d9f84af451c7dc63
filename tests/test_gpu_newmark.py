"""Newmark stages (fx_solver_newmark, beta 0.25, gamma 0.5) on a B200 against a dense Newmark on the
oracle (tests/j2_newton_ref.py): a heterogeneous cube (per-element E, consistent mass) and a
layered box (lumped mass, Rayleigh damping), under a harmonic top shear load.

The plain FP64 CG stage (linear solves to 1e-12) follows the oracle's direct solves to 1e-8 of the
monitored peak; the mixed-precision stage (FP32 CG inside FP64 refinement to a 1e-8 relative
residual per solve) follows the plain one to 1e-6 of the peak.
"""
import math

import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes, serving, stages
from tests.j2_newton_ref import dense_newmark, top_shear_load

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda:0")


def models():
    het = meshes.heterogeneous_cube(5, seed=7, size=5.0)
    lay, _ = meshes.layered_box(4, 3, 6, layers=3, seed=8)
    return {"hetero_consistent": (het, False), "layered_lumped": (lay, True)}


@pytest.mark.parametrize("name", list(models()))
def test_newmark_matches_dense_oracle(oracle_mod, name):
    spec, lumped = models()[name]
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh)
    assert force.info()["path"] == "box"
    F, mon = top_shear_load(spec, serving.equation_map(comp), 2e5)
    dt, steps, f0 = 2e-3, 40, 15.0
    Ft = torch.as_tensor(F, device=DEV)

    def load(t):
        return Ft * math.sin(2 * math.pi * f0 * t)

    want = dense_newmark(oracle_mod.PortMesh(mesh), lambda t: F * math.sin(2 * math.pi * f0 * t), steps, dt, mon,
                         lumped_mass=mesh.lumped_mass if lumped else None, tol=1e-6)
    plain = stages.newmark_run(force, load, steps, dt, mon, mixed=False, tol=1e-6, rtol=1e-12)
    assert plain.converged
    peak = np.max(np.abs(want))
    assert np.max(np.abs(plain.monitor - want)) <= 1e-8 * peak
    mixed = stages.newmark_run(fx.InternalForce(mesh), load, steps, dt, mon, mixed=True, tol=1e-6, rtol=1e-8)
    assert mixed.converged and mixed.refinements.sum() > 0
    assert np.max(np.abs(mixed.monitor - plain.monitor)) <= 1e-6 * peak


def test_newmark_setup_mismatch_is_an_error():
    spec = meshes.box_model(3, 3, 3)
    force = fx.InternalForce(fx.Model(spec).compile().mesh())
    cg = fx.ConjugateGradient(fx.SolveOptions(relative_tolerance=1e-10))
    cg.setup(fx.MatrixFreeOperator(force, fx.OperatorCoefficients(1.0, 0.0, 0.0)))
    n = force.num_equations
    z = [torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(4)]
    with pytest.raises(fx.FxError) as e:
        cg.newmark_step(z[0], z[1], z[2], z[3], 1e-3)
    assert e.value.code == 1
