"""The stable explicit step on a B200, against the reference's own InternalForce (oracle/_ref):
- min_critical_dt on general meshes (distorted, laminar ties, damped consistent-mass block) and box
  grids, both schemes: bit for bit (the device solves each element's eigenproblem with the
  reference's rotations in the reference's order);
- every element's step (element_critical_dts) bit for bit;
- multi-yield soil columns sheared in the plastic stage: the exact step from the points' committed
  moduli and the periodic re-check's bound within 1e-12 of the reference's (the soils' pow may differ
  in the last place), the bound never above the exact step;
- the explicit stage's checks, failures made on the host: a NaN written into u between two calls
  stops the resumed stage at the next check with FX_E_DIVERGED; a step above the stable one stops
  the stage at its start with FX_E_UNSTABLE unless allowed."""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes
from femorax_b200._lib import FX_E_DIVERGED, FX_E_UNSTABLE
from tests.models_for_tests import soil_column, two_region_block

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")

MESHES = {
    "distorted": lambda: meshes.distort(meshes.box_model(6, 5, 4, lumped=True), 0.25, seed=3),
    "column_ties": soil_column,
    "block_damped": two_region_block,
    "layered_box": lambda: meshes.layered_box(10, 9, 8, layers=4, seed=1)[0],
}


def need_ref(ref_available):
    if not ref_available:
        pytest.skip("reference library not built")


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("scheme", ["ExplicitDifference", "CentralDifference"])
def test_min_critical_dt_bitwise(name, scheme, oracle_mod, ref_available):
    need_ref(ref_available)
    spec = MESHES[name]()
    force = fx.InternalForce(fx.Model(spec).compile().mesh())
    rf = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile())
    assert force.min_critical_dt(scheme) == rf.min_critical_dt(scheme)
    assert not force.stability_may_change() and not rf.stability_may_change()


@pytest.mark.parametrize("name", ["distorted", "block_damped"])
def test_element_critical_dts_bitwise(name, oracle_mod, ref_available):
    need_ref(ref_available)
    spec = MESHES[name]()
    force = fx.InternalForce(fx.Model(spec).compile().mesh())
    rf = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile())
    got = force.element_critical_dts("ExplicitDifference").cpu().numpy()
    want = rf.element_critical_dts("ExplicitDifference")
    assert got.shape == want.shape and np.array_equal(got, want)


def sheared_soil(kind, oracle_mod):
    """A 2 x 2 x 5 column of the dense sand (PressureDependMultiYield) or the frictional sand
    (PressureIndependMultiYield), confined, switched to the plastic stage and sheared with commits,
    on both sides."""
    if kind == "pdmy":
        from tests.test_gpu_pdmy_element import SAND, column
        spec = column(SAND)
        mat = fx.PressureDependMultiYield(*SAND[:14], noYieldSurf=int(SAND[14]), e=SAND[15], cs1=SAND[16],
                                          cs2=SAND[17], cs3=SAND[18], pa=SAND[19], c=SAND[20], hv=SAND[21], pv=SAND[22])
    else:
        from tests.test_gpu_pimy_element import MATERIALS, column
        spec = column("sand")
        in9, _ = MATERIALS["sand"]
        mat = fx.PressureIndependMultiYield(*in9[:8], noYieldSurf=int(in9[8]))
    mesh = fx.Model(spec).compile().mesh()
    force = fx.InternalForce(mesh)
    (force.set_pdmy if kind == "pdmy" else force.set_pimy)(0, mat)
    rf = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile())
    n, P = mesh.num_equations, mesh.padded
    node, eq, X = mesh.node.reshape(8, P), mesh.eq.reshape(24, P), mesh.coords.reshape(3, -1)
    zq, dof = np.zeros(n), np.full(n, -1)
    for a in range(8):
        for d in range(3):
            q = eq[3 * a + d, :mesh.count]
            ok = q >= 0
            zq[q[ok]] = X[2, node[a, :mesh.count][ok]]
            dof[q[ok]] = d
    for step in range(8):
        if step == 3:
            force.set_material_stage(0, 1)
            rf.set_stage(0, 1)
        ev = 5e-4 * min(step + 1, 3) / 3
        gam = 0.0 if step < 3 else 2e-3 * np.sin(2 * np.pi * (step - 3) / 8)
        u = np.where(dof == 2, -ev * zq, 0.0) + np.where(dof == 0, gam * zq, 0.0)
        f = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.compute(torch.as_tensor(u, device=DEV), torch.zeros(n, dtype=torch.float64, device=DEV), f)
        rf.force(u, np.zeros(n))
        force.commit_state()
        rf.commit()
    return force, rf


@pytest.mark.parametrize("kind", ["pimy", "pdmy"])
def test_soil_stable_step_and_bound(kind, oracle_mod, ref_available):
    need_ref(ref_available)
    force, rf = sheared_soil(kind, oracle_mod)
    assert force.stability_may_change() and rf.stability_may_change()
    for scheme in ("ExplicitDifference", "CentralDifference"):
        exact, want = force.min_critical_dt(scheme), rf.min_critical_dt(scheme)
        assert abs(exact - want) <= 1e-12 * want, (exact, want)
    force.prepare_stability_bounds()
    rf.prepare_stability_bounds()
    bound, want = force.min_critical_dt_bound(), rf.min_critical_dt_bound()
    assert abs(bound - want) <= 1e-12 * want, (bound, want)
    assert bound <= force.min_critical_dt()


def elastic_stage(nx=4, ny=3, nz=5):
    spec = meshes.box_model(nx, ny, nz, (1.0, 1.0, 1.5), E=2e6, nu=0.3, rho=1800.0, lumped=True)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh)
    mass = torch.as_tensor(mesh.lumped_mass, device=DEV)
    n = mesh.num_equations
    u, v, a = (torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(3))
    gm = fx.GroundMotions([dict(dof=0, fact=1.0, values=np.sin(np.linspace(0.0, 6.0, 200)), dt=1e-3)])
    return force, mass, u, v, a, gm


def test_nan_written_between_calls_stops_the_stage():
    force, mass, u, v, a, gm = elastic_stage()
    force.set_explicit_checks(nan_check_interval=100)
    dt = 0.5 * force.min_critical_dt()
    t, _ = force.explicit_stage("ExplicitDifference", mass, u, v, a, dt, 70, motions=gm)
    u[3] = float("nan")  # the failure, made on the host between two calls
    with pytest.raises(fx.FxError) as e:
        force.explicit_stage("ExplicitDifference", mass, u, v, a, dt, 60, time=t, motions=gm, resume=True)
    assert e.value.code == FX_E_DIVERGED and "step 100" in str(e.value)
    # a fresh stage from a finite state runs again
    u.zero_(), v.zero_(), a.zero_()
    force.explicit_stage("ExplicitDifference", mass, u, v, a, dt, 30, motions=gm)
    assert torch.isfinite(u).all()


@pytest.mark.parametrize("scheme", ["ExplicitDifference", "CentralDifference"])
def test_step_above_stable_step_is_refused_unless_allowed(scheme):
    force, mass, u, v, a, gm = elastic_stage()
    dt = 1.05 * force.min_critical_dt(scheme)
    alpha = torch.zeros_like(mass)
    with pytest.raises(fx.FxError) as e:
        force.explicit_stage(scheme, mass, u, v, a, dt, 10, motions=gm, alpha_mass=alpha)
    assert e.value.code == FX_E_UNSTABLE
    force.set_explicit_checks(allow_unstable_dt=True)
    force.explicit_stage(scheme, mass, u, v, a, dt, 10, motions=gm, alpha_mass=alpha)
