"""SSPbrick (one integration point, physical hourglass stabilization; §8(f) of the path) on a B200,
through the C ABI, against the reference's own InternalForce with SSPbrick groups (oracle/_ref):
- operator y = K_eff x (with Kstab in every stiffness term), its diagonal, the internal force with
  body force and the four Rayleigh terms, M r_dir, and the stable step: bit for bit on meshes of
  SSPbrick alone (the same element arithmetic, the same gather order);
- a mesh of stdBrick and SSPbrick groups: the reference keeps one batch per element type and sums
  the batches one after the other, this library one batch in element order, so within 1e-14;
- Jacobi-PCG on an SSPbrick column against the reference's ConjugateGradient;
- the element constants were checked bit for bit on the host (tests/test_ssp.py)."""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes
from tests.models_for_tests import as_ssp, soil_column, ssp_block

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")


def mixed():
    """A column whose lower half is stdBrick and upper half SSPbrick."""
    spec = soil_column(3, 2, 8)
    spec.groups[1].element = 1
    spec.groups[1].lumped = True
    return spec


MODELS = {
    "block": (lambda: ssp_block(), True),
    "distorted": (lambda: ssp_block(5, 4, 3, distort=0.25, seed=4), True),
    "column_ties": (lambda: as_ssp(soil_column(3, 2, 8)), True),
    "mixed_std_ssp": (mixed, False),
}


def dev(a):
    return torch.as_tensor(np.asarray(a), dtype=torch.float64, device=DEV)


def check(got, want, bitwise):
    if bitwise:
        assert np.array_equal(got, want), np.max(np.abs(got - want)) / np.max(np.abs(want))
    else:
        assert np.max(np.abs(got - want)) <= 1e-14 * np.max(np.abs(want))


@pytest.mark.parametrize("name", list(MODELS))
def test_ssp_matches_reference_internal_force(name, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    build, bitwise = MODELS[name]
    spec = build()
    mesh = fx.Model(spec).compile().mesh()
    force = fx.InternalForce(mesh)
    assert force.info()["path"] == "general"
    rf = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile())
    n = mesh.num_equations
    rng = np.random.default_rng(5)
    for k in ((1.0, 0.0, 0.0), (1.0, 0.3, 2.0), (0.0, 0.0, 1.0)):
        x = rng.standard_normal(n)
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.apply_operator(fx.OperatorCoefficients(*k), dev(x), y)
        check(y.cpu().numpy(), rf.apply_operator(k, x), bitwise)
        d = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.operator_diagonal(fx.OperatorCoefficients(*k), d)
        check(d.cpu().numpy(), rf.operator_diagonal(k), bitwise)
    u, v = 1e-3 * rng.standard_normal(n), 1e-2 * rng.standard_normal(n)
    f = torch.zeros(n, dtype=torch.float64, device=DEV)
    force.compute(dev(u), dev(v), f)
    check(f.cpu().numpy(), rf.force(u, v), bitwise)
    for direction in range(3):
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.mass_times_ground(direction, y)
        check(y.cpu().numpy(), rf.mass_times_ground(direction), bitwise)
    for scheme in ("ExplicitDifference", "CentralDifference"):
        assert force.min_critical_dt(scheme) == rf.min_critical_dt(scheme)


def test_ssp_cg_matches_reference(oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    spec = as_ssp(soil_column(3, 2, 10))
    mesh = fx.Model(spec).compile().mesh()
    force = fx.InternalForce(mesh)
    b = np.random.default_rng(8).standard_normal(mesh.num_equations)
    s = fx.ConjugateGradient(fx.SolveOptions(relative_tolerance=1e-10))
    s.setup(fx.MatrixFreeOperator(force))
    x = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
    r = s.solve(dev(b), x)
    assert r.converged
    rf = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile())
    xr, info = rf.solve(b, method="cg", rtol=1e-10, lanes=1)
    assert np.max(np.abs(x.cpu().numpy() - xr)) <= 1e-8 * np.max(np.abs(xr))
    assert abs(r.iterations - info["iterations"]) <= max(2, info["iterations"] // 50)


def test_ssp_refusals():
    spec = ssp_block()
    force = fx.InternalForce(fx.Model(spec).compile().mesh())
    x = torch.zeros(force.num_equations, dtype=torch.float32, device=DEV)
    with pytest.raises(fx.FxError) as e:  # no FP32 form of the element
        force.apply_operator(fx.OperatorCoefficients(), x, torch.zeros_like(x))
    assert e.value.code == 2
    j2 = ssp_block()
    j2.groups[0].kind, j2.groups[0].sigma_y, j2.groups[0].H = 1, 1e3, 10.0
    with pytest.raises(fx.FxError) as e:  # SSPbrick groups take the elastic material
        fx.Model(j2)
    assert e.value.code == 2
