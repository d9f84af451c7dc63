"""J2 plasticity on the general path, on a B200, against the oracle's J2 restatement (the
reference has no J2: parity with it is unpinned; the oracle is pinned by its own properties in
test_oracle_j2.py).

Both sides form every value in the same order without fused multiply-adds, so the internal
force, the trial state, the tangent operator and its diagonal are compared bit for bit; the
tolerance written for them below (0) is the test's claim.
"""
import numpy as np
import pytest

import femorax_b200 as fx
from tests.models_for_tests import j2_column

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda:0")


def t(a):
    return torch.as_tensor(np.asarray(a), dtype=torch.float64, device=DEV).contiguous()


@pytest.fixture(scope="module", params=[False, True], ids=["consistent", "lumped"])
def case(request, oracle_mod):
    comp = fx.Model(j2_column(lumped=request.param)).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh)
    assert force.info()["path"] == "general"
    return mesh, force, oracle_mod.PortMesh(mesh)


def device_force(force, n, u, v):
    f = torch.zeros(n, dtype=torch.float64, device=DEV)
    force.compute(t(u), t(v), f)
    return f.cpu().numpy()


def device_apply(force, n, k, x):
    y = torch.zeros(n, dtype=torch.float64, device=DEV)
    force.apply_operator(k, t(x), y)
    return y.cpu().numpy()


def test_virgin_operator_is_elastic(case):
    mesh, force, pm = case
    n = mesh.num_equations
    x = np.random.default_rng(1).standard_normal(n)
    # before any force evaluation the tangent is the elastic matrix
    fresh = fx.InternalForce(mesh)
    y = device_apply(fresh, n, fx.OperatorCoefficients(1.0, 0.0, 0.3), x)
    want = pm.apply_j2(np.zeros(36 * 8 * mesh.padded), (1.0, 0.0, 0.3), x, initial=True)
    assert np.array_equal(y, want)


def test_force_state_tangent_two_steps(case):
    mesh, force, pm = case
    n = mesh.num_equations
    rng = np.random.default_rng(2)
    committed = pm.j2_state()
    force.set_j2_state(committed)
    for step in range(2):
        u = rng.standard_normal(n) * 2e-3
        v = rng.standard_normal(n) * 1e-3
        f = device_force(force, n, u, v)
        fr, trial, D, npl = pm.force_j2(committed, u, v)
        assert npl > 0 and force.plastic_points() == npl
        assert np.array_equal(f, fr), step
        assert np.array_equal(force.j2_state("trial"), trial)
        for k in (fx.OperatorCoefficients(1.0, 0.0, 0.0), fx.OperatorCoefficients(1.0, 0.2, 3.0),
                  fx.OperatorCoefficients(1.0, 0.0, 0.0, initial=True)):
            x = rng.standard_normal(n)
            kk = (k.stiffness, k.damping, k.mass)
            assert np.array_equal(device_apply(force, n, k, x), pm.apply_j2(D, kk, x, initial=k.initial))
            d = torch.zeros(n, dtype=torch.float64, device=DEV)
            force.operator_diagonal(k, d)
            assert np.array_equal(d.cpu().numpy(), pm.diagonal_j2(D, kk, initial=k.initial))
        force.commit_state()
        committed = trial
        assert np.array_equal(force.j2_state("committed"), committed)


def test_state_round_trip_and_errors(case):
    mesh, force, pm = case
    s = np.random.default_rng(4).standard_normal(13 * 8 * mesh.padded)
    force.set_j2_state(s)
    assert np.array_equal(force.j2_state(), s)
    with pytest.raises(fx.FxError):
        force.set_j2_state(s[:-1])
    box = fx.InternalForce(fx.Model(fx.meshes.box_model(3, 3, 3)).compile().mesh())
    with pytest.raises(fx.FxError) as e:
        box.j2_state()
    assert e.value.code == 2
