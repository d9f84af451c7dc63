"""stdBrick with PressureIndependMultiYield points on a B200 (the Gauss-point path), against the
reference's own InternalForce with the same material (oracle/_ref), step by step along a load path:
confinement in the elastic stage, the switch to the plastic stage (updateMaterialStage), then cyclic
shear with commits. At every step the internal force, the operator y = K_t x + c M x with every
point's tangent at that displacement (the reference's TangentSource::Recomputed) and its diagonal
agree within 1e-12 of their largest entries, and bit for bit for the materials whose update calls
no pow (friction angle 0); the plastic stage yields points. One case carries Rayleigh damping
(alphaM; betaK through each point's current tangent, betaKcomm through its committed one), one
betaKcomm alone. ModifiedNewton -initial is refused on these sets, as the reference refuses it."""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")

BACKBONE = [1e-05, 0.98, 3e-05, 0.95, 0.0001, 0.85, 0.0003, 0.65, 0.001, 0.35, 0.003, 0.15, 0.01, 0.05, 0.03, 0.018]
MATERIALS = {
    "clay": ((1.8, 40500.0, 108000.0, 8.0, 0.1, 0.0, 100.0, 0.0, 20.0), None),
    "clay_damped": ((1.8, 40500.0, 108000.0, 8.0, 0.1, 0.0, 100.0, 0.0, 20.0), None),
    "sand_betaKcomm": ((2.0, 60000.0, 150000.0, 5.0, 0.1, 30.0, 80.0, 0.5, 20.0), None),
    "sand": ((2.0, 60000.0, 150000.0, 5.0, 0.1, 30.0, 80.0, 0.5, 20.0), None),
    "backbone_clay": ((1.8, 40500.0, 108000.0, 10.0, 0.1, 0.0, 100.0, 0.0, 8.0), BACKBONE),
}


def column(name):
    in9, pairs = MATERIALS[name]
    G, K = in9[1], in9[2]
    E, nu = 9 * K * G / (3 * K + G), (3 * K - 2 * G) / (2 * (3 * K + G))
    spec = meshes.box_model(2, 2, 5, size=(1.0, 1.0, 2.5), E=E, nu=nu, rho=in9[0])
    spec.groups[0].pimy = (np.array(in9), None if pairs is None else np.array(pairs))
    if name.endswith("_damped"):  # stiffness-proportional damping, current and committed tangents
        spec.rayleigh = [meshes.Rayleigh(0.05, 0.002, 0.0, 0.001, spec.groups[0].etags)]
    elif name.endswith("_betaKcomm"):  # betaKcomm alone: each point's committed tangent
        spec.rayleigh = [meshes.Rayleigh(0.0, 0.0, 0.0, 0.001, spec.groups[0].etags)]
    return spec


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name", list(MATERIALS))
def test_column_path_matches_reference(name, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("the reference build is not available")
    spec = column(name)
    in9, pairs = MATERIALS[name]
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh)
    mat = fx.PressureIndependMultiYield(*in9[:8], noYieldSurf=int(in9[8]), pairs=pairs)
    force.set_pimy(0, mat)
    assert force.info()["path"] == "general"
    ref = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile())
    n = mesh.num_equations
    P = mesh.padded
    node = mesh.node.reshape(8, P)
    eq = mesh.eq.reshape(24, P)
    X = mesh.coords.reshape(3, -1)
    zq, xq, yq = np.zeros(n), np.zeros(n), np.zeros(n)
    dof = np.full(n, -1)
    for a in range(8):
        for d in range(3):
            q = eq[3 * a + d, :mesh.count]
            ok = q >= 0
            nn = node[a, :mesh.count][ok]
            xq[q[ok]], yq[q[ok]], zq[q[ok]] = X[0, nn], X[1, nn], X[2, nn]
            dof[q[ok]] = d
    rng = np.random.default_rng(21)
    noise = rng.standard_normal(n) * 2e-5
    damped = name.endswith(("_damped", "_betaKcomm"))
    k = (1.0, 0.3, 0.5) if damped else (1.0, 0.0, 0.5)
    bitwise = in9[5] == 0.0
    plastic_seen = 0
    for step in range(16):
        stage = 0 if step < 3 else 1
        if step == 3:
            force.set_material_stage(0, 1)
            ref.set_stage(0, 1)
        ev = 1e-3 * min(step + 1, 3) / 3
        gam = 0.0 if step < 3 else 8e-3 * np.sin(2 * np.pi * (step - 3) / 8)
        u = np.where(dof == 2, -ev * zq, 0.0) + np.where(dof == 0, gam * zq, 0.0) + noise * (step >= 3)
        v = rng.standard_normal(n) * 1e-2 if damped else np.zeros(n)
        f = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.compute(torch.as_tensor(u, device=DEV), torch.as_tensor(v, device=DEV), f)
        fr = ref.force(u, v)
        got = f.cpu().numpy()
        assert rel(got, fr) <= 1e-12, (step, rel(got, fr))
        if bitwise:
            assert np.array_equal(got, fr), step
        x = rng.standard_normal(n)
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.apply_operator(fx.OperatorCoefficients(*k), torch.as_tensor(x, device=DEV), y)
        yr = ref.apply_operator_at(k, u, x)
        assert rel(y.cpu().numpy(), yr) <= 1e-12, step
        d = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.operator_diagonal(fx.OperatorCoefficients(*k), d)
        dr = ref.operator_diagonal_at(k, u)
        assert rel(d.cpu().numpy(), dr) <= 1e-12, step
        if bitwise:
            assert np.array_equal(y.cpu().numpy(), yr) and np.array_equal(d.cpu().numpy(), dr), step
        if stage == 1:
            plastic_seen = max(plastic_seen, force.plastic_points())
        force.commit_state()
        ref.commit()
    assert plastic_seen > 0
    assert force.pimy_failed() == 0


def test_binding_rules():
    spec = column("clay")
    mesh = fx.Model(spec).compile().mesh()
    force = fx.InternalForce(mesh)
    in9, _ = MATERIALS["clay"]
    wrong_rho = fx.PressureIndependMultiYield(2.5, *in9[1:8], noYieldSurf=20)
    with pytest.raises(fx.FxError):
        force.set_pimy(0, wrong_rho)
    with pytest.raises(fx.FxError):
        force.set_material_stage(0, 1)  # not bound yet
    force.set_pimy(0, fx.PressureIndependMultiYield(*in9[:8], noYieldSurf=20))
    with pytest.raises(fx.FxError):
        force.set_material_stage(0, 2)
    x = torch.zeros(mesh.num_equations, dtype=torch.float32, device=DEV)
    y = torch.zeros_like(x)
    with pytest.raises(fx.FxError) as e:  # no FP32 form of these tangents
        force.apply_operator(fx.OperatorCoefficients(), x, y)
    assert e.value.code == 2
    x64, y64 = x.double(), y.double()
    for call in (lambda k: force.apply_operator(k, x64, y64), lambda k: force.operator_diagonal(k, y64)):
        with pytest.raises(fx.FxError) as e:  # ModifiedNewton -initial (src/io/support.cpp:120-127)
            call(fx.OperatorCoefficients(initial=True))
        assert e.value.code == 2
    spec = column("clay")
    spec.rayleigh = [meshes.Rayleigh(0.0, 0.0, 0.001, 0.0, spec.groups[0].etags)]
    with pytest.raises(fx.FxError):  # betaKinit damping on the set (the reference refuses it too)
        fx.InternalForce(fx.Model(spec).compile().mesh()).set_pimy(0, fx.PressureIndependMultiYield(*in9[:8],
                                                                                                 noYieldSurf=20))


def test_newton_load_path_on_clay_column():
    """Quasi-static Newton (fx_solver_newton) through a cyclic top shear on a clay column in the
    plastic stage: every step converges on the stored tangents, points yield near the peaks, and
    the hysteresis leaves a residual top displacement after the cycle."""
    from femorax_b200 import serving, stages
    spec = column("clay")
    comp = fx.Model(spec).compile()
    force = fx.InternalForce(comp.mesh())
    in9, _ = MATERIALS["clay"]
    force.set_pimy(0, fx.PressureIndependMultiYield(*in9[:8], noYieldSurf=int(in9[8])))
    force.set_material_stage(0, 1)
    # 0.8 kN on the 1 m^2 top: base bending stress ~12 kPa against the clay's ~16 kPa in uniaxial stress
    f, mon = stages.top_shear(spec, serving.equation_map(comp), 0.8)
    factors = stages.cyclic_factors(1, 8)
    res = stages.load_path(force, torch.as_tensor(f, device=DEV), factors, mon, tol=1e-5, max_newton=60)
    assert res.converged
    assert max(res.plastic) > 0
    assert force.pimy_failed() == 0
    assert abs(res.monitor[-1]) > 1e-6 * max(abs(np.asarray(res.monitor)))
