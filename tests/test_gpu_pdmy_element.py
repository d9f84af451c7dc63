"""stdBrick with PressureDependMultiYield points on a B200 (the Gauss-point path), against the
reference's own InternalForce with the same material (oracle/_ref), step by step: confinement in the
elastic stage, the switch to the plastic stage, cyclic shear with commits. Force, operator (each
point's stored tangent at that displacement, upper triangle mirrored as the reference stores it)
and diagonal within 1e-10 of their largest entries: the device's pow (the modulus factor of every
update) may differ from the host's in the last place, so this material is not held bit for bit.
Damped cases: alphaM with betaK (each point's current tangent) and betaKcomm (its committed one);
betaKcomm alone; and ModifiedNewton -initial with damping, where the stiffness term takes the
material's initial tangent and betaK damping stays on the current one (element_operator.hpp:45-56)."""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")

# dense sand of the stored paths (rho, G, K, phi, gamma_peak, p_ref, n, PT angle, contrac, dilat1,
# dilat2, liquefac1..3, surfaces, e, cs1..3, pa, c, hv, pv)
SAND = (2.0285423037716614, 145000.0, 314166.66666666663, 40.0, 0.1, 80.0, 0.5, 27.0, 0.03, 0.8, 5.0, 0.0, 0.0,
        0.0, 20.0, 0.45, 0.9, 0.02, 0.7, 101.0, 0.3, 0.0, 1.0)
LIQ = (1.9469928644240571, 75000.0, 162499.99999999997, 29.0, 0.1, 80.0, 0.5, 29.0, 0.21, 0.0, 0.0, 10.0, 0.02,
       1.0, 20.0, 0.85, 0.9, 0.02, 0.7, 101.0, 0.3, 0.0, 1.0)


def column(p, damping=None):
    G, K = p[1], p[2]
    E, nu = 9 * K * G / (3 * K + G), (3 * K - 2 * G) / (2 * (3 * K + G))
    spec = meshes.box_model(2, 2, 5, size=(1.0, 1.0, 2.5), E=E, nu=nu, rho=p[0])
    spec.groups[0].pdmy = (np.array(p), None)
    if damping == "comm":  # betaKcomm alone: each point's committed tangent
        spec.rayleigh = [meshes.Rayleigh(0.0, 0.0, 0.0, 0.001, spec.groups[0].etags)]
    elif damping:  # Rayleigh damping, betaK through each point's current tangent, betaKcomm its committed one
        spec.rayleigh = [meshes.Rayleigh(0.05, 0.002, 0.0, 0.001, spec.groups[0].etags)]
    return spec


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("p,damping", [(SAND, None), (LIQ, None), (SAND, "full"), (LIQ, "comm"), (SAND, "initial")],
                         ids=["dense_sand", "loose_sand_ppz", "dense_sand_damped", "loose_sand_betaKcomm",
                              "dense_sand_damped_initial"])
def test_column_path_matches_reference(p, damping, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("the reference build is not available")
    spec = column(p, damping)
    damped = damping is not None
    initial = damping == "initial"
    mesh = fx.Model(spec).compile().mesh()
    force = fx.InternalForce(mesh)
    force.set_pdmy(0, fx.PressureDependMultiYield(*p[:14], noYieldSurf=int(p[14]), e=p[15], cs1=p[16], cs2=p[17],
                                                   cs3=p[18], pa=p[19], c=p[20], hv=p[21], pv=p[22]))
    assert force.info()["path"] == "general"
    ref = oracle_mod.RefForce(oracle_mod.RefModel(spec).compile())
    n, P = mesh.num_equations, mesh.padded
    node, eq, X = mesh.node.reshape(8, P), mesh.eq.reshape(24, P), mesh.coords.reshape(3, -1)
    zq, dof = np.zeros(n), np.full(n, -1)
    for a in range(8):
        for d in range(3):
            q = eq[3 * a + d, :mesh.count]
            ok = q >= 0
            zq[q[ok]] = X[2, node[a, :mesh.count][ok]]
            dof[q[ok]] = d
    rng = np.random.default_rng(22)
    noise = rng.standard_normal(n) * 2e-6
    k = (1.0, 0.3, 0.5) if damped else (1.0, 0.0, 0.5)
    plastic_seen = 0
    for step in range(14):
        if step == 3:
            force.set_material_stage(0, 1)
            ref.set_stage(0, 1)
        ev = 2e-4 * min(step + 1, 3) / 3
        gam = 0.0 if step < 3 else 1e-3 * np.sin(2 * np.pi * (step - 3) / 8)
        u = np.where(dof == 2, -ev * zq, 0.0) + np.where(dof == 0, gam * zq, 0.0) + noise * (step >= 3)
        v = rng.standard_normal(n) * 1e-3 if damped else np.zeros(n)
        f = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.compute(torch.as_tensor(u, device=DEV), torch.as_tensor(v, device=DEV), f)
        assert rel(f.cpu().numpy(), ref.force(u, v)) <= 1e-10, step
        x = rng.standard_normal(n)
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.apply_operator(fx.OperatorCoefficients(*k, initial=initial), torch.as_tensor(x, device=DEV), y)
        assert rel(y.cpu().numpy(), ref.apply_operator_at(k, u, x, initial=initial)) <= 1e-10, step
        dg = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.operator_diagonal(fx.OperatorCoefficients(*k, initial=initial), dg)
        assert rel(dg.cpu().numpy(), ref.operator_diagonal_at(k, u, initial=initial)) <= 1e-10, step
        if step >= 3:
            plastic_seen = max(plastic_seen, force.plastic_points())
        force.commit_state()
        ref.commit()
    assert plastic_seen > 0
    assert force.pimy_failed() == 0
