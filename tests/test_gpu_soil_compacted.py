"""The compacted plastic corrector (fx_force_set_soil_corrector FX_SOIL_COMPACTED: a predictor pass,
a compaction of the plastic points, the corrector on those only; src/exec/compacted_kernels.hpp) on
a B200 against the fused point pass: step by step through confinement, the switch to the plastic
stage and cyclic shear with commits, for PressureIndependMultiYield and PressureDependMultiYield
columns (one with Rayleigh damping through each point's current and committed tangents), the
internal force, the operator on the stored tangents, its diagonal and the plastic-point count are
the same bits."""
import numpy as np
import pytest

import femorax_b200 as fx

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")


def case(name):
    if name.startswith("pimy"):
        from tests.test_gpu_pimy_element import MATERIALS, column
        key = "sand" if name == "pimy_sand" else "clay_damped"
        in9, pairs = MATERIALS[key]
        return column(key), lambda: fx.PressureIndependMultiYield(*in9[:8], noYieldSurf=int(in9[8]), pairs=pairs), 8e-3
    from tests.test_gpu_pdmy_element import LIQ, SAND, column
    p = SAND if name == "pdmy_dense_damped" else LIQ
    spec = column(p, "full" if name == "pdmy_dense_damped" else None)
    return spec, lambda: fx.PressureDependMultiYield(*p[:14], noYieldSurf=int(p[14]), e=p[15], cs1=p[16], cs2=p[17],
                                                     cs3=p[18], pa=p[19], c=p[20], hv=p[21], pv=p[22]), 1e-3


@pytest.mark.parametrize("name", ["pimy_sand", "pimy_clay_damped", "pdmy_loose", "pdmy_dense_damped"])
def test_compacted_equals_fused(name):
    spec, material, amp = case(name)
    mesh = fx.Model(spec).compile().mesh()
    forces = [fx.InternalForce(mesh) for _ in range(2)]
    forces[1].set_soil_corrector("compacted")
    for f in forces:
        (f.set_pdmy if name.startswith("pdmy") else f.set_pimy)(0, material())
    n, P = mesh.num_equations, mesh.padded
    node, eq, X = mesh.node.reshape(8, P), mesh.eq.reshape(24, P), mesh.coords.reshape(3, -1)
    zq, dof = np.zeros(n), np.full(n, -1)
    for a in range(8):
        for d in range(3):
            q = eq[3 * a + d, :mesh.count]
            ok = q >= 0
            zq[q[ok]] = X[2, node[a, :mesh.count][ok]]
            dof[q[ok]] = d
    rng = np.random.default_rng(17)
    noise = rng.standard_normal(n) * 2e-6
    k = fx.OperatorCoefficients(1.0, 0.3, 0.5)
    plastic = 0
    for step in range(14):
        if step == 3:
            for f in forces:
                f.set_material_stage(0, 1)
        ev = 4e-4 * min(step + 1, 3) / 3
        gam = 0.0 if step < 3 else amp * np.sin(2 * np.pi * (step - 3) / 8)
        u = torch.as_tensor(np.where(dof == 2, -ev * zq, 0.0) + np.where(dof == 0, gam * zq, 0.0) + noise * (step >= 3),
                            device=DEV)
        v = torch.as_tensor(rng.standard_normal(n) * 1e-3, device=DEV)
        x = torch.as_tensor(rng.standard_normal(n), device=DEV)
        out = []
        for f in forces:
            r, y, d = (torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(3))
            f.compute(u, v, r)
            f.apply_operator(k, x, y)
            f.operator_diagonal(k, d)
            out.append((r, y, d, f.plastic_points()))
            f.commit_state()
        for a, b in zip(out[0][:3], out[1][:3]):
            assert torch.equal(a, b), step
        assert out[0][3] == out[1][3]
        plastic = max(plastic, out[0][3])
    assert plastic > 0
    assert forces[1].pimy_failed() == forces[0].pimy_failed() == 0
