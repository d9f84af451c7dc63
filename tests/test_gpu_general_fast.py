"""The Gauss-point path's fast form (fx_force_set_general_mode FX_GENERAL_FAST: eight threads per
element, fused multiply-adds) on a B200 against its exact form (the reference's arithmetic, bit for
bit the oracle's): the operator with stiffness, damping and mass terms and the internal force with
body force and all four Rayleigh terms, on distorted, tied, consistent- and lumped-mass meshes,
within 1e-12 of the largest entry; meshes with J2 sets keep the exact form (bit for bit)."""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes
from tests.models_for_tests import j2_column, soil_column, two_region_block

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")

MESHES = {
    "distorted": lambda: meshes.distort(meshes.box_model(7, 5, 6, lumped=False), 0.25, seed=9),
    "column_ties": lambda: soil_column(4, 3, 10),
    "block_damped": lambda: meshes.distort(two_region_block(6, 5, 7), 0.1, seed=2),
    "hetero": lambda: meshes.distort(meshes.heterogeneous_cube(5, seed=3), 0.15, seed=4),
}


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("name", list(MESHES))
def test_fast_form_matches_exact(name):
    mesh = fx.Model(MESHES[name]()).compile().mesh()
    exact, fast = fx.InternalForce(mesh), fx.InternalForce(mesh)
    fast.set_general_mode("fast")
    assert exact.info()["path"] == "general"
    n = mesh.num_equations
    rng = np.random.default_rng(3)
    for k in ((1.0, 0.0, 0.0), (1.0, 0.4, 3.0)):
        x = torch.as_tensor(rng.standard_normal(n), device=DEV)
        ye, yf = (torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(2))
        exact.apply_operator(fx.OperatorCoefficients(*k), x, ye)
        fast.apply_operator(fx.OperatorCoefficients(*k), x, yf)
        assert rel(yf.cpu().numpy(), ye.cpu().numpy()) <= 1e-12
    u = torch.as_tensor(1e-3 * rng.standard_normal(n), device=DEV)
    v = torch.as_tensor(1e-2 * rng.standard_normal(n), device=DEV)
    fe, ff = (torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(2))
    exact.compute(u, v, fe)
    fast.compute(u, v, ff)
    assert rel(ff.cpu().numpy(), fe.cpu().numpy()) <= 1e-12


def test_j2_meshes_keep_the_exact_form():
    mesh = fx.Model(j2_column(nx=2, ny=2, nz=4)).compile().mesh()
    exact, fast = fx.InternalForce(mesh), fx.InternalForce(mesh)
    fast.set_general_mode("fast")
    n = mesh.num_equations
    x = torch.as_tensor(np.random.default_rng(1).standard_normal(n), device=DEV)
    ye, yf = (torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(2))
    exact.apply_operator(fx.OperatorCoefficients(), x, ye)
    fast.apply_operator(fx.OperatorCoefficients(), x, yf)
    assert torch.equal(ye, yf)
