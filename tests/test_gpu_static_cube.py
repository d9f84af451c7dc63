"""The static configuration as specified, on a B200 through the C ABI: the 32^3 stdBrick cube
(1 m, E 50 MPa, nu 0.3, base fixed) under a 100 kPa downward traction on its top face, solved by
Jacobi-preconditioned CG to a 1e-10 relative residual (104,544 equations).

The solution is compared with the reference's own ConjugateGradient (oracle/_ref, the reference
built from its sources, its host build: dot products in one lane) on the same compiled model:
within 1e-8 of the largest displacement for plain FP64 CG (iterates differ by rounding: the device
sums its dots in 32 lanes and its vector kernels fuse multiply-adds) and the iteration counts
within 2 %; within 1e-6 for the mixed form (FP32 CG inside FP64 refinement, which stops on its own
FP64 residual at a different iterate); for both, the true FP64 residual by the reference's own
operator below the requested 1e-10."""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def cube(oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    spec = meshes.static_cube(32)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    b = meshes.top_traction_vector(spec, meshes.equation_map(comp), mesh.num_equations)
    rc = oracle_mod.RefModel(spec).compile()
    rf = oracle_mod.RefForce(rc, cache=True)
    x_ref, info = rf.solve(b, method="cg", rtol=1e-10, lanes=1)
    assert info["converged"]
    return mesh, b, rf, x_ref, info


@pytest.mark.parametrize("solver", ["cg", "mixed"])
def test_static_cube_matches_reference_cg(cube, solver):
    mesh, b, rf, x_ref, info = cube
    assert mesh.num_equations == 104_544
    force = fx.InternalForce(mesh)
    assert force.info()["path"] == "box"
    cls = fx.ConjugateGradient if solver == "cg" else fx.MixedPrecisionSolver
    s = cls(fx.SolveOptions(relative_tolerance=1e-10, max_iterations=20000))
    s.setup(fx.MatrixFreeOperator(force))
    x = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
    r = s.solve(torch.as_tensor(b, device=DEV), x)
    assert r.converged, r
    xg = x.cpu().numpy()
    res = np.linalg.norm(b - rf.apply_operator((1.0, 0.0, 0.0), xg)) / np.linalg.norm(b)
    assert res <= 1.0001e-10, res
    assert np.max(np.abs(xg - x_ref)) <= (1e-8 if solver == "cg" else 1e-6) * np.max(np.abs(x_ref))
    if solver == "cg":
        assert abs(r.iterations - info["iterations"]) <= max(2, info["iterations"] // 50), (r.iterations, info)
    # the top settles downward under the downward traction
    assert np.min(xg) < 0
