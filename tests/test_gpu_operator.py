"""Parity of the CUDA paths with the oracle, through the C ABI, on a B200.

- general path (Gauss-point kernel, slot gather, --fmad=false): bit for bit with the oracle
  (which is bit for bit with the reference's host build: test_oracle_reference.py);
- box path (modal node-owner kernel): within 1e-12 of the largest entry (the reference's own
  element-test tolerance, test_std_brick_reference.cpp:28), the difference being rounding;
- FP32 forms: within 1e-5 of the largest entry of the FP64 result.
"""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes
from tests.models_for_tests import soil_column, two_region_block, roller_block

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda:0")
TOL_BOX = 1e-12
TOL_F32 = 1e-5


def rel_err(got, want):
    return np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300)


def build(spec, **kw):
    c = fx.Model(spec).compile(**kw)
    mesh = c.mesh()
    return mesh, fx.InternalForce(mesh), c


def models():
    out = {
        "block_consistent": two_region_block(),
        "block_lumped": two_region_block(lumped=True),
        "column_ties": soil_column(),
        "layered": meshes.layered_box(10, 7, 16, layers=4, seed=3)[0],
        "hetero": meshes.heterogeneous_cube(6, seed=4),
        "rollers": roller_block(),
        "distorted": meshes.distort(meshes.box_model(5, 4, 3), 0.2, seed=5),
    }
    return out


MODELS = models()
KS = [(1.0, 0.0, 0.0), (1.0, 0.4, 3.0), (0.0, 0.0, 1.0), (0.7, 2.0, 0.0)]


@pytest.fixture(scope="module", params=list(MODELS))
def case(request, oracle_mod):
    mesh, force, c = build(MODELS[request.param])
    return request.param, mesh, force, oracle_mod.PortMesh(mesh)


def t(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=DEV).contiguous()


def test_box_path_detection(case):
    name, mesh, force, _ = case
    info = force.info()
    expect_box = name not in ("column_ties", "distorted")
    assert info["box_qualifies"] == int(expect_box), info
    assert info["path"] == ("box" if expect_box else "general")


@pytest.mark.parametrize("k", KS)
def test_general_path_bitwise(case, k):
    name, mesh, force, port = case
    force.set_path("general")
    try:
        x = np.random.default_rng(7).standard_normal(mesh.num_equations)
        y = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
        force.apply_operator(fx.OperatorCoefficients(*k), t(x), y)
        assert np.array_equal(y.cpu().numpy(), port.apply_operator(k, x))
        d = torch.zeros_like(y)
        force.operator_diagonal(fx.OperatorCoefficients(*k), d)
        assert np.array_equal(d.cpu().numpy(), port.operator_diagonal(k))
    finally:
        force.set_path("auto")


def test_general_force_and_ground_bitwise(case):
    name, mesh, force, port = case
    force.set_path("general")
    try:
        rng = np.random.default_rng(8)
        u, v = rng.standard_normal(mesh.num_equations) * 1e-3, rng.standard_normal(mesh.num_equations) * 1e-2
        f = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
        force.compute(t(u), t(v), f)
        assert np.array_equal(f.cpu().numpy(), port.force(u, v))
        for d in range(3):
            force.mass_times_ground(d, f)
            assert np.array_equal(f.cpu().numpy(), port.mass_times_ground(d))
    finally:
        force.set_path("auto")


@pytest.mark.parametrize("k", KS)
def test_box_path_apply(case, k):
    name, mesh, force, port = case
    if force.info()["path"] != "box":
        pytest.skip("not a box grid")
    x = np.random.default_rng(9).standard_normal(mesh.num_equations)
    y = torch.full((mesh.num_equations,), np.nan, dtype=torch.float64, device=DEV)
    force.apply_operator(fx.OperatorCoefficients(*k), t(x), y)
    yy = y.cpu().numpy()
    assert np.all(np.isfinite(yy)), "an equation was not written"
    assert rel_err(yy, port.apply_operator(k, x)) <= TOL_BOX


def test_box_path_force(case):
    name, mesh, force, port = case
    if force.info()["path"] != "box":
        pytest.skip("not a box grid")
    rng = np.random.default_rng(10)
    u, v = rng.standard_normal(mesh.num_equations) * 1e-3, rng.standard_normal(mesh.num_equations) * 1e-2
    f = torch.full((mesh.num_equations,), np.nan, dtype=torch.float64, device=DEV)
    force.compute(t(u), t(v), f)
    assert rel_err(f.cpu().numpy(), port.force(u, v)) <= TOL_BOX


def test_box_path_fp32(case):
    name, mesh, force, port = case
    if force.info()["path"] != "box":
        pytest.skip("not a box grid")
    k = (1.0, 0.4, 3.0)
    x = np.random.default_rng(11).standard_normal(mesh.num_equations)
    y = torch.zeros(mesh.num_equations, dtype=torch.float32, device=DEV)
    force.apply_operator(fx.OperatorCoefficients(*k), t(x, torch.float32), y)
    assert rel_err(y.cpu().numpy().astype(np.float64), port.apply_operator(k, x)) <= TOL_F32
    if not force.info()["box_force"]:
        with pytest.raises(fx.FxError):
            force.compute(t(x, torch.float32), t(x, torch.float32), y)
        return
    u = np.random.default_rng(12).standard_normal(mesh.num_equations) * 1e-3
    v = np.random.default_rng(13).standard_normal(mesh.num_equations) * 1e-2
    f = torch.zeros(mesh.num_equations, dtype=torch.float32, device=DEV)
    force.compute(t(u, torch.float32), t(v, torch.float32), f)
    assert rel_err(f.cpu().numpy().astype(np.float64), port.force(u, v)) <= TOL_F32


def test_box_deterministic_and_host_apply(case):
    name, mesh, force, port = case
    k = fx.OperatorCoefficients(1.0, 0.2, 1.5)
    x = np.random.default_rng(14).standard_normal(mesh.num_equations)
    y1 = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
    y2 = torch.zeros_like(y1)
    force.apply_operator(k, t(x), y1)
    force.apply_operator(k, t(x), y2)
    assert torch.equal(y1, y2)
    yh = np.zeros(mesh.num_equations)
    force.apply_operator_host(k, np.ascontiguousarray(x), yh)
    assert np.array_equal(yh, y1.cpu().numpy())


def test_box_rejected_for_ties():
    mesh, force, _ = build(soil_column())
    with pytest.raises(fx.FxError) as e:
        force.set_path("box")
    assert e.value.code == 2


def test_launch_variants_agree(oracle_mod):
    """Every launch shape and plane count, as a grid or persistent (negative kz), gives the same bits
    (the owner sums in a fixed order): the operator and the internal force."""
    mesh, force, _ = build(meshes.layered_box(33, 17, 21, layers=3, seed=1)[0])
    k = fx.OperatorCoefficients(1.0, 0.1, 2.0)
    rng = np.random.default_rng(15)
    x = t(rng.standard_normal(mesh.num_equations))
    v = t(rng.standard_normal(mesh.num_equations))
    ref = fref = None
    from femorax_b200 import _lib as L
    lib = L.lib()
    for variant in range(11):
        for kz in (1, 3, 8, 64, -3, -8):
            L.check(lib.fx_force_set_launch(force._h, variant, kz))
            y = torch.zeros(mesh.num_equations, dtype=torch.float64, device=DEV)
            force.apply_operator(k, x, y)
            f = torch.zeros_like(y)
            try:
                force.compute(x, v, f)
            except fx.FxError as e:  # u and v staged together exceed a CTA's shared memory
                assert e.code == 2 and variant in (3, 8), (variant, kz)
                f = None
            if ref is None:
                ref = y.clone()
            if fref is None and f is not None:
                fref = f.clone()
            assert torch.equal(y, ref), (variant, kz)
            assert f is None or torch.equal(f, fref), (variant, kz)


@pytest.mark.parametrize("name", ["layered", "rollers"])
def test_host_apply_in_pieces_bitwise(name):
    """The host-buffer apply on a box grid of more than 262,144 equations with page-locked buffers
    copies x in and y out in equation ranges, overlapped with the tiles that read only arrived
    equations: the device apply's bits for every launch shape (the tile order is rebuilt when the
    shape changes, persistent shapes included), and the same as with pageable buffers (one copy
    each way). Rollers: nodes with one or two free DOFs."""
    spec = meshes.layered_box(64, 64, 24, layers=3, seed=2)[0] if name == "layered" else roller_block(70, 60, 40)
    mesh, force, _ = build(spec)
    n = mesh.num_equations
    assert force.info()["path"] == "box" and n > 262144
    k = fx.OperatorCoefficients(1.0, 0.3, 2.0)
    x = np.random.default_rng(16).standard_normal(n)
    xp = torch.from_numpy(x).pin_memory()
    yp = torch.empty(n, dtype=torch.float64, pin_memory=True)
    yn = np.empty(n)
    from femorax_b200 import _lib as L
    lib = L.lib()
    for shape in (None, (0, 5), (8, 12), (2, -10), (2, 10)):
        if shape is not None:
            L.check(lib.fx_force_set_launch(force._h, *shape))
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.apply_operator(k, t(x), y)
        want = y.cpu().numpy()
        yp.fill_(np.nan)
        force.apply_operator_host(k, xp.numpy(), yp.numpy())
        assert np.array_equal(yp.numpy(), want), shape
        yn.fill(np.nan)
        force.apply_operator_host(k, x, yn)
        assert np.array_equal(yn, want), shape
