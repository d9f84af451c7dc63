"""Batched quasi-static Newton (fx_nbatch_*) on a B200: several J2 columns of different sizes,
hardening and loads on one cyclic load path in one batch. Each instance's displacement history
and Newton solve counts must be bit for bit those of the single-instance path (fx_solver_newton
with the same options) on that mesh alone: the combined mesh keeps every instance's gather order,
and every instance's reductions run over its own range in the documented order, in the
block-per-chunk form of the CG kernels (few chunks) and the warp-per-chunk form (more than 1,024).
"""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import serving, stages
from tests.j2_newton_ref import top_shear_load
from tests.models_for_tests import j2_column

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda:0")
CASES = [(1, 1, 4, 0.5, 8e3), (2, 2, 4, 0.0, 30e3), (3, 2, 6, 1.0, 40e3), (2, 3, 8, 0.5, 20e3),
         (1, 2, 2, 0.5, 6e3), (3, 3, 4, 0.25, 45e3)]


def instances():
    out = []
    for nx, ny, nz, hk, total in CASES:
        spec = j2_column(nx=nx, ny=ny, nz=nz, hk=hk)
        comp = fx.Model(spec).compile()
        F, mon = top_shear_load(spec, serving.equation_map(comp), total)
        out.append((comp.mesh(), F, mon))
    return out


def test_batched_newton_equals_single_paths():
    inst = instances()
    factors = stages.cyclic_factors(1, 8)
    batched = stages.batched_load_path([m for m, _, _ in inst], [F for _, F, _ in inst], factors,
                                       [mon for _, _, mon in inst], tol=1e-6)
    assert batched.converged
    for i, (mesh, F, mon) in enumerate(inst):
        single = stages.load_path(fx.InternalForce(mesh), torch.as_tensor(F, device=DEV), factors, mon, tol=1e-6)
        assert single.converged
        assert np.array_equal(batched.monitor[:, i], single.monitor), i
        assert np.array_equal(batched.newton[:, i], single.newton), i


def test_layout():
    inst = instances()
    b = fx.BatchedNewton([m for m, _, _ in inst])
    assert np.all(b.offsets[:-1] % 2048 == 0)
    assert list(b.equations) == [m.num_equations for m, _, _ in inst]
    v = [np.arange(n, dtype=float) + i for i, n in enumerate(b.equations)]
    back = b.split(b.combine(v))
    assert all(np.array_equal(a, c) for a, c in zip(back, v))


def test_mixed_batched_newton_equals_single_mixed_paths():
    """FP32 CG inside FP64 refinement per instance (fx_nbatch_set_inner): each instance's history
    and Newton solve counts bit for bit those of the single-instance path with a
    MixedPrecisionSolver of the same tolerances, and close to the plain FP64 batch."""
    inst = instances()
    factors = stages.cyclic_factors(1, 8)
    args = ([m for m, _, _ in inst], [F for _, F, _ in inst], factors, [mon for _, _, mon in inst])
    mixed = stages.batched_load_path(*args, tol=1e-6, mixed=True, inner_tolerance=1e-4)
    plain = stages.batched_load_path(*args, tol=1e-6)
    assert mixed.converged
    for i, (mesh, F, mon) in enumerate(inst):
        ir = fx.MixedPrecisionSolver(fx.SolveOptions(relative_tolerance=1e-12, max_iterations=20000),
                                     inner_tolerance=1e-4)
        single = stages.load_path(fx.InternalForce(mesh), torch.as_tensor(F, device=DEV), factors, mon, tol=1e-6,
                                  solver=ir)
        assert single.converged
        assert np.array_equal(mixed.monitor[:, i], single.monitor), i
        assert np.array_equal(mixed.newton[:, i], single.newton), i
        peak = np.max(np.abs(plain.monitor[:, i]))
        assert np.max(np.abs(mixed.monitor[:, i] - plain.monitor[:, i])) <= 1e-6 * peak, i


def test_many_instances_warp_form_equals_single_paths():
    """More than 1,024 instances: the combined mesh spans more than 1,024 chunks (each instance's
    range padded to whole chunks), so the batch's CG vector kernels take the warp-per-chunk form,
    while each instance alone (one chunk) takes the block-per-chunk form: the same bits."""
    inst = instances()
    count = 1030
    meshes, loads, mons = [], [], []
    for i in range(count):
        mesh, F, mon = inst[i % len(inst)]
        meshes.append(mesh)
        loads.append(F * (0.6 + 0.4 * (i % 7) / 6.0))
        mons.append(mon)
    b = fx.BatchedNewton(meshes)
    assert b.offsets[-1] // 2048 > 1024
    factors = stages.cyclic_factors(1, 8)[:2]
    batched = stages.batched_load_path(meshes, loads, factors, mons, tol=1e-6)
    for i in (0, 5, 517, count - 1):
        single = stages.load_path(fx.InternalForce(meshes[i]), torch.as_tensor(loads[i], device=DEV), factors,
                                  mons[i], tol=1e-6)
        assert np.array_equal(batched.monitor[:, i], single.monitor), i
        assert np.array_equal(batched.newton[:, i], single.newton), i
        assert single.converged, i
    assert batched.converged
