"""Femora's retry and substep recovery of an implicit step (fx_solver_newmark_recover,
fx_solver_newton_recover; implicit_stage.cpp:261-402) on a B200, on a column with a J2 upper half
under a top shear load. Failures are made on the host, by the Newton limits:
- an attempt that fails goes back to the committed state: with no Newton iteration allowed every
  attempt fails, the step reports the reference's attempt, retry and substep counts, and u, v, a are
  the committed values bit for bit;
- a step that converges at once equals fx_solver_newmark (or fx_solver_newton) followed by a commit,
  bit for bit;
- a step whose Newton limit the full step misses but its halves meet is split in two substeps with
  the load ramped over the step, bit for bit the two half steps taken one after the other."""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import serving
from tests.j2_newton_ref import top_shear_load
from tests.models_for_tests import j2_column

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")
BETA, GAMMA, H = 0.25, 0.5, 2e-3


def setup(total=60e3):
    spec = j2_column(nx=2, ny=2, nz=4, hk=0.5)
    comp = fx.Model(spec).compile()
    F, mon = top_shear_load(spec, serving.equation_map(comp), total)
    return comp.mesh(), torch.as_tensor(F, device=DEV), mon


def solver_for(force, h):
    s = fx.ConjugateGradient(fx.SolveOptions(relative_tolerance=1e-12, max_iterations=20000))
    s.setup(fx.MatrixFreeOperator(force, fx.OperatorCoefficients(1.0, GAMMA / (BETA * h), 1.0 / (BETA * h * h))))
    return s


def state(n):
    return [torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(3)]


def test_every_attempt_fails_and_the_state_is_reverted():
    mesh, F, _ = setup()
    force = fx.InternalForce(mesh)
    s = solver_for(force, H)
    u, v, a = state(mesh.num_equations)
    s.newmark_step(F * 0.25, u, v, a, H, BETA, GAMMA)  # a committed, non-zero state
    force.commit_state()
    u0, v0, a0 = u.clone(), v.clone(), a.clone()
    st, r = s.newmark_step_recover(F * 0.25, F, u, v, a, H, BETA, GAMMA, tol=1e-12, max_newton=0, max_retries=2,
                                   num_sublevels=1, num_substeps=2)
    assert not r.converged
    # the full step and its retries, then the first substep and its retries
    assert st == dict(attempts=6, failed=6, retries=4, substepped=1, newton=0)
    assert torch.equal(u, u0) and torch.equal(v, v0) and torch.equal(a, a0)
    us = u.clone()
    st, r = s.newton_recover(F, u, tol=1e-12, max_newton=0, max_retries=3)
    assert not r.converged and st["attempts"] == 4 and st["retries"] == 3 and torch.equal(u, us)


def test_converged_step_equals_plain_step_and_commit():
    mesh, F, _ = setup()
    runs = []
    for recover in (False, True):
        force = fx.InternalForce(mesh)
        s = solver_for(force, H)
        u, v, a = state(mesh.num_equations)
        for i in range(4):
            f1 = F * ((i + 1) / 4)
            if recover:
                st, r = s.newmark_step_recover(None, f1, u, v, a, H, BETA, GAMMA, tol=1e-6, max_newton=25,
                                               max_retries=1, num_sublevels=2)
                assert r.converged and st["attempts"] == 1
            else:
                it, r = s.newmark_step(f1, u, v, a, H, BETA, GAMMA, tol=1e-6)
                assert r.converged
                force.commit_state()
        runs.append((u, v, a, force.plastic_points()))
    assert all(torch.equal(x, y) for x, y in zip(runs[0][:3], runs[1][:3]))
    assert runs[1][3] > 0  # the column yields


def newton_counts(mesh, F, h):
    """Newton iterations of one step of h from rest, and of its two halves taken in turn."""
    n = mesh.num_equations
    probe = fx.InternalForce(mesh)
    full_it, r = solver_for(probe, h).newmark_step(F, *state(n), h, BETA, GAMMA, tol=1e-6)
    if not r.converged:
        return None, None
    probe = fx.InternalForce(mesh)
    half = solver_for(probe, h / 2)
    uh, vh, ah = state(n)
    its = []
    for f in (F * 0.5, F):
        it, r = half.newmark_step(f, uh, vh, ah, h / 2, BETA, GAMMA, tol=1e-6)
        if not r.converged:
            return None, None
        probe.commit_state()
        its.append(it)
    return full_it, max(its)


def test_substeps_equal_two_half_steps():
    # a load and step size where the full step needs more Newton iterations than either half
    case = None
    for total in (60e3, 120e3, 240e3):
        mesh, F, _ = setup(total)
        for h in (2e-3, 2e-2, 2e-1):
            full_it, half_it = newton_counts(mesh, F, h)
            if full_it is not None and half_it < full_it:
                case = (mesh, F, h, full_it - 1)
                break
        if case:
            break
    assert case is not None, "no load and step size where the halves converge in fewer Newton iterations"
    mesh, F, h, limit = case
    n = mesh.num_equations
    zero = torch.zeros(n, dtype=torch.float64, device=DEV)
    # manual: two half steps with the ramped load, each committed
    f_man = fx.InternalForce(mesh)
    sm = solver_for(f_man, h / 2)
    um, vm, am = state(n)
    for f in (zero + 0.5 * (F - zero), F):
        it, r = sm.newmark_step(f, um, vm, am, h / 2, BETA, GAMMA, tol=1e-6, max_newton=limit)
        assert r.converged
        f_man.commit_state()
    # recovered: the full step fails at the limit, two substeps converge
    f_rec = fx.InternalForce(mesh)
    sr = solver_for(f_rec, h)
    ur, vr, ar = state(n)
    st, r = sr.newmark_step_recover(zero, F, ur, vr, ar, h, BETA, GAMMA, tol=1e-6, max_newton=limit, num_sublevels=1)
    assert r.converged and st["substepped"] == 1 and st["attempts"] == 3 and st["failed"] == 1
    assert torch.equal(ur, um) and torch.equal(vr, vm) and torch.equal(ar, am)
    assert f_rec.plastic_points() == f_man.plastic_points()
    # the solver is set up for the full step again: a plain step runs
    it, r = sr.newmark_step(F, ur, vr, ar, h, BETA, GAMMA, tol=1e-6)
    assert r.converged
