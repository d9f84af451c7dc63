"""Explicit stages on the device (fx_explicit_stage) and the device ground motions (fx_motions),
against the oracle's restatement of ExplicitAnalysis (oracle.PortMesh.stage) and of
GroundMotions (oracle.PortMotions, itself pinned to the reference's GroundMotions on the CPU).

On the general path the force is the reference's arithmetic and the stage kernels round every
operation as the host build does, so whole stages are compared bit for bit; on the box path the
force agrees to 1e-12, so stage histories are compared to 1e-10 of their peak."""
import numpy as np
import pytest
import torch

import femorax_b200 as fx
from femorax_b200 import meshes
from tests.models_for_tests import j2_column
from tests.test_oracle_reference import motion_patterns

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
SCHEMES = {"ExplicitDifference": 1, "CentralDifference": 0}


def stage_case(general):
    """A damped layered soil box (lumped mass, Rayleigh alphaM and betaK); distorted, it runs on
    the general path."""
    spec, _ = meshes.layered_box(5, 4, 7, layers=3, seed=11, h=1.0)
    if general:
        spec = meshes.distort(spec, 0.15, seed=3)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh)
    assert force.info()["path"] == ("general" if general else "box")
    return comp, mesh, force


def dev(a):
    return torch.as_tensor(np.asarray(a, np.float64), device=DEV).contiguous()


def test_device_motions_match_oracle(oracle_mod):
    pats = motion_patterns(seed=4)
    gm = fx.GroundMotions(pats)
    port = oracle_mod.PortMotions(pats)
    for t in list(np.arange(-0.02, 0.75, 0.0041)) + [0.3, 0.1, 0.05, 0.6, 0.0, 0.35]:
        assert np.array_equal(gm.evaluate(t), port.evaluate(t)), t


def run_both(oracle_mod, comp, mesh, force, scheme, steps, dt, time0=0.0, state=None):
    pats = motion_patterns(seed=2)
    n = mesh.num_equations
    rng = np.random.default_rng(5)
    u0, v0, a0 = state if state is not None else (rng.standard_normal(n) * 1e-4, rng.standard_normal(n) * 1e-3,
                                                   np.zeros(n))
    mass, cm = mesh.lumped_mass, comp.array("lumped_alpha_mass")
    eq_dof = comp.array("eq_dof").astype(np.int8)
    rec = n // 2
    u, v, a = dev(u0), dev(v0), dev(a0)
    t_end, hist = force.explicit_stage(scheme, dev(mass), u, v, a, dt, steps, time=time0,
                                       motions=fx.GroundMotions(pats), alpha_mass=dev(cm), record_eq=rec)
    port = oracle_mod.PortMesh(mesh)
    uo, vo, ao, to, ho = port.stage(SCHEMES[scheme], mass, cm, eq_dof, pats, dt, steps, time=time0, u=u0, v=v0, a=a0,
                                    record_eq=rec)
    return (u.cpu().numpy(), v.cpu().numpy(), a.cpu().numpy(), t_end, hist), (uo, vo, ao, to, ho)


@pytest.mark.parametrize("scheme", list(SCHEMES))
def test_stage_general_path_bitwise(oracle_mod, scheme):
    comp, mesh, force = stage_case(general=True)
    dt = 0.4 * force.min_critical_dt(scheme)
    got, want = run_both(oracle_mod, comp, mesh, force, scheme, 53, dt, time0=-0.01)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    assert np.max(np.abs(want[0])) > 0


@pytest.mark.parametrize("scheme", list(SCHEMES))
def test_stage_box_path(oracle_mod, scheme):
    comp, mesh, force = stage_case(general=False)
    dt = 0.4 * force.min_critical_dt(scheme)
    got, want = run_both(oracle_mod, comp, mesh, force, scheme, 41, dt)
    assert got[3] == want[3]  # the stage time: the same additions
    for g, w in zip(got[:3] + got[4:], want[:3] + want[4:]):
        assert np.max(np.abs(g - w)) <= 1e-10 * np.max(np.abs(w))


@pytest.mark.parametrize("scheme", list(SCHEMES))
def test_stage_in_pieces_equals_one_call(scheme):
    """A stage run as 17 + 23 + 1 steps with resume equals 41 steps in one call, bit for bit."""
    comp, mesh, force = stage_case(general=False)
    dt = 0.4 * force.min_critical_dt(scheme)
    n = mesh.num_equations
    mass, cm = dev(mesh.lumped_mass), dev(comp.array("lumped_alpha_mass"))
    pats = motion_patterns(seed=9)
    out = []
    for pieces in ([41], [17, 23, 1]):
        u, v, a = (torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(3))
        gm = fx.GroundMotions(pats)
        t = 0.0
        for i, k in enumerate(pieces):
            t, _ = force.explicit_stage(scheme, mass, u, v, a, dt, k, time=t, motions=gm, alpha_mass=cm,
                                        resume=i > 0)
        out.append((u.cpu().numpy(), v.cpu().numpy(), a.cpu().numpy(), t))
    for x, y in zip(*out):
        assert np.array_equal(x, y)


def test_stage_j2_commits_every_step(oracle_mod):
    """ExplicitDifference on a J2 column under a strong base motion: the device stage (force with
    the committed state, commit after each step) against the same loop on the oracle's J2 force,
    bit for bit, and some points yield."""
    spec = j2_column(lumped=True)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh)
    port = oracle_mod.PortMesh(mesh)
    n = mesh.num_equations
    mass = mesh.lumped_mass
    eq_dof = comp.array("eq_dof").astype(np.int8)
    dt = 0.3 * force.min_critical_dt("ExplicitDifference")
    steps = 60
    amp = 400.0
    pats = [dict(dof=0, fact=amp, values=np.sin(np.linspace(0.0, 3.0, 64)), dt=steps * dt / 40.0)]
    u, v, a = (torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(3))
    force.explicit_stage("ExplicitDifference", dev(mass), u, v, a, dt, steps, motions=fx.GroundMotions(pats))
    # the oracle loop: ed_predict, time += dt, ground motion, J2 force, ed_correct, commit
    mot = oracle_mod.PortMotions(pats)
    committed = port.j2_state()
    uo, vh, ao, vo = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
    t = 0.0
    plastic_any = 0
    for _ in range(steps):
        vh = vh + ao * dt
        uo = uo + vh * dt
        t += dt
        g = mot.evaluate(t)
        f, trial, _, plastic = port.force_j2(committed, uo, vh)
        plastic_any = max(plastic_any, plastic)
        gl = np.where(eq_dof == 0, 0.0 - mass * g[0], 0.0)
        an = (-f + gl) / mass
        vo = vh + (3.0 * an + ao) * (dt * 0.125)
        ao = an
        committed = trial
    assert plastic_any > 0
    assert np.array_equal(u.cpu().numpy(), uo)
    assert np.array_equal(v.cpu().numpy(), vo)
    assert np.array_equal(a.cpu().numpy(), ao)
    assert np.array_equal(force.j2_state("committed"), committed)
