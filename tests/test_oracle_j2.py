"""The oracle's J2 restatement (oracle/port/fx_oracle.c). The reference has no J2 material; the
restatement is pinned to the reference's own PressureIndependMultiYield in its two-surface,
pressure-independent form, which under proportional straining is linear kinematic hardening
(stresses equal within 1e-12 through loading and reversal), and checked against its own defining
properties on the CPU:
- after a plastic step the stress lies on the yield surface of the hardened state;
- the returned tangent is the derivative of the stress (central differences, 1e-6);
- at the mesh level the J2 tangent operator is the derivative of the internal force, and with
  `initial` it is the elastic operator.
"""
import ctypes as C

import numpy as np
import pytest

import femorax_b200 as fx
from tests.models_for_tests import j2_column

E, NU, SY, H = 40e6, 0.33, 60e3, 2e6


def point(O, committed, eps, hk=0.5):
    p = O.p_f64
    committed = np.ascontiguousarray(committed, np.float64)
    eps = np.ascontiguousarray(eps, np.float64)
    trial, sigma, D = np.zeros(13), np.zeros(6), np.zeros(36)
    pl = O.port().fxo_j2_update(E, NU, SY, H, hk, committed.ctypes.data_as(p), trial.ctypes.data_as(p),
                                eps.ctypes.data_as(p), sigma.ctypes.data_as(p), D.ctypes.data_as(p))
    return pl, trial, sigma, D.reshape(6, 6)


@pytest.mark.parametrize("hk", [0.0, 0.5, 1.0])
def test_point_on_yield_surface_and_tangent(oracle_mod, hk):
    O = oracle_mod
    rng = np.random.default_rng(int(10 * hk))
    committed = np.zeros(13)
    plastic = 0
    for step in range(6):
        eps = rng.standard_normal(6) * 4e-3
        pl, trial, sigma, D = point(O, committed, eps, hk)
        if not pl:
            committed = trial
            continue
        plastic += 1
        s = sigma.copy()
        s[:3] -= s[:3].mean()
        xi = s - trial[7:]
        norm = np.sqrt(np.sum(xi[:3] ** 2) + 2 * np.sum(xi[3:] ** 2))
        assert norm == pytest.approx(np.sqrt(2 / 3) * (SY + (1 - hk) * H * trial[6]), rel=1e-10)
        h = 1e-9
        for j in range(6):
            de = np.zeros(6)
            de[j] = h
            _, _, sp, _ = point(O, committed, eps + de, hk)
            _, _, sm, _ = point(O, committed, eps - de, hk)
            np.testing.assert_allclose((sp - sm) / (2 * h), D[:, j], rtol=1e-5, atol=1e-6 * np.abs(D).max())
        committed = trial
    assert plastic >= 2


def test_mesh_tangent_is_the_force_derivative(oracle_mod):
    comp = fx.Model(j2_column()).compile()
    mesh = comp.mesh()
    pm = oracle_mod.PortMesh(mesh)
    rng = np.random.default_rng(3)
    n = mesh.num_equations
    u = rng.standard_normal(n) * 2e-3
    v = rng.standard_normal(n) * 1e-3
    f, trial, D, npl = pm.force_j2(pm.j2_state(), u, v)
    assert npl > 0
    x = rng.standard_normal(n)
    y = pm.apply_j2(D, (1.0, 0.0, 0.0), x)
    h = 1e-9
    fp = pm.force_j2(pm.j2_state(), u + h * x, v)[0]
    fm = pm.force_j2(pm.j2_state(), u - h * x, v)[0]
    np.testing.assert_allclose((fp - fm) / (2 * h), y, rtol=1e-4, atol=1e-5 * np.abs(y).max())
    # initial: the elastic operator (K and G of the J2 set equal lame's to rounding)
    ye = pm.apply_j2(D, (1.0, 0.0, 0.0), x, initial=True)
    np.testing.assert_allclose(ye, pm.apply_operator((1.0, 0.0, 0.0), x), rtol=0, atol=1e-12 * np.abs(ye).max())
    # the diagonal is the operator's diagonal
    d = pm.diagonal_j2(D, (1.0, 0.0, 0.0))
    for q in rng.choice(n, 5, replace=False):
        e = np.zeros(n)
        e[q] = 1.0
        assert d[q] == pytest.approx(pm.apply_j2(D, (1.0, 0.0, 0.0), e)[q], rel=1e-12)


@pytest.mark.parametrize("direction", [(0, 0, 0, 1, 0, 0), (0.3, -0.3, 0, 1, 0.5, -0.2)], ids=["simple_shear", "mixed"])
def test_kinematic_j2_pinned_to_reference_two_surface_pimy(direction, oracle_mod, ref_available):
    """The pin of the J2 restatement against the reference: the reference's own
    PressureIndependMultiYield (oracle/_ref), pressure-independent (friction angle 0) with a
    two-point user backbone, is von Mises plasticity with one yield surface and a failure surface;
    under proportional deviatoric straining, as long as the stress stays inside the failure surface,
    it is linear kinematic (Prager) hardening. Backbone: the first point on the elastic line at the
    J2 yield stress in shear, sigma_y / sqrt(3); the segment to the second point with J2's
    elasto-plastic shear modulus G H / (3 G + H) (the reference then sets the plastic modulus
    2 H / 3, Simo-Hughes' kinematic coefficient); the second point far beyond the path. Along a
    monotonic path to ten times the yield strain and a full reversal, the stresses of the J2 return
    map with purely kinematic hardening (hk = 1) equal the reference's within 1e-12 of the largest
    stress."""
    if not ref_available:
        pytest.skip("reference library not built")
    O = oracle_mod
    G0, K0 = 20e6, 50e6
    e_mod, nu = 9 * K0 * G0 / (3 * K0 + G0), (3 * K0 - 2 * G0) / (2 * (3 * K0 + G0))
    tau1 = SY / np.sqrt(3.0)
    g1 = tau1 / G0
    g2 = 60 * g1
    tau2 = tau1 + G0 * H / (3 * G0 + H) * (g2 - g1)
    ref = O.RefPimy((2.0, G0, K0, 10.0, 0.1, 0.0, 100.0, 0.0, 2), (g1, 1.0, g2, tau2 / (G0 * g2)))
    sizes, moduli = ref.setup_values()[1:]
    assert abs(sizes[0] - np.sqrt(3.0) * tau1) <= 1e-9 * sizes[0] and abs(moduli[0] - 2 * H / 3) <= 1e-9 * moduli[0]
    d = np.array(direction, float)
    path = list(np.linspace(0.0, 10 * g1, 41)[1:]) + list(np.linspace(10 * g1, -10 * g1, 81)[1:])
    c_ref, c_j2 = ref.initial_state(), np.zeros(13)
    worst = peak = 0.0
    plastic = 0
    p = O.p_f64
    for gam in path:
        eps = np.ascontiguousarray(gam * d)
        c_ref, s_ref, _ = ref.update(1, c_ref, eps)
        trial, s_j2, D = np.zeros(13), np.zeros(6), np.zeros(36)
        plastic += O.port().fxo_j2_update(e_mod, nu, SY, H, 1.0, np.ascontiguousarray(c_j2).ctypes.data_as(p),
                                          trial.ctypes.data_as(p), eps.ctypes.data_as(p), s_j2.ctypes.data_as(p),
                                          D.ctypes.data_as(p))
        c_j2 = trial
        worst = max(worst, float(np.max(np.abs(s_j2 - s_ref))))
        peak = max(peak, float(np.max(np.abs(s_ref))))
    assert plastic > 60  # most of the path is plastic, on loading and after the reversal
    assert worst <= 1e-12 * peak, worst / peak
