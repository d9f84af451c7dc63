"""The oracle's J2 restatement (oracle/port/fx_oracle.c): it has no counterpart in the reference
(parity unpinned), so it is checked against its own defining properties on the CPU:
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
