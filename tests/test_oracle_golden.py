"""The oracle against the reference's stored OpenSees Brick data (tests/golden/brick_elements.npz,
from tests/reference/data/element/Brick_*), at the reference's own tolerance: relative 1e-12 of
the largest entry (tests/unit/test_std_brick_reference.cpp:28)."""
import os

import numpy as np
import pytest

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "brick_elements.npz"))
CASES = [str(c) for c in GOLD["cases"]]
TOL = 1e-12


def row(case, mass_type, body=True):
    E, nu, rho = GOLD[case + "/material"]
    b = GOLD[case + "/body"] if body else np.zeros(3)
    return [0, mass_type, E, nu, rho, b[0], b[1], b[2], 0, 0, 0, 0, 0, 0, 0]


def close(got, want):
    scale = np.max(np.abs(want))
    return np.max(np.abs(got - want)) <= TOL * scale


@pytest.mark.parametrize("case", CASES)
def test_force_and_tangent(case, oracle_mod):
    xe = GOLD[case + "/coords"].reshape(-1)
    for f in range(GOLD[case + "/u"].shape[0]):
        fe, Ke = oracle_mod.port_brick_compute(row(case, 0), (0, 0, 0, 0), xe, GOLD[case + "/u"][f], GOLD[case + "/v"][f])
        assert close(fe, GOLD[case + "/f"][f]), (case, f)
        assert close(Ke, GOLD[case + "/K"][f]), (case, f)


@pytest.mark.parametrize("case", CASES)
def test_damping_forces(case, oracle_mod):
    xe = GOLD[case + "/coords"].reshape(-1)
    ray = tuple(GOLD[case + "/rayleigh"])
    for f in range(GOLD[case + "/u"].shape[0]):
        v = GOLD[case + "/v"][f]
        dc, _ = oracle_mod.port_brick_compute(row(case, 0, body=False), ray, xe, np.zeros(24), v, want_k=False)
        dl, _ = oracle_mod.port_brick_compute(row(case, 1, body=False), ray, xe, np.zeros(24), v, want_k=False)
        assert close(dc, GOLD[case + "/dc"][f]), (case, f)
        assert close(dl, GOLD[case + "/dl"][f]), (case, f)


@pytest.mark.parametrize("case", CASES)
def test_mass(case, oracle_mod):
    xe = GOLD[case + "/coords"].reshape(-1)
    assert close(oracle_mod.port_brick_mass(row(case, 0), xe), GOLD[case + "/Mc"])
    assert close(oracle_mod.port_brick_mass(row(case, 1), xe), GOLD[case + "/Ml"])


@pytest.mark.parametrize("case", CASES)
def test_operator_is_tangent_times_x(case, oracle_mod):
    """element_operator_apply with k = (1, 0, 0) is K x (the golden K), k = (0, 0, 1) is M x."""
    xe = GOLD[case + "/coords"].reshape(-1)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(24)
    K = GOLD[case + "/K"][0]
    assert close(oracle_mod.port_brick_operator(row(case, 0), (0, 0, 0, 0), (1, 0, 0), xe, x), K @ x)
    assert close(oracle_mod.port_brick_operator(row(case, 0), (0, 0, 0, 0), (0, 0, 1), xe, x), GOLD[case + "/Mc"] @ x)
    assert close(oracle_mod.port_brick_operator(row(case, 1), (0, 0, 0, 0), (0, 0, 1), xe, x), GOLD[case + "/Ml"] @ x)
