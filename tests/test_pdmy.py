"""PressureDependMultiYield material points on the CPU.

- the oracle (the reference's own material, compiled from its sources in oracle/_ref) reproduces
  every stored OpenSees path (tests/golden/pdmy_paths.npz, 32 strain paths of dense and loose sands,
  hyperbolic and user backbones, with and without the phase-transformation zone: cyclic, monotonic,
  random reversals, stage switches, confinement changes, tension) bit for bit: the pin;
- this library's restatement (fx_pdmy_*_host, the same arithmetic as the device kernel) gives the
  oracle's setup and, along every path, OpenSees' stress and tangent within 1e-14 of the path's
  largest value (the reference's own tolerance, tests/unit/test_pdmy_reference.cpp), bit for bit;
- many identical points at once give identical results.
"""
import os

import numpy as np
import pytest

import femorax_b200 as fx

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "pdmy_paths.npz"))
CASES = list(GOLDEN["cases"])


def material(name):
    p = GOLDEN[name + "/params"]
    pairs = GOLDEN[name + "/pairs"]
    return fx.PressureDependMultiYield(*p[:14], noYieldSurf=int(p[14]), pairs=pairs if pairs.size else None,
                                       e=p[15], cs1=p[16], cs2=p[17], cs3=p[18], pa=p[19], c=p[20])


def replay_host(m, stage, pre, pre_eps, eps, copies=1):
    n = len(eps)
    c = m.initial_state(copies)
    t = np.zeros_like(c)
    sig, D = np.zeros((n, 6)), np.zeros((n, 6, 6))
    same = True
    for k in range(n):
        s = np.zeros((6, copies))
        d = np.zeros((36, copies))
        if pre[k]:
            m.update_host(int(stage[k]), c, t, np.ascontiguousarray(np.repeat(pre_eps[k][:, None], copies, 1)), s, d)
        assert m.update_host(int(stage[k]), c, t, np.ascontiguousarray(np.repeat(eps[k][:, None], copies, 1)), s, d) == 0
        sig[k], D[k] = s[:, 0], d[:, 0].reshape(6, 6)
        same = same and all(np.array_equal(s[:, 0], s[:, j]) and np.array_equal(d[:, 0], d[:, j])
                            for j in range(1, copies))
        c, t = t, c
    return sig, D, same


def test_oracle_pinned_to_opensees(oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("the reference build is not available")
    for name in CASES:
        g = {k: GOLDEN[name + "/" + k] for k in ("params", "pairs", "stage", "pre", "pre_eps", "eps", "sig", "D")}
        m = oracle_mod.RefPdmy(np.concatenate([g["params"], [0.0, 1.0]]), g["pairs"])
        sig, D = m.replay(g["stage"], g["pre"], g["pre_eps"], g["eps"])
        assert np.array_equal(sig, g["sig"]) and np.array_equal(D, g["D"]), name


@pytest.mark.parametrize("name", CASES)
def test_setup_matches_oracle(name, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("the reference build is not available")
    m = material(name)
    r = oracle_mod.RefPdmy(np.concatenate([GOLDEN[name + "/params"], [0.0, 1.0]]), GOLDEN[name + "/pairs"])
    for a, b in zip(m.setup_values(), r.setup_values()):
        assert np.array_equal(a, b)
    assert m.nstate == 89 + 6 * int(GOLDEN[name + "/params"][14])


@pytest.mark.parametrize("name", CASES)
def test_paths_match_opensees(name):
    g = {k: GOLDEN[name + "/" + k] for k in ("stage", "pre", "pre_eps", "eps", "sig", "D")}
    sig, D, same = replay_host(material(name), g["stage"], g["pre"], g["pre_eps"], g["eps"], copies=2)
    assert same
    for got, want in ((sig, g["sig"]), (D, g["D"])):
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) <= 1e-14, name
    assert np.array_equal(sig, g["sig"]) and np.array_equal(D, g["D"]), "not bit for bit: " + name


def test_inputs_reset_or_rejected():
    # OpenSees clamps the surfaces to 40 and the phase-transformation angle to the friction angle
    m = fx.PressureDependMultiYield(2.0, 1e5, 2e5, 35, 0.1, 80, 0.5, 37, 0.05, 0.6, 3, 10, 0.02, 1, noYieldSurf=41)
    assert m.surfaces == 40 and m.setup_values()[0][2] == 35.0
    with pytest.raises(fx.FxError):
        fx.PressureDependMultiYield(2.0, 1e5, 2e5, 0.0, 0.1, 80, 0.5, 27, 0.05, 0.6, 3, 10, 0.02, 1)  # no friction
