"""PressureIndependMultiYield material points on the CPU.

- the oracle (the reference's own material, compiled from its sources in oracle/_ref) reproduces
  every stored OpenSees path (tests/golden/pimy_paths.npz, 34 strain paths: hyperbolic and user
  backbones, friction angle zero and 30 degrees, stage switches, discarded trials, confinement
  changes, tension) bit for bit: the pin;
- this library's restatement (fx_pimy_*_host, the same arithmetic as the device kernel) gives the
  same setup (surface sizes, moduli, residual pressure, friction angle, cohesion) as the oracle
  and, along every path, OpenSees' stress and tangent within 1e-14 of the path's largest value
  (the reference's own tolerance, tests/unit/test_pimy_reference.cpp:33), bit for bit where the
  arithmetic agrees;
- many points at once: each point the same as alone; a commit is a swap of the two buffers.
"""
import os

import numpy as np
import pytest

import femorax_b200 as fx

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "pimy_paths.npz"))
CASES = list(GOLDEN["cases"])
TOL = 1e-14


def material(name):
    p = GOLDEN[name + "/params"]
    pairs = GOLDEN[name + "/pairs"]
    return fx.PressureIndependMultiYield(*p[:8], noYieldSurf=int(p[8]), pairs=pairs if pairs.size else None)


def replay_host(m, stage, pre, pre_eps, eps, copies=1):
    """A path on `copies` identical points: per step the stage, the discarded trial, the update and
    the commit (a swap). Stresses [n, 6], tangents [n, 6, 6] of point 0, and whether all points agree."""
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
        bad = m.update_host(int(stage[k]), c, t, np.ascontiguousarray(np.repeat(eps[k][:, None], copies, 1)), s, d)
        assert bad == 0
        sig[k], D[k] = s[:, 0], d[:, 0].reshape(6, 6)
        same = same and all(np.array_equal(s[:, 0], s[:, j]) and np.array_equal(d[:, 0], d[:, j])
                            for j in range(1, copies))
        c, t = t, c
    return sig, D, same


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_oracle_pinned_to_opensees(oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("the reference build is not available")
    for name in CASES:
        g = {k: GOLDEN[name + "/" + k] for k in ("params", "pairs", "stage", "pre", "pre_eps", "eps", "sig", "D")}
        m = oracle_mod.RefPimy(g["params"], g["pairs"])
        sig, D = m.replay(g["stage"], g["pre"], g["pre_eps"], g["eps"])
        assert np.array_equal(sig, g["sig"]) and np.array_equal(D, g["D"]), name


@pytest.mark.parametrize("name", CASES)
def test_setup_matches_oracle(name, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("the reference build is not available")
    m = material(name)
    r = oracle_mod.RefPimy(GOLDEN[name + "/params"], GOLDEN[name + "/pairs"])
    a, sz, hm = m.setup_values()
    b, sz2, hm2 = r.setup_values()
    assert np.array_equal(a, b) and np.array_equal(sz, sz2) and np.array_equal(hm, hm2)
    assert m.nstate == 31 + 8 * int(GOLDEN[name + "/params"][8])


@pytest.mark.parametrize("name", CASES)
def test_paths_match_opensees(name):
    g = {k: GOLDEN[name + "/" + k] for k in ("stage", "pre", "pre_eps", "eps", "sig", "D")}
    sig, D, same = replay_host(material(name), g["stage"], g["pre"], g["pre_eps"], g["eps"], copies=3)
    assert same
    assert rel(sig, g["sig"]) <= TOL and rel(D, g["D"]) <= TOL, name
    assert np.array_equal(sig, g["sig"]) and np.array_equal(D, g["D"]), "not bit for bit: " + name


def test_rejected_inputs():
    with pytest.raises(fx.FxError) as e:
        fx.PressureIndependMultiYield(1.8, 40500, 108000, 10, 0.1, 0, 100, 0, 41)
    assert e.value.code == 2
    with pytest.raises(fx.FxError):
        fx.PressureIndependMultiYield(1.8, -1.0, 108000, 10, 0.1, 0, 100, 0, 20)
    with pytest.raises(fx.FxError):
        fx.PressureIndependMultiYield(1.8, 40500, 108000, 0.0, 0.1, 0.0, 100, 0, 20)  # no strength
