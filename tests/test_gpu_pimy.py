"""PressureIndependMultiYield material points on a B200 (fx_pimy_update), against OpenSees' stored
paths and against this library's host restatement (the same arithmetic, which tests/test_pimy.py
shows equal to OpenSees bit for bit):

- every stored path (tests/golden/pimy_paths.npz) on 64 identical points: OpenSees' stress and
  tangent within 1e-14 of the path's largest value (the reference's tolerance), every point the
  same; bit for bit with the host where the path never calls pow (friction angle 0: the switch to
  the plastic stage scales nothing); with a friction angle the device's pow may differ from the
  host's in the last place;
- 20,000 points on distinct seeded strain paths (cyclic shear of random amplitude and direction on a
  random confinement, the stage switched after 4 steps): the device against the host point by
  point, no failed points; a commit is a swap of the buffers.
"""
import os

import numpy as np
import pytest

import femorax_b200 as fx

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")
GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "pimy_paths.npz"))
CASES = list(GOLDEN["cases"])


def material(name):
    p = GOLDEN[name + "/params"]
    pairs = GOLDEN[name + "/pairs"]
    return fx.PressureIndependMultiYield(*p[:8], noYieldSurf=int(p[8]), pairs=pairs if pairs.size else None)


def col(v, n):
    return torch.as_tensor(np.repeat(np.asarray(v)[:, None], n, 1), dtype=torch.float64, device=DEV).contiguous()


@pytest.mark.parametrize("name", CASES)
def test_path_on_device(name):
    g = {k: GOLDEN[name + "/" + k] for k in ("params", "stage", "pre", "pre_eps", "eps", "sig", "D")}
    m = material(name)
    n = 64
    c, t = m.initial_state(n, 0), torch.empty((m.nstate, n), dtype=torch.float64, device=DEV)
    s = torch.empty((6, n), dtype=torch.float64, device=DEV)
    d = torch.empty((36, n), dtype=torch.float64, device=DEV)
    failed = torch.zeros(1, dtype=torch.int32, device=DEV)
    hc, ht = m.initial_state(1), np.zeros((m.nstate, 1))
    hs, hd = np.zeros((6, 1)), np.zeros((36, 1))
    sig, D = [], []
    bitwise = True
    for k in range(len(g["eps"])):
        st = int(g["stage"][k])
        if g["pre"][k]:
            m.update(st, c, t, col(g["pre_eps"][k], n), s, d, failed)
        m.update(st, c, t, col(g["eps"][k], n), s, d, failed)
        m.update_host(st, hc, ht, np.ascontiguousarray(g["eps"][k][:, None]), hs, hd)
        ss, dd = s.cpu().numpy(), d.cpu().numpy()
        assert all(np.array_equal(ss[:, 0], ss[:, j]) and np.array_equal(dd[:, 0], dd[:, j]) for j in range(1, n))
        sig.append(ss[:, 0])
        D.append(dd[:, 0].reshape(6, 6))
        bitwise = bitwise and np.array_equal(ss[:, :1], hs) and np.array_equal(dd[:, :1], hd)
        c, t = t, c
        hc, ht = ht, hc
    sig, D = np.array(sig), np.array(D)
    assert int(failed.item()) == 0
    for got, want in ((sig, g["sig"]), (D, g["D"])):
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) <= 1e-14, name
    if g["params"][5] == 0.0:
        assert bitwise, name


@pytest.mark.parametrize("name", ["basin_clay_cyclic_1e-2_150", "frictional_cyclic_1e-2_150",
                                  "backbone_frictional_random_reversals_150"])
def test_many_points_equal_host(name):
    m = material(name)
    n, steps = 20000, 24
    rng = np.random.default_rng(3)
    amp = rng.uniform(2e-4, 2e-2, n)
    direction = rng.standard_normal((3, n))
    direction /= np.linalg.norm(direction, axis=0)
    conf = rng.uniform(-2e-3, -5e-4, n)  # volumetric strain at the switch (compression)
    c, t = m.initial_state(n, 0), torch.empty((m.nstate, n), dtype=torch.float64, device=DEV)
    hc, ht = m.initial_state(n), np.zeros((m.nstate, n))
    s = torch.empty((6, n), dtype=torch.float64, device=DEV)
    d = torch.empty((36, n), dtype=torch.float64, device=DEV)
    hs, hd = np.zeros((6, n)), np.zeros((36, n))
    failed = torch.zeros(1, dtype=torch.int32, device=DEV)
    worst = 0.0
    for k in range(steps):
        stage = 0 if k < 4 else 1
        e = np.zeros((6, n))
        e[0:3] = conf * min(k + 1, 4) / 4 / 3
        ph = np.sin(2 * np.pi * max(k - 4, 0) / 10)
        e[3:6] = amp * ph * direction
        e = np.ascontiguousarray(e)
        m.update(stage, c, t, torch.as_tensor(e, device=DEV), s, d, failed)
        bad = m.update_host(stage, hc, ht, e, hs, hd)
        assert bad == 0
        ss, dd = s.cpu().numpy(), d.cpu().numpy()
        scale_s, scale_d = np.max(np.abs(hs)), np.max(np.abs(hd))
        worst = max(worst, np.max(np.abs(ss - hs)) / scale_s, np.max(np.abs(dd - hd)) / scale_d)
        if m.setup_values()[0][1] == 0.0:
            assert np.array_equal(ss, hs) and np.array_equal(dd, hd), k
        c, t = t, c
        hc, ht = ht, hc
    assert int(failed.item()) == 0
    assert worst <= 1e-12, worst
    assert np.allclose(c.cpu().numpy(), hc, rtol=1e-12, atol=1e-12 * np.max(np.abs(hc)))
