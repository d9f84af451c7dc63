"""The elementary functions of the PressureDependMultiYield device update on a B200: fx_math_eval on
the device gives, bit for bit, fx_math_eval_host's results on 10^7 seeded arguments of each of exp,
log, pow and cos (the functions are built from IEEE-exact operations only; their accuracy and their
agreement with the host C library are tests/test_fx_math.py's)."""
import numpy as np
import pytest

import femorax_b200 as fx

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)
DEV = torch.device("cuda:0")
N = 10_000_000


def arguments(name, seed):
    rng = np.random.default_rng(seed)
    if name == "exp":
        return np.concatenate([rng.uniform(-745, 710, N // 2), rng.uniform(-5, 5, N - N // 2)]), None
    if name == "log":
        return np.concatenate([np.exp(rng.uniform(-744, 709, N // 2)), rng.uniform(0.5, 2.0, N - N // 2)]), None
    if name == "pow":
        return np.exp(rng.uniform(-8, 8, N)), rng.uniform(-4, 4, N)
    return np.concatenate([rng.uniform(-10, 10, N // 2), rng.uniform(-1e5, 1e5, N - N // 2)]), None


@pytest.mark.parametrize("name", ["exp", "log", "pow", "cos"])
def test_device_equals_host(name):
    x, y = arguments(name, 11)
    host = fx.math_eval_host(name, x, y)
    dev = fx.math_eval(name, torch.as_tensor(x, device=DEV), torch.as_tensor(y, device=DEV) if y is not None else None)
    torch.cuda.synchronize()
    d = dev.cpu().numpy()
    same = np.array_equal(d.view(np.int64), host.view(np.int64))
    assert same, (name, int(np.sum(d.view(np.int64) != host.view(np.int64))))
