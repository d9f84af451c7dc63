import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    if not os.path.exists(O.PORT_LIB):
        O.build("")
    return O


@pytest.fixture(scope="session")
def ref_available(oracle_mod):
    return oracle_mod.have_ref()
