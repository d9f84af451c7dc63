"""The reference-side binding shown in INTEGRATION.md is the file the oracle compiles
(tests/integration/b200_operator.hpp), and, where the build had the reference checkout, that
compiled binding exports its solver driver (no device work: runs without a GPU)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "tests", "integration", "b200_operator.hpp")
ADAPTER = os.path.join(ROOT, "oracle", "_ref", "libfxadapter.so")


def test_integration_notes_show_the_compiled_binding():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    assert open(HEADER).read() in blocks


def test_compiled_binding_exports_its_driver(ref_available):
    if not os.path.exists(ADAPTER):
        pytest.skip("adapter library not built (needs the reference checkout at build time)")
    for src in ("b200_operator.hpp", "reference_cg_driver.cpp"):
        assert os.path.getmtime(ADAPTER) >= os.path.getmtime(os.path.join(ROOT, "tests", "integration", src))
    lib = C.CDLL(ADAPTER)
    assert hasattr(lib, "fxadapt_cg_solve") and hasattr(lib, "fxadapt_last_error")
