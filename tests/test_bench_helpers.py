"""Host helpers of bench.py that shape its JSON line: the roofline's traffic comes from the committed
ncu summary only for the launch shape that summary captured, and the HBM peak names its source."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_traffic_only_for_the_captured_launch():
    b, src = bench.load_traffic(2, 10)
    assert b == 31000064 and "box_apply_layered128" in src
    b, src = bench.load_traffic(3, 8)
    assert b is None and "not the same kernel" in src


def test_peak_names_its_source():
    peak, kind = bench.load_peaks()
    assert peak > 0 and kind in ("measured", "fallback")
    if not os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert (peak, kind) == (6650.0, "fallback")
