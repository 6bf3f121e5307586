"""The copy roofline (src/bench.ts:61-95 method) on the device: a plausible stream rate."""
import json
import os

import pytest

import bench

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp16", "fp64"])
def test_copy_roofline_rate_is_plausible(precision):
    n = 192 * 96 * 96
    r = bench.copy_roofline(0, precision, n, launches=50)
    peak = 8000.0
    path = os.path.join(os.path.dirname(os.path.dirname(__file__)), "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            peak = float(json.load(f).get("hbm_gbs", peak))
    # a 19-array copy of 134-537 MB streams from HBM: between a third of the copy peak and a bit above it
    assert peak / 3 < r["gbps"] < 1.15 * peak, r
