"""bench.py's host-side helpers on CPU: the clock summary, the committed ncu
traffic figure and the measured-peaks file (the JSON line's roofline and clocks
come from these)."""
from __future__ import annotations

import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_clock_summary_takes_median_and_active_reasons():
    c = bench.ClockSampler(0)
    c.lines = [
        "0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1320, 1965, 998.7, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1500, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
        "garbage",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    s = c.summary()
    assert s == {"sm_mhz": 1500.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert bench.ClockSampler(0).summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                                               "samples": 0}


def test_committed_traffic_and_peaks_are_read():
    t = bench.ncu_traffic("cholesky")
    assert t is not None and 1e9 < t < 1e11  # one full-size factorization's DRAM bytes
    assert bench.ncu_traffic("no_such_kernel") is None
    peaks = bench.measured_peaks()
    if os.path.exists(os.path.join(REPO, "MEASURED_PEAKS.json")):
        assert peaks["hbm_gbs"] > 0 and peaks["bf16_tflops"] > 0
