"""Host-side helpers of bench.py: the CPU-baseline sample sizing, the
whole-job rate and the algorithmic byte model of the roofline."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_scaled_sample_targets_seconds_and_caps_at_the_workload():
    wl = bench.WORKLOADS["ns"]
    # 200k reads with 120 k-mers each at 80 M k-mers/s -> 10 s is 6.67 M reads
    n = bench.scaled_sample(wl, 200_000, 24_000_000, 80e6, 10.0)
    assert n == pytest.approx(80e6 * 10 / 120, rel=1e-6)
    assert bench.scaled_sample(wl, 200_000, 24_000_000, 1e12, 10.0) == 20_000_000  # all reads of the workload
    assert bench.scaled_sample(wl, 200_000, 24_000_000, 1.0, 10.0) == 200_000     # never below the calibration
    assert bench.scaled_sample(bench.WORKLOADS["config1"], 100, 12_000, 1e12, 10.0) == 20_000


def test_whole_job_rate_counts_every_rank():
    assert bench.whole_job_rate(100, 4, 2, 1000.0) == pytest.approx(800.0)


def test_byte_model_at_ns():
    m = bench.algorithmic_bytes(3.0e9, 2e7, 2.28e8, 2.4e9, 4.36e8, 31)
    assert m["w"] == 8 and m["P"] == 8
    assert m["sort"] == pytest.approx(8 * 2.4e9 * (1 + 2 * 8))
    assert m["count"] == pytest.approx(8 * 2.4e9 + 12 * 4.36e8)
    assert m["total"] == pytest.approx(m["partition"] + m["expand"] + m["sort"] + m["count"])
    assert bench.algorithmic_bytes(1, 1, 1, 1, 1, 63)["w"] == 16
