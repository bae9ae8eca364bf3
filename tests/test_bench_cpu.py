"""The bench's CPU baseline leg (no GPU): the reference's kma.cl as host C
on all host threads and on one thread, each on a bounded sample of the
config-2 work-items."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_cpu_baseline_reports_all_threads_and_one_thread():
    c = bench.measure_cpu_baseline()
    assert c["value"] and c["value"] > 0, c
    assert c["cores"] == (os.cpu_count() or 1)
    assert c["kind"] in ("reference", "port")
    one = c["one_thread"]
    assert one["value"] and one["value"] > 0, one
    assert "1 thread" in one["sample"]
