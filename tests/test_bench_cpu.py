"""The bench's CPU baseline leg (no GPU): the reference's kma.cl as host C
on all host threads and on one thread, each over the same sample of the
config-2 work-items (a small one here, so the suite stays quick)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from oracle import oracle  # noqa: E402


@pytest.mark.skipif(not (oracle.ref_available(bench.SB_LOG2) or os.path.exists(oracle.PORT_LIB)),
                    reason="oracle libraries not built (make -C oracle)")
def test_cpu_baseline_reports_all_threads_and_one_thread():
    items = 2048
    c = bench.measure_cpu_baseline(items=items)
    assert c["value"] and c["value"] > 0, c
    assert c["cores"] == (os.cpu_count() or 1)
    assert c["kind"] in ("reference", "port")
    one = c["one_thread"]
    assert one["value"] and one["value"] > 0, one
    assert one["cores"] == 1
    # both legs cover the same work-items
    assert f"{items} of the {bench.ITEMS} work-items" in c["sample"]
    assert f"{items} of the {bench.ITEMS} work-items" in one["sample"]
    assert "1 pthread," in one["sample"]
