"""kma_wl_run_noalloc: the allocation-free workload run, for hosts that may
not call cudaMalloc/cudaFree while a batch runs (those calls synchronise the
whole device and a host framework's caching allocator may own the memory
budget).  Its results must equal those of the allocating entry points, on
two calls in a row, since every call reuses the same fixed scratch.

Named test_zz_* so that pytest collects it last; it needs nothing from the
other test files and runs alone as well.
"""
import ctypes
import json
import os

import numpy as np
import pytest

import kma_b200
from kma_b200 import MODE_PLAIN, MODE_WARP, WL_C2, Heap, Workload, _lib
from kma_b200 import inspect as ins

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "workloads.json")))
STAT_KEYS = ["mallocs", "frees", "nulls", "bad_tags", "offset_hash", "fill_bytes", "verify_bytes"]


def seeds_of(seed, items):
    g = np.arange(items, dtype=np.uint64)
    return (np.uint64(seed) ^ (g * np.uint64(0x9E3779B97F4A7C15))).view(np.int64)


def run_noalloc(h, items, seeds_np, rounds, mode, serial):
    """One kma_wl_run_noalloc call through the C ABI; the caller's device
    buffers hold the inputs and outputs."""
    import torch
    seeds = torch.from_numpy(seeds_np).cuda()
    hashes = torch.zeros(items, dtype=torch.int64, device="cuda")
    stats = torch.zeros(7, dtype=torch.int64, device="cuda")
    rc = kma_b200.lib().kma_wl_run_noalloc(h.handle, WL_C2, items, seeds.data_ptr(), rounds, mode,
                                           int(serial), hashes.data_ptr(), stats.data_ptr(), None)
    assert rc == _lib.KMA_OK, kma_b200._lib.strerror(rc)
    torch.cuda.synchronize()
    st = dict(zip(STAT_KEYS, (int(x) for x in stats.cpu().numpy().view(np.uint64))))
    return st, hashes.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("mode", [MODE_PLAIN, MODE_WARP], ids=["plain", "warp"])
def test_noalloc_serial_equals_allocating_path(mode):
    # the golden serial C2 run (2048 items x 64 rounds, 1 GiB heap of 16 KiB
    # superblocks, round-major): same counters and hashes as kma_wl_serial,
    # and as the reference, on two calls in a row
    w = GOLD["c2_round_small"]
    items, rounds = w["items"], w["rounds"]
    sd = seeds_of(w["seed"], items)
    with Heap(w["sblocks"], w["sb_size_log2"]) as h:
        with Workload(h, WL_C2, items) as wl:
            wl.begin(w["seed"])
            wl.serial(rounds, True, mode)
            want = wl.stats()
        for _ in range(2):
            got, hashes = run_noalloc(h, items, sd, rounds, mode, serial=True)
            assert got == {k: int(want[k]) for k in STAT_KEYS}
            assert {k: got[k] for k in w["stats"]} == w["stats"]
            assert int(np.bitwise_xor.reduce(hashes)) == got["offset_hash"]
            assert ins.check_canonical_empty(h.snapshot(), h.bitmaps()) == []
        assert h.error_flags() == 0


def test_noalloc_concurrent_equals_allocating_path():
    # the largest batch the fixed scratch takes, concurrent warp-collaborative
    # rounds: the counters (exact when no malloc returns NULL) equal the
    # allocating kma_wl_run_host's, on two calls in a row
    import torch
    items = _lib_max_items()
    sd = seeds_of(0xA11C, items)
    with Heap(65536, 14) as h:
        with Workload(h, WL_C2, items) as wl:
            seeds_host = torch.from_numpy(sd.copy()).pin_memory()
            hashes_host = torch.zeros(items, dtype=torch.int64).pin_memory()
            want = wl.run_host(seeds_host.data_ptr(), 64, MODE_WARP, hashes_host.data_ptr())
        assert want["nulls"] == 0 and want["bad_tags"] == 0
        for _ in range(2):
            got, hashes = run_noalloc(h, items, sd, 64, MODE_WARP, serial=False)
            for k in ("mallocs", "frees", "nulls", "bad_tags", "fill_bytes", "verify_bytes"):
                assert got[k] == want[k], k
            assert int(np.bitwise_xor.reduce(hashes)) == got["offset_hash"]
            assert ins.check_canonical_empty(h.snapshot(), h.bitmaps()) == []
        assert h.error_flags() == 0


def test_noalloc_rejects_more_items_than_its_scratch():
    import torch
    n = _lib_max_items() + 1
    buf = torch.zeros(n, dtype=torch.int64, device="cuda")
    st = torch.zeros(7, dtype=torch.int64, device="cuda")
    with Heap(64, 12) as h:
        rc = kma_b200.lib().kma_wl_run_noalloc(h.handle, WL_C2, n, buf.data_ptr(), 4, MODE_WARP, 0,
                                               buf.data_ptr(), st.data_ptr(), None)
        assert rc == _lib.KMA_EINVAL


def _lib_max_items():
    # KMA_WL_NOALLOC_MAX_ITEMS in include/kma.h
    import re
    src = open(os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "kma.h")).read()
    return int(re.search(r"#define KMA_WL_NOALLOC_MAX_ITEMS (\d+)", src).group(1))
