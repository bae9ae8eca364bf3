"""GPU parity: the CUDA heap through the C ABI against the oracle.

Serial replay (one op at a time, plain and warp-collaborative paths) must
return the reference's offsets bit for bit and leave the same decoded heap
and the same superblock bytes; the stress programs run serially must
reproduce the reference's counters and hashes, and run concurrently must
keep every heap invariant and return to the canonical empty state.
"""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

import kma_b200
from kma_b200 import MODE_PLAIN, MODE_WARP, WL_C1, WL_C2, Heap, Workload
from kma_b200 import inspect as ins
from opstream import drain_stream, make_stream
from oracle import oracle

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REPLAYS = sorted(glob.glob(os.path.join(GOLD, "replay_*.npz")))
WORKLOADS = json.load(open(os.path.join(GOLD, "workloads.json")))
MODES = [MODE_PLAIN, MODE_WARP]
MODE_IDS = ["plain", "warp"]
# heap structures: the reference's (one class table, tagged-CAS MS queue),
# the default (ticket-ring free list, shards by size), and 8 shards forced
HEAPS = [dict(compat=True), dict(), dict(shards=8)]
HEAP_IDS = ["compat", "default", "shards8"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def assert_canon(canon, want):
    assert np.array_equal(canon.cls, np.asarray(want["cls"])), "class table"
    assert np.array_equal(canon.sb_size, np.asarray(want["sb_size"])), "superblock sizes"
    assert np.array_equal(canon.sb_slots, np.asarray(want["sb_slots"])), "slots"
    assert np.array_equal(canon.sb_free, np.asarray(want["sb_free"])), "free counts"
    assert np.array_equal(canon.freelist, np.asarray(want["freelist"])), "free-list order"


def test_create_matches_reference_initial_state():
    with Heap(64, 12) as h, oracle.Port(64, 12) as p:
        img = h.snapshot(region=True)
        assert_canon(ins.decode(img), p.decode())
        assert ins.check_canonical_empty(img) == []
        assert h.error_flags() == 0


@pytest.mark.parametrize("heap", HEAPS, ids=HEAP_IDS)
@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("path", REPLAYS, ids=os.path.basename)
def test_replay_matches_golden(path, mode, heap):
    g = np.load(path)
    log2 = int(os.path.basename(path).split("_")[1])
    with Heap(int(g["sblocks"]), log2, **heap) as h:
        out = h.replay(g["ops"], mode)
        assert np.array_equal(out, g["out"]), np.nonzero(out != g["out"])[0][:5]
        canon = ins.decode(h.snapshot(region=True))
        assert_canon(canon, g)
        assert digest(canon.region) == str(g["region_sha256"])
        assert h.error_flags() == 0


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("log2,sblocks,seed", [(12, 33, 21), (12, 300, 22), (14, 11, 23),
                                               (16, 7, 24), (12, 2, 25), (12, 3, 26)])
@pytest.mark.parametrize("heap", HEAPS[:2], ids=HEAP_IDS[:2])
def test_replay_matches_port_live(log2, sblocks, seed, mode, heap):
    ops = drain_stream(make_stream(seed, 2500, log2))
    with Heap(sblocks, log2, **heap) as h, oracle.Port(sblocks, log2) as p:
        want = p.replay(ops)
        got = h.replay(ops, mode)
        assert np.array_equal(got, want)
        canon = ins.decode(h.snapshot(region=True))
        assert_canon(canon, p.decode())
        assert np.array_equal(canon.region, p.region())


@pytest.mark.parametrize("heap", HEAPS[:2], ids=HEAP_IDS[:2])
def test_replay_beyond_reference_index_limit(heap):
    # 70 000 superblocks: past the reference's 16-bit queue index; the port
    # (widened index) is the oracle here
    sblocks = 70000
    n = 2 * sblocks
    ops = np.zeros((2 * n, 2), np.int64)
    ops[:n, 0], ops[:n, 1] = 0, 2000
    ops[n:, 0], ops[n:, 1] = 1, np.arange(n)
    with Heap(sblocks, 12, **heap) as h, oracle.Port(sblocks, 12) as p:
        assert np.array_equal(h.replay(ops), p.replay(ops))
        assert_canon(ins.decode(h.snapshot()), p.decode())


def test_reset_restores_initial_state():
    ops = make_stream(31, 1500, 12)
    with Heap(48, 12) as h:
        h.replay(ops)
        h.reset()
        img = h.snapshot(region=False)
        with oracle.Port(48, 12) as p:
            assert_canon(ins.decode(img), p.decode())
        # and the heap behaves like a fresh one
        with oracle.Port(48, 12) as p:
            assert np.array_equal(h.replay(ops), p.replay(ops))


@pytest.mark.parametrize("heap", HEAPS[:2], ids=HEAP_IDS[:2])
@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("name", sorted(WORKLOADS))
def test_serial_workload_matches_golden(name, mode, heap):
    w = WORKLOADS[name]
    with Heap(w["sblocks"], w["sb_size_log2"], **heap) as h, \
            Workload(h, w["program"], w["items"]) as wl:
        wl.begin(w["seed"])
        wl.serial(w["rounds"], bool(w["round_major"]), mode)
        st = wl.stats()
        assert {k: st[k] for k in w["stats"]} == w["stats"]
        canon = ins.decode(h.snapshot())
        assert len(canon.freelist) == w["freelist_len"]
        assert digest(canon.freelist) == w["freelist_sha256"]
        assert h.error_flags() == 0


@pytest.mark.parametrize("heap", HEAPS, ids=HEAP_IDS)
@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_c1_concurrent(mode, heap):
    # config 1: 16 MiB heap of 4 KiB superblocks, 4 x 64 items, 16 rounds
    with Heap(4096, 12, **heap) as h, Workload(h, WL_C1, 256) as wl:
        wl.begin(0xC1)
        wl.rounds(16, mode, block_dim=64)
        st = wl.stats()
        assert st["mallocs"] == 4096 and st["frees"] == 4096
        assert st["nulls"] == 0 and st["bad_tags"] == 0
        img = h.snapshot()
        assert ins.check_canonical_empty(img, h.bitmaps()) == []
        assert h.error_flags() == 0


@pytest.mark.parametrize("mode,heap", [(MODE_PLAIN, dict(compat=True)), (MODE_PLAIN, dict()),
                                       (MODE_WARP, dict(compat=True)), (MODE_WARP, dict())],
                         ids=["plain-compat", "plain-default", "warp-compat", "warp-default"])
def test_c2_full_size_invariants(mode, heap):
    # config 2: 1 GiB heap of 16 KiB superblocks, 148 x 2048 items, 64 rounds
    items = 148 * 2048
    with Heap(65536, 14, **heap) as h, Workload(h, WL_C2, items) as wl:
        wl.begin(0xC2)
        wl.rounds(64, mode)
        st = wl.stats()
        assert st["bad_tags"] == 0 and st["mallocs"] == items * 64
        if not h.compat:
            # NULL returns are legal (exhaustion) and timing-dependent: the
            # reference never re-attaches a partly free superblock, so items
            # that progress unevenly pin superblocks longer.  The scalable
            # heap keeps them rare; the reference's structures starve threads
            # under this contention and fragment far more.
            assert st["nulls"] <= st["mallocs"] // 20
        nlive, off, size = wl.live()
        sel = np.arange(off.shape[0])[:, None] < nlive[None, :]
        live_off, live_size = off[sel], size[sel]
        assert len(live_off) == st["mallocs"] - st["nulls"] - st["frees"]
        img = h.snapshot()
        res = ins.check_live_blocks(img, live_off, live_size, h.bitmaps())
        assert ins.violations(res) == 0, res
        # per superblock: allocated bits == slots - free for in-use superblocks
        wl.drain(mode)
        st = wl.stats()
        assert st["bad_tags"] == 0 and st["frees"] == st["mallocs"] - st["nulls"]
        img = h.snapshot()
        flags = h.error_flags()
        assert ins.check_canonical_empty(img, h.bitmaps()) == [], f"error flags {flags}"
        assert not flags & kma_b200.KMA_FLAG_BADFREE
        # the warp path gives up only on a spin limit, and none is reached
        # here; the plain path on the single-queue heap may starve a thread
        if not h.compat or mode == MODE_WARP:
            assert flags == 0


def test_double_free_is_refused_not_corrupting():
    ops = np.array([[0, 64], [0, 64], [1, 0], [1, 0], [1, 1]], np.int64)
    for mode, heap in zip(MODES * 2, [HEAPS[0]] * 2 + [HEAPS[1]] * 2):
        with Heap(16, 12, **heap) as h:
            h.replay(ops, mode)
            assert h.error_flags(clear=True) & kma_b200.KMA_FLAG_BADFREE
            img = h.snapshot()
            assert ins.check_canonical_empty(img, h.bitmaps()) == []


@pytest.mark.parametrize("heap", HEAPS, ids=HEAP_IDS)
@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_stale_class_slot_is_cleared_not_waited_on(mode, heap):
    # a class slot naming a superblock that cannot serve the class (here one
    # formatted for another class; concurrently, one whose last slots were
    # taken through another shard's slot after a recycle): the request
    # clears the slot and refills instead of waiting out the spin limit
    with Heap(32, 12, spin_limit=2000, **heap) as h:
        a = h.replay(np.array([[0, 8]], np.int64), mode)  # a class-1 superblock
        assert a[0] >= 0
        s = int(a[0]) >> 12
        h.debug_set_class_word(2, s + 2)  # KMA_CLS_BASE + s, in every shard
        out = h.replay(np.array([[0, 16], [0, 16], [1, 0], [1, 1]], np.int64), mode)
        assert (out[:2] >= 0).all()
        assert ((out[:2] >> 12) != s).all()
        assert h.error_flags() == 0


def test_bounded_wait_times_out_without_fault():
    # a class word stuck at POISON (nothing will clear it): every request
    # of that class gives up after spin_limit iterations and returns NULL
    for mode, heap in zip(MODES * 2, [HEAPS[0]] * 2 + [HEAPS[2]] * 2):
        with Heap(32, 12, spin_limit=2000, **heap) as h:
            h.debug_set_class_word(2, 1)
            out = h.replay(np.array([[0, 16], [0, 8]], np.int64), mode)
            assert out[0] == -1  # class 2 (16 B): timed out
            assert out[1] >= 0   # class 1 unaffected
            flags = h.error_flags()
            assert flags & kma_b200.KMA_FLAG_TIMEOUT
            # and the flags name the wait: the per-thread reservation, or
            # the warp path's reservation (KMA_ERR_AT_MALLOC / _AT_RESERVE)
            assert flags & ((1 << 13) if mode == MODE_PLAIN else (1 << 15))
