"""Heap images on the GPU: kma_image_save / kma_image_load through the C ABI.

A saved image decodes to the same state kma_snapshot reports; loaded into
another heap of the same geometry (another allocation, so another device
address) it makes that heap continue exactly as the saved one would:
the same offsets for the same requests, the same final bytes.  Images of
other geometry, truncated ones and ones holding words that would address
outside the heap are refused, leaving the target unchanged.
"""
import numpy as np
import pytest
import torch

from kma_b200 import MODE_PLAIN, MODE_WARP, Heap, KmaError
from kma_b200 import inspect as ins
from opstream import make_stream

pytestmark = pytest.mark.gpu

HEAPS = [dict(compat=True), dict(), dict(shards=8)]
HEAP_IDS = ["compat", "default", "shards8"]
EINVAL = -1


def full_state(h):
    img = h.snapshot(region=True)
    return img.cls_raw.copy(), img.state.copy(), img.freelist.copy(), img.region.copy()


def assert_same_state(a, b):
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("heap", HEAPS, ids=HEAP_IDS)
@pytest.mark.parametrize("mode", [MODE_PLAIN, MODE_WARP], ids=["plain", "warp"])
def test_image_round_trip_continues_identically(mode, heap):
    first = make_stream(71, 900, 12)
    cont = make_stream(72, 900, 12)
    with Heap(64, 12, **heap) as a, Heap(64, 12, **heap) as b:
        a.replay(first, mode)  # leaves live blocks, a partial free list
        img = a.image_save()
        assert img.nbytes == a.image_bytes()
        # the image decodes to what the snapshot reports
        snap = a.snapshot(region=True)
        dec = ins.image_from_bytes(img, a.cls_size, a.cls_slots)
        ca, cb = ins.decode(snap), ins.decode(dec)
        for f in ("cls", "sb_size", "sb_slots", "sb_free", "freelist", "region"):
            assert np.array_equal(getattr(ca, f), getattr(cb, f)), f
        b.image_load(img)
        assert_same_state(full_state(a), full_state(b))
        # both continue with the same offsets and end in the same state
        assert np.array_equal(a.replay(cont, mode), b.replay(cont, mode))
        assert_same_state(full_state(a), full_state(b))
        assert a.error_flags() == 0 and b.error_flags() == 0


def test_image_in_device_memory():
    with Heap(64, 12) as a, Heap(64, 12) as b:
        a.replay(make_stream(73, 700, 12), MODE_WARP)
        buf = torch.empty(a.image_bytes(), dtype=torch.uint8, device="cuda")
        a.image_save(buf.data_ptr(), buf.numel())
        b.image_load(buf.data_ptr(), buf.numel())
        assert_same_state(full_state(a), full_state(b))
        host = a.image_save()
        assert np.array_equal(host, buf.cpu().numpy())


def test_image_of_other_geometry_is_refused():
    # 1023 pages: 31 class-table shards per class by default (pages/32),
    # 8 under a cap of 8, one on the compat heap
    with Heap(1024, 12) as a:
        assert a.cls_shards[0] == 31
        img = a.image_save()
    for other in (dict(sblocks=1025, log2=12), dict(sblocks=1024, log2=14),
                  dict(sblocks=1024, log2=12, compat=True), dict(sblocks=1024, log2=12, shards=8)):
        sb, lg = other.pop("sblocks"), other.pop("log2")
        with Heap(sb, lg, **other) as b:
            before = full_state(b)
            with pytest.raises(KmaError) as e:
                b.image_load(img)
            assert e.value.code == EINVAL
            assert_same_state(before, full_state(b))


def test_damaged_image_is_refused_and_heap_unchanged():
    with Heap(64, 12) as a, Heap(64, 12) as b:
        a.replay(make_stream(74, 600, 12), MODE_PLAIN)
        img = a.image_save()
        h = ins.image_header(img)
        b.replay(make_stream(75, 300, 12), MODE_PLAIN)
        before = full_state(b)

        def refused(buf):
            with pytest.raises(KmaError) as e:
                b.image_load(buf)
            assert e.value.code == EINVAL
            assert_same_state(before, full_state(b))

        refused(img[:-1])                                  # truncated
        bad = img.copy(); bad[0] ^= 1; refused(bad)        # magic
        cls = lambda buf: buf[h["off_cls"]:h["off_cls"] + 4 * h["cls_lines"]].view("<u4")
        st = lambda buf: buf[h["off_state"]:h["off_state"] + 4 * h["sblocks"]].view("<u4")
        bad = img.copy(); cls(bad)[1] = h["sblocks"] + 2; refused(bad)   # class word past the heap
        bad = img.copy(); cls(bad)[1] = 1; refused(bad)                  # a refill in flight
        bad = img.copy(); st(bad)[3] = (15 << 28) | (1 << 14); refused(bad)  # unknown class
        s = int(np.flatnonzero(st(img))[0])
        bad = img.copy(); v = int(st(bad)[s]); slots = (v >> 14) & 0x3FFF
        st(bad)[s] = (v & ~0x3FFF) | (slots + 1); refused(bad)           # more free than slots
        fl = lambda buf: buf[h["off_flist"]:h["off_flist"] + 8 * h["flist_words"]].view("<u8")
        bad = img.copy(); fl(bad)[0] = (int(fl(bad)[0]) & ~0xFFFFFFFF) | h["sblocks"]
        refused(bad)                                                     # free-list entry past the heap
        # the untouched image still loads
        b.image_load(img)
        assert_same_state(full_state(a), full_state(b))


def _header_view(buf):
    return buf[:ins.IMAGE_HEADER.itemsize].view(ins.IMAGE_HEADER)


def test_inconsistent_ring_free_list_is_refused():
    """A ring free list that a quiescent heap cannot hold: a superblock
    queued twice, a slot sequence number off its ticket, an availability
    count that is not the queued count, a queued superblock with free
    slots.  Each would hand out blocks twice or leave waits to run out."""
    with Heap(64, 12) as a, Heap(64, 12) as b:
        a.replay(make_stream(76, 600, 12), MODE_WARP)
        img = a.image_save()
        h = ins.image_header(img)
        assert h["ring"] == 1 and h["free_tail"] - h["free_head"] >= 2
        cap, hd = h["flist_words"], h["free_head"]
        fl = lambda buf: buf[h["off_flist"]:h["off_flist"] + 8 * cap].view("<u8")
        st = lambda buf: buf[h["off_state"]:h["off_state"] + 4 * h["sblocks"]].view("<u4")
        before = full_state(b)

        def refused(buf):
            with pytest.raises(KmaError) as e:
                b.image_load(buf)
            assert e.value.code == EINVAL
            assert_same_state(before, full_state(b))

        s0 = int(fl(img)[hd % cap]) & 0xFFFFFFFF
        bad = img.copy(); w = int(fl(bad)[(hd + 1) % cap])
        fl(bad)[(hd + 1) % cap] = (w & ~0xFFFFFFFF) | s0; refused(bad)       # queued twice
        bad = img.copy(); fl(bad)[hd % cap] = int(fl(bad)[hd % cap]) + (1 << 32)
        refused(bad)                                                         # seq off its ticket
        bad = img.copy(); _header_view(bad)["ring_avail"] += 1; refused(bad)  # count off
        bad = img.copy(); st(bad)[s0] = (0 << 28) | (a.cls_slots[0] << 14) | 1
        refused(bad)                                                         # queued with free slots
        b.image_load(img)
        assert_same_state(full_state(a), full_state(b))


def test_inconsistent_queue_free_list_is_refused():
    """The compat heap's MS-queue free list: a chain with a cycle, and a
    chain that does not end at the tail, are refused."""
    with Heap(64, 12, compat=True) as a, Heap(64, 12, compat=True) as b:
        a.replay(make_stream(77, 600, 12), MODE_PLAIN)
        img = a.image_save()
        h = ins.image_header(img)
        nw = h["flist_words"]
        fl = lambda buf: buf[h["off_flist"]:h["off_flist"] + 8 * nw].view("<u8")
        hi, ti = h["free_head"] & 0xFFFFFFFF, h["free_tail"] & 0xFFFFFFFF
        assert hi != ti
        before = full_state(b)

        def refused(buf):
            with pytest.raises(KmaError) as e:
                b.image_load(buf)
            assert e.value.code == EINVAL
            assert_same_state(before, full_state(b))

        bad = img.copy(); fl(bad)[ti - 1] = (int(fl(bad)[ti - 1]) & ~0xFFFFFFFF) | hi
        refused(bad)                                                         # tail links to head
        bad = img.copy(); hv = _header_view(bad)
        hv["free_tail"] = (int(hv["free_tail"][0]) & ~0xFFFFFFFF) | hi
        refused(bad)                                                         # chain ends past the tail
        b.image_load(img)
        assert_same_state(full_state(a), full_state(b))
