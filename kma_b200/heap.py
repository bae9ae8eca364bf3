"""Host-side mirror of the reference's heap API over libkma_b200.so.

``Heap`` is ``kma_create`` / ``kma_destroy`` (kma.c:79-127) with a CUDA
device and stream in place of the OpenCL device/queue; ``Workload`` drives
the C1/C2 stress programs; both only ever call the CUDA library.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_float, c_uint32, c_uint64, c_void_p

import numpy as np

from . import _lib
from ._lib import KmaConfig, KmaInfo, KmaWlStats, check, lib

SB_HDR = 12


def _stream_ptr(stream) -> int | None:
    """Accept None, an int handle, or an object with .cuda_stream (torch)."""
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream or None
    return int(getattr(stream, "cuda_stream")) or None


def size_by_sbid(sb_size_log2: int, sbid: int) -> int:
    """kma.cl:55-90 (_kma_size_by_sbid)."""
    return int(lib().kma_size_by_sbid(sb_size_log2, sbid))


def slots_by_size(sb_size_log2: int, size: int) -> int:
    """kma.cl:95-113 (_kma_slots_by_size)."""
    return int(lib().kma_slots_by_size(sb_size_log2, size))


def sbid_by_size(sb_size_log2: int, size: int) -> int:
    """kma.cl:119-148 (_kma_sbid_by_size)."""
    return int(lib().kma_sbid_by_size(sb_size_log2, size))


class Heap:
    """A device heap of ``sblocks`` superblocks of ``2**sb_size_log2`` bytes.

    Mirrors ``kma_create(dev, ctx, cq, prg, sblocks)`` (kma.c:79-127); raises
    ``KmaError`` where the reference prints and returns NULL.
    """

    def __init__(self, sblocks: int, sb_size_log2: int = 12, spin_limit: int = 0,
                 device: int = -1, stream=None, shards: int = 0, compat: bool = False):
        L = lib()
        cfg = KmaConfig(sblocks, sb_size_log2, spin_limit, device, shards,
                        _lib.KMA_CFG_COMPAT if compat else 0)
        h = c_void_p()
        check(L.kma_create_ex(byref(cfg), _stream_ptr(stream), byref(h)), "kma_create")
        self._h = h
        inf = KmaInfo()
        check(L.kma_get_info(h, byref(inf)), "kma_get_info")
        self.sblocks = int(inf.sblocks)
        self.pages = int(inf.pages)
        self.sb_size_log2 = int(inf.sb_size_log2)
        self.sb_size = 1 << self.sb_size_log2
        self.nclasses = int(inf.nclasses)
        self.max_request = int(inf.max_request)
        self.region_bytes = int(inf.region_bytes)
        self.device_bytes = int(inf.device_bytes)
        self.cls_size = [int(inf.cls_size[i]) for i in range(self.nclasses)]
        self.cls_slots = [int(inf.cls_slots[i]) for i in range(self.nclasses)]
        self.cls_shards = [int(inf.cls_shards[i]) for i in range(self.nclasses)]
        self.cls_lines = int(inf.cls_lines)
        self.compat = bool(inf.flags & _lib.KMA_CFG_COMPAT)

    # -- lifetime ---------------------------------------------------------
    @property
    def handle(self) -> c_void_p:
        if self._h is None:
            raise ValueError("heap destroyed")
        return self._h

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None:
            self._h = None  # never destroyed twice, even when destroy reports an error
            check(lib().kma_destroy(h), "kma_destroy")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    @property
    def device_ptr(self) -> int:
        """struct kma_heap* for kernels (kma_malloc / kma_free)."""
        return int(lib().kma_heap_device_ptr(self.handle))

    def reset(self, stream=None) -> None:
        """Stream-ordered re-initialisation (kma.cl:27-52 by bulk stores)."""
        check(lib().kma_reset(self.handle, _stream_ptr(stream)), "kma_reset")

    def error_flags(self, clear: bool = False, stream=None) -> int:
        f = c_uint32()
        check(lib().kma_error_flags(self.handle, _stream_ptr(stream), byref(f), int(clear)),
              "kma_error_flags")
        return int(f.value)

    def error_flags_async(self, dst_ptr: int, stream=None) -> None:
        """Stream-ordered copy of the flags to dst_ptr (pinned host or device)."""
        check(lib().kma_error_flags_async(self.handle, _stream_ptr(stream), dst_ptr), "kma_error_flags_async")

    def debug_set_class_word(self, cls: int, value: int, stream=None) -> None:
        """Fault injection for tests: write a raw class-table word."""
        check(lib().kma_debug_set_class_word(self.handle, cls, value, _stream_ptr(stream)),
              "kma_debug_set_class_word")

    def bitmaps(self, stream=None) -> np.ndarray:
        """Every superblock's allocation bitmap, (sblocks, words) u32, with
        words = ceil(slots of class 0 / 32) (the widest bitmap)."""
        import torch  # device scratch for the gather; torch is plumbing only
        words = (self.cls_slots[0] + 31) // 32
        buf = torch.empty(self.sblocks * words, dtype=torch.int32, device="cuda")
        check(lib().kma_gather_bitmaps(self.handle, _stream_ptr(stream), buf.data_ptr(), words),
              "kma_gather_bitmaps")
        torch.cuda.synchronize()
        return buf.cpu().numpy().view(np.uint32).reshape(self.sblocks, words)

    # -- images -----------------------------------------------------------
    def snapshot(self, region: bool = False, stream=None):
        """Copy the heap's metadata (and optionally its superblock region) to
        host numpy arrays; see ``kma_b200.inspect``."""
        from .inspect import HeapImage
        cls = np.zeros(self.cls_lines, np.uint32)
        state = np.zeros(self.sblocks, np.uint32)
        fl = np.zeros(self.sblocks, np.uint32)
        fl_len = np.zeros(1, np.uint64)
        reg = np.zeros(self.region_bytes if region else 0, np.uint8)
        check(lib().kma_snapshot(self.handle, _stream_ptr(stream), cls.ctypes.data,
                                 state.ctypes.data, fl.ctypes.data, fl_len.ctypes.data, 0,
                                 self.region_bytes if region else 0,
                                 reg.ctypes.data if region else None), "kma_snapshot")
        n = int(fl_len[0])
        freelist = None if n == 2**64 - 1 else fl[:n].astype(np.int64)
        return HeapImage(sb_size_log2=self.sb_size_log2, sblocks=self.sblocks, pages=self.pages,
                         nclasses=self.nclasses, cls_size=list(self.cls_size),
                         cls_slots=list(self.cls_slots), cls_raw=cls, cls_shards=list(self.cls_shards),
                         state=state, freelist=freelist, region=reg if region else None)

    def image_bytes(self) -> int:
        """Size of a heap image (kma_image_bytes)."""
        n = c_uint64()
        check(lib().kma_image_bytes(self.handle, byref(n)), "kma_image_bytes")
        return int(n.value)

    def image_save(self, dst_ptr: int | None = None, dst_bytes: int = 0, stream=None):
        """Save a position-independent image of the heap (kma_image_save):
        into host or device memory at dst_ptr, or, with no pointer, into a
        new host numpy uint8 array, which is returned.  The heap must be
        quiescent."""
        if dst_ptr is None:
            buf = np.zeros(self.image_bytes(), np.uint8)
            check(lib().kma_image_save(self.handle, _stream_ptr(stream), buf.ctypes.data, buf.nbytes),
                  "kma_image_save")
            return buf
        check(lib().kma_image_save(self.handle, _stream_ptr(stream), dst_ptr, dst_bytes), "kma_image_save")
        return None

    def image_load(self, src, src_bytes: int | None = None, stream=None) -> None:
        """Replace the heap's state with an image (kma_image_load): a numpy
        uint8 array, or a host/device address with its size.  KmaError
        (KMA_EINVAL) for an image of other geometry or one that does not
        validate; the heap is then unchanged."""
        if isinstance(src, np.ndarray):
            src = np.ascontiguousarray(src, np.uint8)
            check(lib().kma_image_load(self.handle, _stream_ptr(stream), src.ctypes.data, src.nbytes),
                  "kma_image_load")
            return
        check(lib().kma_image_load(self.handle, _stream_ptr(stream), int(src), int(src_bytes)),
              "kma_image_load")

    # -- serial replay ------------------------------------------------------
    def replay(self, ops: np.ndarray, mode: int = _lib.MODE_PLAIN) -> np.ndarray:
        """One-op-at-a-time replay on the device; ops is an (n, 2) int64
        array of (kind, arg) (kind 0 = malloc(arg), 1 = free(result of op
        arg)).  Returns offsets from the first superblock (-1 = NULL)."""
        ops = np.ascontiguousarray(ops, dtype=np.int64).reshape(-1, 2)
        out = np.zeros(len(ops), np.int64)
        check(lib().kma_replay_host(self.handle, ops.ctypes.data, len(ops), out.ctypes.data,
                                    int(mode)), "kma_replay")
        return out


class Workload:
    """Per-item stress program state (C1 or C2) bound to a heap."""

    def __init__(self, heap: Heap, program: int, items: int):
        self.heap = heap
        self.items = int(items)
        self.program = int(program)
        w = c_void_p()
        check(lib().kma_wl_create(heap.handle, self.program, self.items, byref(w)), "kma_wl_create")
        self._w = w

    def close(self) -> None:
        w = getattr(self, "_w", None)
        if w is not None:
            self._w = None
            check(lib().kma_wl_destroy(w), "kma_wl_destroy")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def begin(self, seed: int, stream=None) -> None:
        check(lib().kma_wl_begin(self._w, seed & (2**64 - 1), _stream_ptr(stream)), "kma_wl_begin")

    def begin_seeds(self, seeds_dev_ptr: int, stream=None) -> None:
        check(lib().kma_wl_begin_seeds(self._w, seeds_dev_ptr, _stream_ptr(stream)),
              "kma_wl_begin_seeds")

    def rounds(self, nrounds: int, mode: int, block_dim: int = 0, stream=None) -> None:
        check(lib().kma_wl_rounds(self._w, nrounds, mode, block_dim, _stream_ptr(stream)),
              "kma_wl_rounds")

    def drain(self, mode: int, block_dim: int = 0, stream=None) -> None:
        check(lib().kma_wl_drain(self._w, mode, block_dim, _stream_ptr(stream)), "kma_wl_drain")

    def serial(self, nrounds: int, round_major: bool, mode: int, stream=None) -> None:
        check(lib().kma_wl_serial(self._w, nrounds, int(round_major), mode, _stream_ptr(stream)),
              "kma_wl_serial")

    def stats(self, stream=None) -> dict:
        s = KmaWlStats()
        check(lib().kma_wl_stats_get(self._w, _stream_ptr(stream), byref(s)), "kma_wl_stats_get")
        return {"mallocs": s.mallocs, "frees": s.frees, "nulls": s.nulls,
                "bad_tags": s.bad_tags, "offset_hash": s.offset_hash,
                "fill_bytes": s.fill_bytes, "verify_bytes": s.verify_bytes}

    def run_host(self, seeds_host_ptr: int, nrounds: int, mode: int, hashes_host_ptr: int | None,
                 stream=None) -> dict:
        """kma_wl_run_host: reset, seeds in from host memory, all rounds and
        the drain in one launch, hashes and counters back to host."""
        s = KmaWlStats()
        check(lib().kma_wl_run_host(self._w, seeds_host_ptr, nrounds, mode, hashes_host_ptr,
                                    byref(s), _stream_ptr(stream)), "kma_wl_run_host")
        return {"mallocs": s.mallocs, "frees": s.frees, "nulls": s.nulls,
                "bad_tags": s.bad_tags, "offset_hash": s.offset_hash,
                "fill_bytes": s.fill_bytes, "verify_bytes": s.verify_bytes}

    def phase_cycles(self, stream=None) -> list:
        """Cycles per phase [malloc, fill, verify, free] of runs launched
        with mode | KMA_MODE_PROFILE, summed over warps."""
        out = np.zeros(4, np.uint64)
        check(lib().kma_wl_phase_cycles(self._w, _stream_ptr(stream), out.ctypes.data),
              "kma_wl_phase_cycles")
        return [int(x) for x in out]

    def tally(self, stream=None) -> dict:
        """kma_malloc_warp event counts of KMA_MODE_PROFILE runs."""
        out = np.zeros(8, np.uint64)
        check(lib().kma_wl_tally(self._w, _stream_ptr(stream), out.ctypes.data), "kma_wl_tally")
        names = ("turns", "tries", "poison_waits", "stale", "cas_lost", "refills", "claims",
                 "empty_claims")
        return {k: int(v) for k, v in zip(names, out)}

    @property
    def item_hashes_ptr(self) -> int:
        return int(lib().kma_wl_item_hashes(self._w))

    def live(self, stream=None):
        """(nlive[items], off[32, items], size[32, items]) of the live blocks."""
        n = self.items
        nlive = np.zeros(n, np.uint32)
        off = np.zeros((_lib.WL_CAP, n), np.uint64)
        size = np.zeros((_lib.WL_CAP, n), np.uint32)
        check(lib().kma_wl_live(self._w, _stream_ptr(stream), nlive.ctypes.data, off.ctypes.data,
                                size.ctypes.data), "kma_wl_live")
        return nlive, off, size


def bench_atomics(distinct: bool, threads: int, iters: int, stride_words: int = 32,
                  stream=None) -> float:
    """Milliseconds for threads*iters returning 32-bit atomicAdds."""
    ms = c_float()
    check(lib().kma_bench_atomics(int(distinct), threads, iters, stride_words, _stream_ptr(stream),
                                  byref(ms)), "kma_bench_atomics")
    return float(ms.value)
