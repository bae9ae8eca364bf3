"""The batched form (include/kma_batch.h): many uneven jobs in one
persistent, graph-captured launch on one heap, and the autotuner over
superblock size x block dim x per-warp cache depth.  No counterpart in the
reference (one OpenCL kernel per job, test/tb_kma.c); every allocation
goes through the device heap's warp-collaborative malloc/free."""
from __future__ import annotations

import ctypes
from ctypes import byref, c_uint32, c_void_p

import numpy as np

from ._lib import KmaBatchJob, KmaBatchStats, KmaBatchTuneEntry, check, lib
from .heap import Heap, _stream_ptr


def _jobs(threads, seeds):
    threads = [int(t) for t in threads]
    seeds = [int(s) & (2**64 - 1) for s in seeds]
    arr = (KmaBatchJob * len(threads))()
    for i, (t, s) in enumerate(zip(threads, seeds)):
        arr[i].threads, arr[i].seed = t, s
    return arr


def c4_jobs(seed: int = 0xC4, njobs: int = 64, lo: float = 1e3, hi: float = 1e6):
    """The batched configuration's jobs: thread counts log-uniform in
    [lo, hi], one seed per job (both from `seed`)."""
    rng = np.random.default_rng(seed)
    threads = np.exp(rng.uniform(np.log(lo), np.log(hi), njobs)).astype(np.int64)
    seeds = rng.integers(0, 2**63, njobs)
    return threads, seeds


def _stats(st: KmaBatchStats) -> dict:
    return {k: int(getattr(st, k)) for k, _ in KmaBatchStats._fields_}


class Batch:
    """The jobs on a Heap, or on a structs.Pma (the same kernel compiled for
    the bump heap); mode MODE_WARP (warp-collaborative calls, default) or
    MODE_PLAIN (every thread calls malloc / free itself)."""

    def __init__(self, heap, threads, seeds, rounds: int, mode: int | None = None):
        self.heap = heap
        jobs = _jobs(threads, seeds)
        b = c_void_p()
        if isinstance(heap, Heap):
            check(lib().kma_batch_create(heap.handle, jobs, len(jobs), rounds, byref(b)), "kma_batch_create")
        else:
            check(lib().kma_batch_create_pma(heap.handle, jobs, len(jobs), rounds, byref(b)),
                  "kma_batch_create_pma")
        self._b = b
        self.items = int(lib().kma_batch_items(b))
        self.rounds = rounds
        if mode is not None:
            check(lib().kma_batch_set_mode(b, mode), "kma_batch_set_mode")

    def close(self) -> None:
        b = getattr(self, "_b", None)
        if b is not None:
            self._b = None
            check(lib().kma_batch_destroy(b), "kma_batch_destroy")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def run(self, block_dim: int = 256, cache_depth: int = 0, stream=None) -> None:
        check(lib().kma_batch_run(self._b, block_dim, cache_depth, _stream_ptr(stream)), "kma_batch_run")

    def capture(self, block_dim: int, cache_depth: int, stream) -> None:
        check(lib().kma_batch_capture(self._b, block_dim, cache_depth, _stream_ptr(stream)), "kma_batch_capture")

    def launch(self, stream=None) -> None:
        check(lib().kma_batch_launch(self._b, _stream_ptr(stream)), "kma_batch_launch")

    def stats(self, stream=None) -> dict:
        st = KmaBatchStats()
        check(lib().kma_batch_stats_get(self._b, _stream_ptr(stream), byref(st)), "kma_batch_stats_get")
        return _stats(st)


def autotune(threads, seeds, rounds: int, heap_bytes: int, sb_log2s=(12, 14, 16), block_dims=(128, 256, 512),
             depths=(0, 2, 4), warmup: int = 1, reps: int = 2, device: int = -1, shards: int = 0):
    """Run the native autotuner; returns (entries, best index)."""
    jobs = _jobs(threads, seeds)
    sb = np.ascontiguousarray(sb_log2s, np.uint32)
    bd = np.ascontiguousarray(block_dims, np.uint32)
    dp = np.ascontiguousarray(depths, np.uint32)
    n = len(sb) * len(bd) * len(dp)
    ent = (KmaBatchTuneEntry * n)()
    best = c_uint32()
    check(lib().kma_batch_autotune(jobs, len(jobs), rounds, heap_bytes, shards, sb.ctypes.data, len(sb),
                                   bd.ctypes.data, len(bd), dp.ctypes.data, len(dp), warmup, reps, device,
                                   ent, byref(best)), "kma_batch_autotune")
    out = []
    for e in ent:
        out.append({"sb_size": 1 << e.sb_size_log2, "block_dim": e.block_dim, "cache_depth": e.cache_depth,
                    "serves_all": bool(e.serves_all), "ms": round(e.ms, 3), "mops": round(e.mops, 1),
                    **_stats(e.stats)})
    b = int(best.value)
    return out, (b if b != 0xFFFFFFFF else None)
