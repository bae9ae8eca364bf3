"""Host-side mirror of the reference's structure and PMA APIs over
libkma_b200.so (include/kma_structs.h).

``Pma`` is ``pma_create`` (pma.c:80); ``ClQueue``, ``IQueue``, ``ClTree``
and ``ClArrayList`` are the handles of ``clQueue_create`` (clQueue.c:62),
``clIndexedQueue_create`` (clIndexedQueue.c:64), the tree root and
``clArrayList_create`` (clArrayList.c:58); the ``*_replay`` functions run
op streams one operation at a time on the device, and ``c3_*`` run the
concurrent microbenchmarks.  Everything calls the CUDA library.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_int64, c_uint32, c_uint64, c_void_p

import numpy as np

from ._lib import KmaC3QueueStats, KmaC3TreeStats, check, lib
from .heap import Heap, _stream_ptr

C3_CLQUEUE = 0
C3_IQUEUE = 1
C3_WARP = 0x100  # or into the kind: warp-combined enqueues and dequeues
C3_BLOCK = 0x200  # or into the kind: warp-combined enqueues, block-combined dequeues (one queue)


class _Handle:
    _destroy = ""

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None:
            self._h = None  # never destroyed twice, even when destroy reports an error
            check(getattr(lib(), self._destroy)(h), self._destroy)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


class Pma(_Handle):
    """Bump heap of `nbytes` data bytes (pma.c:31-53, pma.cl:24-48)."""
    _destroy = "kma_pma_destroy"

    def __init__(self, nbytes: int, device: int = -1, stream=None):
        h = c_void_p()
        check(lib().kma_pma_create(nbytes, device, _stream_ptr(stream), byref(h)), "kma_pma_create")
        self._h = h
        self.nbytes = nbytes

    @property
    def handle(self):
        return self._h

    @property
    def device_ptr(self) -> int:
        return int(lib().kma_pma_device_ptr(self._h))

    @property
    def base(self) -> int:
        return int(lib().kma_pma_base(self._h))

    def reset(self, stream=None) -> None:
        check(lib().kma_pma_reset(self._h, _stream_ptr(stream)), "kma_pma_reset")

    def head(self, stream=None) -> int:
        v = c_uint64()
        check(lib().kma_pma_head(self._h, _stream_ptr(stream), byref(v)), "kma_pma_head")
        return int(v.value)

    def replay(self, ops: np.ndarray) -> np.ndarray:
        ops = np.ascontiguousarray(ops, np.int64).reshape(-1, 2)
        out = np.zeros(len(ops), np.int64)
        check(lib().kma_pma_replay_host(self._h, ops.ctypes.data, len(ops), out.ctypes.data),
              "kma_pma_replay_host")
        return out


class ClQueue(_Handle):
    _destroy = "kma_clqueue_destroy"

    def __init__(self, device: int = -1, stream=None):
        h = c_void_p()
        check(lib().kma_clqueue_create(device, _stream_ptr(stream), byref(h)), "kma_clqueue_create")
        self._h = h

    @property
    def device_ptr(self) -> int:
        return int(lib().kma_clqueue_device_ptr(self._h))


class IQueue(_Handle):
    _destroy = "kma_iqueue_destroy"

    def __init__(self, base: int, stride_l2: int, capacity: int, first: int, shards: int = 1,
                 device: int = -1, stream=None):
        h = c_void_p()
        check(lib().kma_iqueue_create(base, stride_l2, capacity, first, shards, device,
                                      _stream_ptr(stream), byref(h)), "kma_iqueue_create")
        self._h = h

    @property
    def device_ptr(self) -> int:
        return int(lib().kma_iqueue_device_ptr(self._h))

    def error_flags(self, clear: bool = False, stream=None) -> int:
        f = c_uint32()
        check(lib().kma_iqueue_error_flags(self._h, _stream_ptr(stream), byref(f), int(clear)),
              "kma_iqueue_error_flags")
        return int(f.value)


class ClTree(_Handle):
    _destroy = "kma_cltree_destroy"

    def __init__(self, device: int = -1, stream=None):
        h = c_void_p()
        check(lib().kma_cltree_create(device, _stream_ptr(stream), byref(h)), "kma_cltree_create")
        self._h = h

    @property
    def device_ptr(self) -> int:
        return int(lib().kma_cltree_device_ptr(self._h))


class ClArrayList(_Handle):
    _destroy = "kma_clarraylist_destroy"

    def __init__(self, obj_size: int, heap: Heap | None = None, pma: Pma | None = None, stream=None):
        h = c_void_p()
        check(lib().kma_clarraylist_create(obj_size, heap.handle if heap else None,
                                           pma.handle if pma else None, _stream_ptr(stream), byref(h)),
              "kma_clarraylist_create")
        self._h = h

    @property
    def device_ptr(self) -> int:
        return int(lib().kma_clarraylist_device_ptr(self._h))


def _ops(ops) -> np.ndarray:
    return np.ascontiguousarray(ops, np.int64).reshape(-1, 2)


def clqueue_replay(n_items: int, ops) -> tuple[np.ndarray, np.ndarray]:
    ops = _ops(ops)
    out = np.zeros(len(ops), np.int64)
    fin = np.zeros(n_items + 2, np.int64)
    check(lib().kma_clqueue_replay_host(n_items, ops.ctypes.data, len(ops), out.ctypes.data,
                                        fin.ctypes.data), "kma_clqueue_replay_host")
    return out, fin


def iqueue_replay(n_items: int, stride_l2: int, ops) -> tuple[np.ndarray, np.ndarray]:
    ops = _ops(ops)
    out = np.zeros(len(ops), np.int64)
    fin = np.zeros(n_items + 2, np.int64)
    check(lib().kma_iqueue_replay_host(n_items, stride_l2, ops.ctypes.data, len(ops), out.ctypes.data,
                                       fin.ctypes.data), "kma_iqueue_replay_host")
    return out, fin


def cltree_replay(ops) -> tuple[np.ndarray, np.ndarray]:
    ops = _ops(ops)
    out = np.zeros(len(ops), np.int64)
    keys = np.zeros(len(ops), np.uint32)
    nk = c_int64()
    check(lib().kma_cltree_replay_host(ops.ctypes.data, len(ops), out.ctypes.data, keys.ctypes.data,
                                       byref(nk)), "kma_cltree_replay_host")
    return out, keys[: nk.value].astype(np.int64)


def clarraylist_replay(obj_size: int, ops, heap: Heap | None = None, pma: Pma | None = None) -> np.ndarray:
    ops = _ops(ops)
    out = np.zeros(len(ops), np.int64)
    check(lib().kma_clarraylist_replay_host(heap.handle if heap else None, pma.handle if pma else None,
                                            obj_size, ops.ctypes.data, len(ops), out.ctypes.data),
          "kma_clarraylist_replay_host")
    return out


def clarraylist_group(obj_size: int, objs, mode: int = 0, heap: Heap | None = None,
                      pma: Pma | None = None) -> np.ndarray:
    objs = np.ascontiguousarray(objs, np.uint32)
    out = np.zeros(len(objs), np.int64)
    check(lib().kma_clarraylist_group_host(heap.handle if heap else None, pma.handle if pma else None,
                                           obj_size, objs.ctypes.data, len(objs), mode, out.ctypes.data),
          "kma_clarraylist_group_host")
    return out


def c3_queue(kind: int, threads: int, per_thread: int, shards: int = 1, seed: int = 0xC3,
             device: int = -1) -> dict:
    st = KmaC3QueueStats()
    check(lib().kma_c3_queue_run(kind, threads, per_thread, shards, seed & (2**64 - 1), device, byref(st)),
          "kma_c3_queue_run")
    return {k: getattr(st, k) for k, _ in KmaC3QueueStats._fields_}


def c3_tree(kinds, keys, threads: int, device: int = -1) -> tuple[np.ndarray, dict]:
    kinds = np.ascontiguousarray(kinds, np.uint8)
    keys = np.ascontiguousarray(keys, np.uint32)
    res = np.zeros(len(keys), np.int8)
    st = KmaC3TreeStats()
    check(lib().kma_c3_tree_run(kinds.ctypes.data, keys.ctypes.data, len(keys), threads, device,
                                res.ctypes.data, byref(st)), "kma_c3_tree_run")
    return res, {k: getattr(st, k) for k, _ in KmaC3TreeStats._fields_}
