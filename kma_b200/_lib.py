"""ctypes binding of libkma_b200.so (the C ABI of include/kma.h).

Loading never falls back to anything: if the library is missing or stale
the import raises, and every compute call goes through the CUDA library.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_uint,
                    c_uint32, c_uint64, c_void_p)

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libkma_b200.so")

KMA_OK = 0
KMA_EINVAL = -1
KMA_ENOMEM = -2
KMA_ECUDA = -3
KMA_ETIMEDOUT = -4
KMA_ENODEV = -5
KMA_EFAULT = -6

KMA_FLAG_TIMEOUT = 1
KMA_FLAG_BADFREE = 2

MODE_PLAIN = 0
MODE_WARP = 1

WL_C1 = 1
WL_C2 = 2
WL_CAP = 32


class KmaError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {strerror(code)} ({code})")


KMA_CFG_COMPAT = 1


class KmaConfig(Structure):
    _fields_ = [("sblocks", c_uint32), ("sb_size_log2", c_uint32),
                ("spin_limit", c_uint32), ("device", c_int32), ("shards", c_uint32),
                ("flags", c_uint32)]


class KmaInfo(Structure):
    _fields_ = [("region_bytes", c_uint64), ("device_bytes", c_uint64),
                ("sblocks", c_uint32), ("pages", c_uint32), ("sb_size_log2", c_uint32),
                ("nclasses", c_uint32), ("max_request", c_uint32),
                ("cls_size", c_uint32 * 16), ("cls_slots", c_uint32 * 16),
                ("cls_shards", c_uint32 * 16), ("cls_lines", c_uint32), ("flags", c_uint32)]


class KmaWlStats(Structure):
    _fields_ = [("mallocs", c_uint64), ("frees", c_uint64), ("nulls", c_uint64),
                ("bad_tags", c_uint64), ("offset_hash", c_uint64), ("fill_bytes", c_uint64),
                ("verify_bytes", c_uint64)]


class KmaC3QueueStats(Structure):
    _fields_ = [("enqueued", c_uint64), ("dequeued", c_uint64), ("empty", c_uint64),
                ("remaining", c_uint64), ("out_count", c_uint64), ("out_xor", c_uint64),
                ("out_sum", c_uint64), ("in_xor", c_uint64), ("in_sum", c_uint64),
                ("err", c_uint32), ("walk_ok", c_uint32), ("enqueue_ms", c_float),
                ("dequeue_ms", c_float), ("log_chains", c_uint32), ("pad", c_uint32)]


class KmaC3TreeStats(Structure):
    _fields_ = [("live_keys", c_uint64), ("keys_xor", c_uint64), ("keys_sum", c_uint64),
                ("sorted", c_uint32), ("err", c_uint32), ("ms", c_float)]


class KmaBatchJob(Structure):
    _fields_ = [("threads", c_uint32), ("pad", c_uint32), ("seed", c_uint64)]


class KmaBatchStats(Structure):
    _fields_ = [("mallocs", c_uint64), ("frees", c_uint64), ("nulls", c_uint64), ("bad_tags", c_uint64),
                ("fill_bytes", c_uint64), ("verify_bytes", c_uint64), ("cache_hits", c_uint64),
                ("cache_puts", c_uint64), ("retired", c_uint64), ("refused", c_uint64)]


class KmaBatchTuneEntry(Structure):
    _fields_ = [("sb_size_log2", c_uint32), ("block_dim", c_uint32), ("cache_depth", c_uint32),
                ("serves_all", c_uint32), ("ms", c_float), ("mops", c_float), ("stats", KmaBatchStats)]


class KmaServeCfg(Structure):
    _fields_ = [("slots", c_uint32), ("max_vertices", c_uint32), ("deg_max", c_uint32),
                ("block_dim", c_uint32), ("gamma", c_float), ("occupancy_limit", c_float)]


class KmaServeReq(Structure):
    _fields_ = [("n_vertices", c_uint32), ("pad", c_uint32), ("seed", c_uint64), ("arrival_s", c_double)]


class KmaServeResult(Structure):
    _fields_ = [("checksum", c_uint64), ("edges", c_uint64), ("mallocs", c_uint64), ("frees", c_uint64),
                ("nulls", c_uint64), ("admit_s", c_double), ("done_s", c_double),
                ("reserved_bytes", c_uint64), ("slot", c_uint32), ("status", c_uint32)]


class KmaServeSummary(Structure):
    _fields_ = [("wall_s", c_double), ("ops", c_uint64), ("max_running", c_uint32),
                ("max_sb_in_use", c_uint32), ("max_occupancy", c_double), ("max_reserved", c_double),
                ("admit_waits", c_uint32), ("pad", c_uint32)]


class KmaGraphStats(Structure):
    _fields_ = [("nodes", c_uint64), ("links", c_uint64), ("lost_adds", c_uint64), ("nulls", c_uint64),
                ("edge_xor", c_uint64), ("edge_sum", c_uint64), ("sorted", c_uint32), ("err", c_uint32),
                ("build_ms", c_float), ("pad", c_float)]


# (name, restype, argtypes) for every symbol include/*.h declares
SIGNATURES = [
    ("kma_size_by_sbid", c_uint32, [c_uint32, c_int]),
    ("kma_slots_by_size", c_int, [c_uint32, c_uint64]),
    ("kma_sbid_by_size", c_int, [c_uint32, c_uint64]),
    ("kma_create", c_void_p, [c_int, c_void_p, c_uint]),
    ("kma_create_ex", c_int, [POINTER(KmaConfig), c_void_p, POINTER(c_void_p)]),
    ("kma_destroy", c_int, [c_void_p]),
    ("kma_reset", c_int, [c_void_p, c_void_p]),
    ("kma_heap_device_ptr", c_void_p, [c_void_p]),
    ("kma_get_info", c_int, [c_void_p, POINTER(KmaInfo)]),
    ("kma_error_flags", c_int, [c_void_p, c_void_p, POINTER(c_uint32), c_int]),
    ("kma_error_flags_async", c_int, [c_void_p, c_void_p, c_void_p]),
    ("kma_strerror", c_char_p, [c_int]),
    ("kma_version", c_char_p, []),
    ("kma_snapshot", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                             c_uint64, c_uint64, c_void_p]),
    ("kma_gather_bitmaps", c_int, [c_void_p, c_void_p, c_void_p, c_uint32]),
    ("kma_image_bytes", c_int, [c_void_p, POINTER(c_uint64)]),
    ("kma_image_save", c_int, [c_void_p, c_void_p, c_void_p, c_uint64]),
    ("kma_image_load", c_int, [c_void_p, c_void_p, c_void_p, c_uint64]),
    ("kma_replay", c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int, c_void_p]),
    ("kma_replay_host", c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int]),
    ("kma_wl_create", c_int, [c_void_p, c_int, c_uint64, POINTER(c_void_p)]),
    ("kma_wl_destroy", c_int, [c_void_p]),
    ("kma_wl_begin", c_int, [c_void_p, c_uint64, c_void_p]),
    ("kma_wl_begin_seeds", c_int, [c_void_p, c_void_p, c_void_p]),
    ("kma_wl_rounds", c_int, [c_void_p, c_uint32, c_int, c_uint32, c_void_p]),
    ("kma_wl_drain", c_int, [c_void_p, c_int, c_uint32, c_void_p]),
    ("kma_wl_serial", c_int, [c_void_p, c_uint32, c_int, c_int, c_void_p]),
    ("kma_wl_run_host", c_int, [c_void_p, c_void_p, c_uint32, c_int, c_void_p,
                                POINTER(KmaWlStats), c_void_p]),
    ("kma_wl_run_noalloc", c_int, [c_void_p, c_int, c_uint64, c_void_p, c_uint32, c_int, c_int,
                                   c_void_p, c_void_p, c_void_p]),
    ("kma_wl_stats_get", c_int, [c_void_p, c_void_p, POINTER(KmaWlStats)]),
    ("kma_wl_item_hashes", c_void_p, [c_void_p]),
    ("kma_wl_phase_cycles", c_int, [c_void_p, c_void_p, c_void_p]),
    ("kma_wl_tally", c_int, [c_void_p, c_void_p, c_void_p]),
    ("kma_wl_live", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("kma_debug_set_class_word", c_int, [c_void_p, c_uint32, c_uint32, c_void_p]),
    ("kma_debug_queue_stuck_dequeue", c_int, [c_int, c_int, c_uint32, c_int, c_void_p, c_void_p]),
    ("kma_debug_queue_block_fifo", c_int, [c_int, c_uint32, c_uint32, c_int, c_void_p, c_void_p]),
    ("kma_bench_atomics", c_int, [c_int, c_uint64, c_uint32, c_uint32, c_void_p, POINTER(c_float)]),
    # include/kma_structs.h
    ("kma_pma_create", c_int, [c_uint64, c_int, c_void_p, POINTER(c_void_p)]),
    ("kma_pma_destroy", c_int, [c_void_p]),
    ("kma_pma_device_ptr", c_void_p, [c_void_p]),
    ("kma_pma_base", c_void_p, [c_void_p]),
    ("kma_pma_reset", c_int, [c_void_p, c_void_p]),
    ("kma_pma_head", c_int, [c_void_p, c_void_p, POINTER(c_uint64)]),
    ("kma_pma_replay_host", c_int, [c_void_p, c_void_p, c_int64, c_void_p]),
    ("kma_clqueue_create", c_int, [c_int, c_void_p, POINTER(c_void_p)]),
    ("kma_clqueue_destroy", c_int, [c_void_p]),
    ("kma_clqueue_device_ptr", c_void_p, [c_void_p]),
    ("kma_iqueue_create", c_int, [c_void_p, c_uint32, c_uint32, c_void_p, c_uint32, c_int, c_void_p,
                                  POINTER(c_void_p)]),
    ("kma_chain_log_create", c_int, [c_uint32, c_int, c_void_p, POINTER(c_void_p)]),
    ("kma_chain_log_destroy", c_int, [c_void_p]),
    ("kma_chain_log_device_ptr", c_void_p, [c_void_p]),
    ("kma_iqueue_set_chain_log", c_int, [c_void_p, c_void_p, c_void_p]),
    ("kma_iqueue_destroy", c_int, [c_void_p]),
    ("kma_iqueue_device_ptr", c_void_p, [c_void_p]),
    ("kma_iqueue_error_flags", c_int, [c_void_p, c_void_p, POINTER(c_uint32), c_int]),
    ("kma_cltree_create", c_int, [c_int, c_void_p, POINTER(c_void_p)]),
    ("kma_cltree_destroy", c_int, [c_void_p]),
    ("kma_cltree_device_ptr", c_void_p, [c_void_p]),
    ("kma_clarraylist_create", c_int, [c_uint32, c_void_p, c_void_p, c_void_p, POINTER(c_void_p)]),
    ("kma_clarraylist_destroy", c_int, [c_void_p]),
    ("kma_clarraylist_device_ptr", c_void_p, [c_void_p]),
    ("kma_clqueue_replay_host", c_int, [c_uint32, c_void_p, c_int64, c_void_p, c_void_p]),
    ("kma_iqueue_replay_host", c_int, [c_uint32, c_uint32, c_void_p, c_int64, c_void_p, c_void_p]),
    ("kma_cltree_replay_host", c_int, [c_void_p, c_int64, c_void_p, c_void_p, POINTER(c_int64)]),
    ("kma_clarraylist_replay_host", c_int, [c_void_p, c_void_p, c_uint32, c_void_p, c_int64, c_void_p]),
    ("kma_clarraylist_group_host", c_int, [c_void_p, c_void_p, c_uint32, c_void_p, c_uint32, c_int,
                                           c_void_p]),
    ("kma_c3_queue_run", c_int, [c_int, c_uint32, c_uint32, c_uint32, c_uint64, c_int,
                                 POINTER(KmaC3QueueStats)]),
    ("kma_c3_tree_run", c_int, [c_void_p, c_void_p, c_uint64, c_uint32, c_int, c_void_p,
                                POINTER(KmaC3TreeStats)]),
    # include/kma_batch.h
    ("kma_batch_create", c_int, [c_void_p, POINTER(KmaBatchJob), c_uint32, c_uint32, POINTER(c_void_p)]),
    ("kma_batch_create_pma", c_int, [c_void_p, POINTER(KmaBatchJob), c_uint32, c_uint32, POINTER(c_void_p)]),
    ("kma_batch_set_mode", c_int, [c_void_p, c_int]),
    ("kma_batch_destroy", c_int, [c_void_p]),
    ("kma_batch_items", c_uint64, [c_void_p]),
    ("kma_batch_run", c_int, [c_void_p, c_uint32, c_uint32, c_void_p]),
    ("kma_batch_capture", c_int, [c_void_p, c_uint32, c_uint32, c_void_p]),
    ("kma_batch_launch", c_int, [c_void_p, c_void_p]),
    ("kma_batch_stats_get", c_int, [c_void_p, c_void_p, POINTER(KmaBatchStats)]),
    ("kma_batch_autotune", c_int, [POINTER(KmaBatchJob), c_uint32, c_uint32, c_uint64, c_uint32, c_void_p, c_uint32,
                                   c_void_p, c_uint32, c_void_p, c_uint32, c_uint32, c_uint32, c_int,
                                   POINTER(KmaBatchTuneEntry), POINTER(c_uint32)]),
    # include/kma_graph.h
    ("kma_graph_edge_mix", c_uint64, [c_uint32, c_uint32]),
    ("kma_graph_build", c_int, [c_void_p, c_void_p, c_uint64, c_uint32, c_int, POINTER(KmaGraphStats),
                                c_void_p, c_void_p, c_void_p, c_void_p]),
    ("kma_graph_build_pma", c_int, [c_void_p, c_void_p, c_uint64, c_uint32, POINTER(KmaGraphStats),
                                    c_void_p, c_void_p, c_void_p, c_void_p]),
    # include/kma_serve.h
    ("kma_serve_create", c_int, [c_void_p, POINTER(KmaServeCfg), POINTER(c_void_p)]),
    ("kma_serve_set_mode", c_int, [c_void_p, c_int]),
    ("kma_serve_destroy", c_int, [c_void_p]),
    ("kma_serve_estimate", c_uint64, [c_void_p, c_uint32]),
    ("kma_serve_run", c_int, [c_void_p, POINTER(KmaServeReq), c_uint32, c_int, POINTER(KmaServeResult),
                              POINTER(KmaServeSummary)]),
]

_lib = None


def lib() -> ctypes.CDLL:
    """Load libkma_b200.so (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    from . import build as _build
    if _build.stale():
        _build.build()
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run python -m kma_b200.build")
    L = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def strerror(code: int) -> str:
    try:
        return lib().kma_strerror(code).decode()
    except Exception:  # noqa: BLE001 - only used to format an error
        return "error"


def check(code: int, what: str) -> None:
    if code != KMA_OK:
        raise KmaError(code, what)
