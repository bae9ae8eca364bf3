"""The C ABI: the library loads without a GPU and exports every function
include/kma.h declares; pure host entry points work without a device."""
import ctypes
import os
import re

import kma_b200
from kma_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(kma_\w+|pma_\w+|cl\w+)\s*\(", src, re.M):
            if not m.group(0).lstrip().startswith(("#", "typedef", "return")):
                names.add(m.group(1))
    return names


def test_header_parses():
    names = declared_functions()
    assert {"kma_create", "kma_destroy", "kma_reset", "kma_replay"} <= names


def test_every_declared_symbol_exported():
    L = kma_b200.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(L, n)]
    assert not missing, missing


def test_signature_table_covers_header():
    have = {n for n, _, _ in _lib.SIGNATURES}
    assert declared_functions() <= have


def test_host_only_calls_without_gpu():
    L = kma_b200.lib()
    assert L.kma_version().decode().startswith("kma_b200")
    assert L.kma_strerror(_lib.KMA_EINVAL).decode() == "invalid argument"
    # kma_create(sblocks == 0) is NULL, like kma.c:89-90, before any CUDA call
    assert not L.kma_create(0, None, 0)
    cfg = _lib.KmaConfig(0, 12, 0, -1)
    h = ctypes.c_void_p()
    assert L.kma_create_ex(ctypes.byref(cfg), None, ctypes.byref(h)) == _lib.KMA_EINVAL
    cfg = _lib.KmaConfig(16, 11, 0, -1)  # superblocks below 4 KiB are rejected
    assert L.kma_create_ex(ctypes.byref(cfg), None, ctypes.byref(h)) == _lib.KMA_EINVAL
    assert L.kma_destroy(None) == _lib.KMA_EINVAL
    # queue entry points that refuse their arguments before any CUDA call
    log = ctypes.c_void_p()
    assert L.kma_chain_log_create(1 << 25, -1, None, ctypes.byref(log)) == _lib.KMA_EINVAL  # above 2^24 records
    assert L.kma_chain_log_create(3, -1, None, ctypes.byref(log)) == _lib.KMA_EINVAL        # not a power of two
    taken, flags = ctypes.c_int64(), ctypes.c_uint32()
    assert L.kma_debug_queue_stuck_dequeue(1, 1, 64, -1, ctypes.byref(taken),
                                           ctypes.byref(flags)) == _lib.KMA_EINVAL  # no such indexed-queue case
    assert L.kma_debug_queue_stuck_dequeue(0, 0, 0, -1, ctypes.byref(taken),
                                           ctypes.byref(flags)) == _lib.KMA_EINVAL  # spin limit 0
