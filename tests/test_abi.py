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
