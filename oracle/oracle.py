"""ctypes access to the oracle libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs, as the checker -- never by kma_b200.

  Ref(log2)   the reference's own kma.cl/clIndexedQueue.cl built unmodified
              (oracle/_ref/libkmaref_<log2>.so, present where the reference
              sources were available at build time)
  Port(log2)  the C restatement oracle/kma_port.c (libkmaport.so), which also
              covers heaps beyond the reference's 65 535-superblock limit
Both expose the same calls: create / malloc / free / replay / decode /
run_workload, with offsets measured from the first superblock.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_int64, c_uint, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PORT_LIB = os.path.join(HERE, "libkmaport.so")


def build() -> None:
    """Build whatever the Makefile can (the port always; the reference units
    only where the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def ref_available(log2: int = 12) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libkmaref_{log2}.so"))


def _load(path: str) -> ctypes.CDLL:
    if not os.path.exists(path):
        build()
    return ctypes.CDLL(path)


class _HeapOracle:
    """Common wrapper; subclasses bind the symbol prefix."""

    def __init__(self, handle, L, sb_size_log2, sblocks, prefix):
        self.h, self.L, self.sb_size_log2, self.sblocks, self.p = handle, L, sb_size_log2, sblocks, prefix
        self.sb_size = 1 << sb_size_log2
        self.nclasses = sb_size_log2 - 1

    def _f(self, name):
        return getattr(self.L, self.p + name)

    def malloc(self, n: int) -> int:
        return int(self._f("malloc")(self.h, n))

    def free(self, off: int) -> None:
        self._f("free")(self.h, off)

    def replay(self, ops: np.ndarray) -> np.ndarray:
        ops = np.ascontiguousarray(ops, np.int64).reshape(-1, 2)
        out = np.zeros(len(ops), np.int64)
        self._f("replay")(self.h, ops.ctypes.data, len(ops), out.ctypes.data)
        return out

    def decode(self) -> dict:
        n = self.sblocks
        cls = np.zeros(16, np.int64)
        size = np.zeros(n, np.uint32)
        slots = np.zeros(n, np.uint32)
        free = np.zeros(n, np.uint32)
        fl = np.zeros(n + 2, np.int64)
        m = self._f("decode")(self.h, cls.ctypes.data, size.ctypes.data, slots.ctypes.data,
                              free.ctypes.data, fl.ctypes.data, n + 2)
        return {"cls": cls[: self.nclasses], "sb_size": size, "sb_slots": slots,
                "sb_free": free, "freelist": fl[:m] if m >= 0 else None}

    def region(self) -> np.ndarray:
        """The superblock region (sblocks * SB bytes), headers masked."""
        base = self._base()
        buf = (ctypes.c_uint8 * (self.sblocks << self.sb_size_log2)).from_address(base)
        r = np.frombuffer(buf, np.uint8).copy().reshape(self.sblocks, self.sb_size)
        r[:, :12] = 0
        return r.reshape(-1)

    def run_workload(self, which: int, items: int, rounds: int, seed: int, mode: int,
                     threads: int = 1) -> dict:
        st = (c_uint64 * 5)()
        sec = c_double()
        rc = self._f("run_workload")(self.h, which, items, rounds, seed & (2**64 - 1), mode,
                                     threads, st, ctypes.byref(sec))
        if rc != 0:
            raise RuntimeError("oracle workload failed")
        return {"mallocs": st[0], "frees": st[1], "nulls": st[2], "bad_tags": st[3],
                "offset_hash": st[4], "seconds": sec.value}

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *e):
        self.close()


def _sig(L, prefix):
    f = lambda n: getattr(L, prefix + n)  # noqa: E731
    f("malloc").restype = c_int64
    f("malloc").argtypes = [c_void_p, c_uint64]
    f("free").restype = None
    f("free").argtypes = [c_void_p, c_int64]
    f("replay").restype = None
    f("replay").argtypes = [c_void_p, c_void_p, c_int64, c_void_p]
    f("decode").restype = c_int64
    f("decode").argtypes = [c_void_p] + [c_void_p] * 5 + [c_int64]
    f("run_workload").restype = c_int
    f("run_workload").argtypes = [c_void_p, c_int, c_uint64, c_uint32, c_uint64, c_int, c_uint,
                                  POINTER(c_uint64), POINTER(c_double)]
    f("destroy").restype = None
    f("destroy").argtypes = [c_void_p]


class Ref(_HeapOracle):
    """The unmodified reference (needs oracle/_ref/libkmaref_<log2>.so)."""

    def __init__(self, sblocks: int, sb_size_log2: int = 12):
        path = os.path.join(REF_DIR, f"libkmaref_{sb_size_log2}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        for n, r, a in [("oref_kma_create", c_void_p, [c_uint]),
                        ("oref_kma_sb_base", c_void_p, [c_void_p]),
                        ("oref_size_by_sbid", c_uint64, [c_int]),
                        ("oref_slots_by_size", c_int, [c_uint64]),
                        ("oref_sbid_by_size", c_int, [c_uint64]),
                        ("oref_buckets", c_uint, []), ("oref_header_bytes", c_uint, [])]:
            getattr(L, n).restype = r
            getattr(L, n).argtypes = a
        _sig(L, "oref_kma_")
        h = L.oref_kma_create(sblocks)
        if not h:
            raise ValueError("oref_kma_create failed")
        super().__init__(h, L, sb_size_log2, sblocks, "oref_kma_")

    def _base(self):
        return self.L.oref_kma_sb_base(self.h)


class Port(_HeapOracle):
    """The C restatement (oracle/kma_port.c)."""

    def __init__(self, sblocks: int, sb_size_log2: int = 12):
        L = _load(PORT_LIB)
        for n, r, a in [("oport_create", c_void_p, [c_uint32, c_uint32]),
                        ("oport_sb_base", c_void_p, [c_void_p]),
                        ("oport_size_by_sbid", c_uint32, [c_uint32, c_int]),
                        ("oport_slots_by_size", c_int, [c_uint32, c_uint64]),
                        ("oport_sbid_by_size", c_int, [c_uint32, c_uint64])]:
            getattr(L, n).restype = r
            getattr(L, n).argtypes = a
        _sig(L, "oport_")
        h = L.oport_create(sblocks, sb_size_log2)
        if not h:
            raise ValueError("oport_create failed")
        super().__init__(h, L, sb_size_log2, sblocks, "oport_")

    def _base(self):
        return self.L.oport_sb_base(self.h)


def ref_tables(sb_size_log2: int):
    """(size_by_sbid, slots_by_size(size), sbid_by_size for 0..SB) from the
    reference build."""
    L = ctypes.CDLL(os.path.join(REF_DIR, f"libkmaref_{sb_size_log2}.so"))
    L.oref_size_by_sbid.restype = c_uint64
    L.oref_size_by_sbid.argtypes = [c_int]
    L.oref_slots_by_size.argtypes = [c_uint64]
    L.oref_sbid_by_size.argtypes = [c_uint64]
    nb = sb_size_log2 - 1
    sizes = [int(L.oref_size_by_sbid(i)) for i in range(nb)]
    slots = [int(L.oref_slots_by_size(s)) for s in sizes]
    sb = 1 << sb_size_log2
    sbid = np.array([L.oref_sbid_by_size(n) for n in range(sb + 1)], np.int32)
    return sizes, slots, sbid


def port_tables(sb_size_log2: int):
    L = _load(PORT_LIB)
    L.oport_size_by_sbid.restype = c_uint32
    L.oport_size_by_sbid.argtypes = [c_uint32, c_int]
    L.oport_slots_by_size.argtypes = [c_uint32, c_uint64]
    L.oport_sbid_by_size.argtypes = [c_uint32, c_uint64]
    nb = sb_size_log2 - 1
    sizes = [int(L.oport_size_by_sbid(sb_size_log2, i)) for i in range(nb)]
    slots = [int(L.oport_slots_by_size(sb_size_log2, s)) for s in sizes]
    sb = 1 << sb_size_log2
    sbid = np.array([L.oport_sbid_by_size(sb_size_log2, n) for n in range(sb + 1)], np.int32)
    return sizes, slots, sbid
