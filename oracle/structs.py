"""ctypes access to the reference's lock-free structures and PMA heap.

TEST INFRASTRUCTURE ONLY: used by tests/golden/make_golden_structs.py (and
the CPU tests that pin its fixtures) as the checker, never by kma_b200.

The libraries are the reference's clQueue.cl, clIndexedQueue.cl, clTree.cl,
clArrayList.cl (over kma.cl) and pma.cl compiled unmodified by
oracle/Makefile into oracle/_ref/libclref.so and libpmaref.so
(ref_struct_unit.c, ref_pma_unit.c).  Every replay runs one operation at a
time on the calling thread, with items and nodes in host memory, and
reports results in the same index/offset encoding as the device replays
of include/kma_structs.h.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_int, c_int64, c_uint, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CL_LIB = os.path.join(HERE, "_ref", "libclref.so")
PMA_LIB = os.path.join(HERE, "_ref", "libpmaref.so")

POISON = 1


def available() -> bool:
    return os.path.exists(CL_LIB) and os.path.exists(PMA_LIB)


_cl = None
_pma = None


def _cl_lib() -> ctypes.CDLL:
    global _cl
    if _cl is None:
        L = ctypes.CDLL(CL_LIB)
        for name, res, args in [
            ("oref_q_create", c_void_p, []), ("oref_q_destroy", None, [c_void_p]),
            ("oref_q_enqueue", c_int, [c_void_p, c_void_p]), ("oref_q_dequeue", c_void_p, [c_void_p]),
            ("oref_q_head", c_uint64, [c_void_p]), ("oref_q_tail", c_uint64, [c_void_p]),
            ("oref_iq_create", c_void_p, [c_void_p, c_uint32, c_void_p]),
            ("oref_iq_destroy", None, [c_void_p]),
            ("oref_iq_enqueue", c_int, [c_void_p, c_void_p]), ("oref_iq_dequeue", c_void_p, [c_void_p]),
            ("oref_iq_head", c_uint32, [c_void_p]), ("oref_iq_tail", c_uint32, [c_void_p]),
            ("oref_tree_create", c_void_p, []), ("oref_tree_destroy", None, [c_void_p]),
            ("oref_tree_node_size", c_uint32, []),
            ("oref_tree_add", c_uint, [c_void_p, c_void_p]), ("oref_tree_get", c_void_p, [c_void_p, c_uint]),
            ("oref_heap_create", c_void_p, [c_uint]), ("oref_heap_destroy", None, [c_void_p]),
            ("oref_heap_sb_base", c_void_p, [c_void_p]),
            ("oref_al_create", c_void_p, [c_uint32, c_void_p]), ("oref_al_destroy", None, [c_void_p]),
            ("oref_al_grow", c_uint64, [c_void_p, c_uint32]), ("oref_al_get", c_uint64, [c_void_p, c_uint64]),
            ("oref_al_clear", None, [c_void_p]),
            ("oref_al_grow_local_group", c_int, [c_void_p, c_uint32, c_void_p, c_void_p]),
            ("oref_graph_node_size", c_uint32, []), ("oref_graph_link_size", c_uint32, []),
            ("oref_graph_build_serial", None, [c_void_p, c_void_p, c_void_p, c_uint32]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _cl = L
    return _cl


def _pma_lib() -> ctypes.CDLL:
    global _pma
    if _pma is None:
        L = ctypes.CDLL(PMA_LIB)
        for name, res, args in [
            ("oref_pma_create", c_void_p, [c_uint64]), ("oref_pma_destroy", None, [c_void_p]),
            ("oref_pma_replay", None, [c_void_p, c_void_p, c_int64, c_void_p]),
            ("oref_pma_head", c_uint32, [c_void_p]), ("oref_pma_header_bytes", c_uint32, []),
            ("oref_pma_data_base", c_uint64, [c_void_p]),
            ("oref_pma_graph_build_serial", None, [c_void_p, c_void_p, c_void_p, c_uint32]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _pma = L
    return _pma


def _index(ptr: int, base: int, stride: int) -> int:
    if ptr == 0:
        return -1
    if ptr == POISON:
        return -2
    return (ptr - base) // stride


def clqueue_replay(n_items: int, ops: np.ndarray):
    """clQueue.cl enqueue/dequeue, one at a time, over n_items 16-byte
    items: (out, final) as kma_clqueue_replay_host."""
    L = _cl_lib()
    items = np.zeros(n_items * 2, np.uint64)  # 16 bytes per item, link first
    base = items.ctypes.data
    q = L.oref_q_create()
    out = np.zeros(len(ops), np.int64)
    try:
        for i, (kind, arg) in enumerate(np.asarray(ops, np.int64).reshape(-1, 2)):
            if kind == 0:
                out[i] = L.oref_q_enqueue(q, base + int(arg) * 16)
            else:
                out[i] = _index(L.oref_q_dequeue(q) or 0, base, 16)
        fin = [_index(L.oref_q_head(q), base, 16), _index(L.oref_q_tail(q), base, 16)]
        fin += [_index(int(items[2 * k]), base, 16) for k in range(n_items)]
    finally:
        L.oref_q_destroy(q)
    return out, np.array(fin, np.int64)


def iqueue_replay(n_items: int, stride_l2: int, ops: np.ndarray):
    """clIndexedQueue.cl idxd_enqueue/idxd_dequeue, one at a time; item 0 is
    the initial dummy: (out, final) as kma_iqueue_replay_host."""
    L = _cl_lib()
    stride = 1 << stride_l2
    items = np.zeros(n_items * stride // 4, np.uint32)
    base = items.ctypes.data
    q = L.oref_iq_create(base, stride_l2, base)
    out = np.zeros(len(ops), np.int64)

    def idx(w: int) -> int:  # {tag:10 | index:16 | poison:1} -> item
        return ((w & 0x1FFFE) >> 1) - 1

    try:
        for i, (kind, arg) in enumerate(np.asarray(ops, np.int64).reshape(-1, 2)):
            if kind == 0:
                out[i] = L.oref_iq_enqueue(q, base + int(arg) * stride)
            else:
                p = L.oref_iq_dequeue(q) or 0
                out[i] = -1 if p == 0 else (p - base) // stride
        fin = [idx(L.oref_iq_head(q)), idx(L.oref_iq_tail(q))]
        fin += [idx(int(items[k * stride // 4])) for k in range(n_items)]
    finally:
        L.oref_iq_destroy(q)
    return out, np.array(fin, np.int64)


def tree_replay(ops: np.ndarray):
    """clTree.cl add (kind 0) / get (kind 1), one at a time, node i for op
    i: (out, in-order keys)."""
    L = _cl_lib()
    ops = np.asarray(ops, np.int64).reshape(-1, 2)
    ns = L.oref_tree_node_size()
    assert ns == 24
    pool = np.zeros(len(ops) * 3, np.uint64)  # key(+pad), left, right
    base = pool.ctypes.data
    t = L.oref_tree_create()
    out = np.zeros(len(ops), np.int64)
    try:
        for i, (kind, key) in enumerate(ops):
            if kind == 0:
                pool[3 * i] = int(key)
                out[i] = L.oref_tree_add(t, base + 24 * i)
            elif kind == 1:
                p = L.oref_tree_get(t, int(key)) or 0
                out[i] = -1 if p == 0 else (p - base) // 24
            else:
                raise ValueError("the reference tree has no remove")
        root = ctypes.c_uint64.from_address(t).value
    finally:
        L.oref_tree_destroy(t)
    keys, stack, cur = [], [], root
    while cur or stack:
        while cur:
            stack.append(cur)
            cur = int(pool[(cur - base) // 8 + 1])
        cur = stack.pop()
        k = (cur - base) // 8
        keys.append(int(pool[k]) & 0xFFFFFFFF)
        cur = int(pool[k + 2])
    return out, np.array(keys, np.int64)


def arraylist_replay(sblocks: int, obj_size: int, ops: np.ndarray):
    """clArrayList.cl grow (0) / get (1) / clear (2) over a fresh reference
    KMA heap of `sblocks` 4 KiB superblocks; offsets from its first
    superblock."""
    L = _cl_lib()
    h = L.oref_heap_create(sblocks)
    base = L.oref_heap_sb_base(h)
    lst = L.oref_al_create(obj_size, h)
    out = np.zeros(len(ops), np.int64)
    try:
        for i, (kind, arg) in enumerate(np.asarray(ops, np.int64).reshape(-1, 2)):
            if kind == 0:
                p = L.oref_al_grow(lst, int(arg))
                out[i] = -1 if p == 0 else p - base
            elif kind == 1:
                out[i] = L.oref_al_get(lst, int(arg)) - base
            else:
                L.oref_al_clear(lst)
                out[i] = 0
    finally:
        L.oref_al_destroy(lst)
        L.oref_heap_destroy(h)
    return out


def arraylist_group(sblocks: int, obj_size: int, objs: np.ndarray, pre_grow: int = 0):
    """One work-group of len(objs) work-items (<= 64) calling
    clArrayList_grow_local together on a fresh list (after pre_grow single
    grows of one object, to move the heap off its start)."""
    L = _cl_lib()
    objs = np.ascontiguousarray(objs, np.uint32)
    h = L.oref_heap_create(sblocks)
    base = L.oref_heap_sb_base(h)
    lst = L.oref_al_create(obj_size, h)
    res = np.zeros(len(objs), np.uint64)
    try:
        for _ in range(pre_grow):
            L.oref_al_grow(lst, 1)
        rc = L.oref_al_grow_local_group(lst, len(objs), objs.ctypes.data, res.ctypes.data)
        if rc != 0:
            raise ValueError("group too large for the reference (<= 64)")
    finally:
        L.oref_al_destroy(lst)
        L.oref_heap_destroy(h)
    return np.array([-1 if r == 0 else int(r) - base for r in res], np.int64)


def pma_replay(nbytes: int, ops: np.ndarray):
    """pma.cl malloc (0) / free (1) over a fresh heap of nbytes data bytes;
    offsets from its data base."""
    L = _pma_lib()
    ops = np.ascontiguousarray(np.asarray(ops, np.int64).reshape(-1, 2))
    p = L.oref_pma_create(nbytes)
    out = np.zeros(len(ops), np.int64)
    try:
        L.oref_pma_replay(p, ops.ctypes.data, len(ops), out.ctypes.data)
    finally:
        L.oref_pma_destroy(p)
    return out


def _graph_walk(root_addr: int, base: int):
    """In-order walk of a reference graph: (keys, node offsets from `base`,
    link sinks, link start), nodes in key order, each node's links in queue
    order.  clGraph_node = {clTree_node (key, left, right), clQueue links};
    clGraph_link = {next, sink}."""
    u64 = lambda a: ctypes.c_uint64.from_address(a).value  # noqa: E731
    u32 = lambda a: ctypes.c_uint32.from_address(a).value  # noqa: E731
    keys, offs, sinks, start = [], [], [], []
    stack, cur = [], u64(root_addr)
    while cur or stack:
        while cur:
            stack.append(cur)
            cur = u64(cur + 8)
        cur = stack.pop()
        keys.append(u32(cur))
        offs.append(cur - base)
        start.append(len(sinks))
        link = u64(cur + 24)  # links.head
        while link:
            sinks.append(u32(u64(link + 8)))
            link = u64(link)
        cur = u64(cur + 16)
    start.append(len(sinks))
    return (np.array(keys, np.int64), np.array(offs, np.int64), np.array(sinks, np.int64),
            np.array(start, np.int64))


def graph_build(sblocks: int, edges: np.ndarray):
    """tb_clTree.cl clTree_test run by one work-item over a fresh reference
    KMA heap of `sblocks` 4 KiB superblocks: (keys, node offsets from the
    first superblock, link sinks, link start) with nodes in key order and
    each node's links in queue order."""
    L = _cl_lib()
    assert L.oref_graph_node_size() == 40 and L.oref_graph_link_size() == 16
    edges = np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)
    h = L.oref_heap_create(sblocks)
    base = L.oref_heap_sb_base(h)
    t = L.oref_tree_create()
    try:
        L.oref_graph_build_serial(h, t, edges.ctypes.data, len(edges))
        return _graph_walk(t, base)
    finally:
        L.oref_tree_destroy(t)
        L.oref_heap_destroy(h)


def graph_build_pma(nbytes: int, edges: np.ndarray):
    """The same build over the reference's pma.cl (as test/tb_clTree.c:478-480
    runs it) on a fresh PMA heap of `nbytes` data bytes; node offsets are
    from the heap's data base."""
    L, P = _cl_lib(), _pma_lib()
    edges = np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)
    p = P.oref_pma_create(nbytes)
    base = P.oref_pma_data_base(p)
    t = L.oref_tree_create()
    try:
        P.oref_pma_graph_build_serial(p, t, edges.ctypes.data, len(edges))
        return _graph_walk(t, base)
    finally:
        L.oref_tree_destroy(t)
        P.oref_pma_destroy(p)
