"""The graph-build workload (include/kma_graph.h): the reference's tree
driver (test/tb_clTree.cl:12-85) -- nodes in a clTree, a clQueue of links
per node, every node and link a heap block."""
from __future__ import annotations

from ctypes import byref

import numpy as np

from ._lib import KmaGraphStats, check, lib
from .heap import Heap


def edge_mix(source: int, sink: int) -> int:
    return int(lib().kma_graph_edge_mix(source, sink))


def synth_edges(seed: int, n_edges: int, n_vertices: int, skew: float = 1.1) -> np.ndarray:
    """Synthetic (source, sink) u32 pairs (the reference's edge file is not
    shipped): vertex ranks Zipf(skew) over n_vertices, mapped to distinct
    random u32 keys."""
    rng = np.random.default_rng(seed)
    keys = rng.choice(2**32 - 1, size=n_vertices, replace=False).astype(np.uint32)
    p = np.arange(1, n_vertices + 1, dtype=np.float64) ** -skew
    p /= p.sum()
    src = rng.choice(n_vertices, size=n_edges, p=p)
    dst = rng.choice(n_vertices, size=n_edges, p=p)
    return np.stack([keys[src], keys[dst]], axis=1).astype(np.uint32)


def build(heap, edges: np.ndarray, threads: int, free_after: bool = True, export: bool = False):
    """Run the build on a Heap, or on a structs.Pma (the same kernels
    instantiated for the bump heap, which frees nothing: free_after does
    not apply); returns (stats, export) where export is None or
    (keys, node_offsets, link_sinks, link_start) in key order."""
    edges = np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)
    n = len(edges)
    st = KmaGraphStats()
    if export:
        keys = np.zeros(2 * n, np.uint32)
        offs = np.zeros(2 * n, np.int64)
        sinks = np.zeros(n, np.uint32)
        start = np.zeros(2 * n + 1, np.uint64)
        ptrs = (keys.ctypes.data, offs.ctypes.data, sinks.ctypes.data, start.ctypes.data)
    else:
        ptrs = (None, None, None, None)
    if isinstance(heap, Heap):
        check(lib().kma_graph_build(heap.handle, edges.ctypes.data, n, threads, int(free_after), byref(st),
                                    *ptrs), "kma_graph_build")
    else:
        check(lib().kma_graph_build_pma(heap.handle, edges.ctypes.data, n, threads, byref(st), *ptrs),
              "kma_graph_build_pma")
    stats = {k: getattr(st, k) for k, _ in KmaGraphStats._fields_ if k != "pad"}
    if not export:
        return stats, None
    m = int(st.nodes)
    return stats, (keys[:m].astype(np.int64), offs[:m], sinks[: int(start[m])].astype(np.int64),
                   start[: m + 1].astype(np.int64))
