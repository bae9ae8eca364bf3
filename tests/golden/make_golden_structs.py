"""Generate tests/golden/structs.npz from the reference's own structures.

Runs the UNMODIFIED reference clQueue.cl, clIndexedQueue.cl, clTree.cl,
clArrayList.cl (over kma.cl) and pma.cl, built by oracle/Makefile into
oracle/_ref/ (needs the reference tree, so it runs where that is mounted;
the fixture is committed and the GPU tests only read it):

    python tests/golden/make_golden_structs.py

Each case stores its op stream and the reference's results (and, for the
queues, the final head/tail/links; for the tree, the in-order keys; for
the graph build of test/tb_clTree.cl, every node's key, block offset and
links in queue order).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import structs  # noqa: E402
import struct_streams as ss  # noqa: E402

CLQ = [(1, 40, 600), (2, 8, 400), (3, 200, 1500)]          # (seed, items, ops)
IQ = [(11, 40, 600), (12, 8, 400), (13, 300, 1500)]
TREE = [(21, 400, 64), (22, 1500, 100000)]                   # (seed, ops, key space)
AL = [(31, 64, 4, 300, 6, 1), (32, 64, 24, 200, 40, 1), (33, 64, 4, 300, 200, 1),
      (34, 3, 16, 120, 60, 0)]  # (seed, sblocks, objsize, ops, max objs, gets)
AL_GROUP = [(41, 64, 4, [1, 2, 1, 2, 3, 0, 5, 1]), (42, 64, 8, list(range(33))),
            (43, 64, 4, [2] * 64), (44, 64, 12, [0, 0, 7, 0, 1])]  # (seed, sblocks, objsize, objs)
PMA = [(51, 4096, 300), (52, 100000, 2000)]                  # (seed, bytes, ops)
PMA_EDGE = [4096, 1000]
GRAPH = [(61, 64, 400, 60), (62, 256, 3000, 700)]          # (seed, sblocks, edges, vertices)


GRAPH_PMA_BYTES = 2097152


def graph_edges(seed: int, n_edges: int, n_vertices: int) -> np.ndarray:
    """Synthetic edges (the reference's edge file is not shipped): Zipf(1.1)
    vertex ranks mapped to distinct random u32 keys."""
    rng = np.random.default_rng(seed)
    keys = rng.choice(2**32 - 1, size=n_vertices, replace=False).astype(np.uint32)
    p = np.arange(1, n_vertices + 1, dtype=np.float64) ** -1.1
    p /= p.sum()
    return np.stack([keys[rng.choice(n_vertices, size=n_edges, p=p)],
                     keys[rng.choice(n_vertices, size=n_edges, p=p)]], axis=1).astype(np.uint32)


def cases() -> dict:
    out = {}
    for seed, n, m in CLQ:
        ops = ss.clqueue_stream(seed, n, m)
        res, fin = structs.clqueue_replay(n, ops)
        out[f"clq_{seed}_ops"], out[f"clq_{seed}_out"], out[f"clq_{seed}_fin"] = ops, res, fin
        out[f"clq_{seed}_n"] = np.array([n])
    for seed, n, m in IQ:
        ops = ss.iqueue_stream(seed, n, m)
        res, fin = structs.iqueue_replay(n, 4, ops)
        out[f"iq_{seed}_ops"], out[f"iq_{seed}_out"], out[f"iq_{seed}_fin"] = ops, res, fin
        out[f"iq_{seed}_n"] = np.array([n])
    for seed, m, ks in TREE:
        ops = ss.tree_stream(seed, m, ks, remove=False)
        res, keys = structs.tree_replay(ops)
        out[f"tree_{seed}_ops"], out[f"tree_{seed}_out"], out[f"tree_{seed}_keys"] = ops, res, keys
    for seed, sblocks, osz, m, mx, gets in AL:
        ops = ss.arraylist_stream(seed, m, mx, bool(gets))
        res = structs.arraylist_replay(sblocks, osz, ops)
        out[f"al_{seed}_ops"], out[f"al_{seed}_out"] = ops, res
        out[f"al_{seed}_cfg"] = np.array([sblocks, osz])
    for seed, sblocks, osz, objs in AL_GROUP:
        res = structs.arraylist_group(sblocks, osz, np.array(objs, np.uint32))
        out[f"alg_{seed}_objs"], out[f"alg_{seed}_out"] = np.array(objs, np.int64), res
        out[f"alg_{seed}_cfg"] = np.array([sblocks, osz])
    for seed, nb, m in PMA:
        ops = ss.pma_stream(seed, m, nb)
        out[f"pma_{seed}_ops"], out[f"pma_{seed}_out"] = ops, structs.pma_replay(nb, ops)
        out[f"pma_{seed}_bytes"] = np.array([nb])
    for nb in PMA_EDGE:
        ops = ss.pma_edge_stream(nb)
        out[f"pmaedge_{nb}_ops"], out[f"pmaedge_{nb}_out"] = ops, structs.pma_replay(nb, ops)
        out[f"pmaedge_{nb}_bytes"] = np.array([nb])
    for seed, sblocks, ne, nv in GRAPH:
        e = graph_edges(seed, ne, nv)
        k, o, sk, st = structs.graph_build(sblocks, e)
        out[f"graph_{seed}_edges"], out[f"graph_{seed}_keys"] = e.astype(np.int64), k
        out[f"graph_{seed}_offs"], out[f"graph_{seed}_sinks"], out[f"graph_{seed}_start"] = o, sk, st
        out[f"graph_{seed}_cfg"] = np.array([sblocks])
        # the same build over the reference's pma.cl (test/tb_clTree.c:478-480,
        # its 2 MiB PMA heap): the same nodes and links, bump-allocated
        k, o, sk, st = structs.graph_build_pma(GRAPH_PMA_BYTES, e)
        out[f"graphpma_{seed}_keys"], out[f"graphpma_{seed}_offs"] = k, o
        out[f"graphpma_{seed}_sinks"], out[f"graphpma_{seed}_start"] = sk, st
        out[f"graphpma_{seed}_cfg"] = np.array([GRAPH_PMA_BYTES])
    return out


def main() -> int:
    if not structs.available():
        print("reference structure libraries missing: run make -C oracle where the reference is mounted")
        return 1
    np.savez_compressed(os.path.join(HERE, "structs.npz"), **cases())
    print("wrote", os.path.join(HERE, "structs.npz"))
    return 0


if __name__ == "__main__":
    sys.exit(main())
