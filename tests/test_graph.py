"""The graph-build workload (include/kma_graph.h) after test/tb_clTree.cl:
one thread gives the reference's graph block for block (node offsets,
keys, every node's links in queue order); many threads give the same
multiset of edges, a search tree, and an empty heap after teardown."""
import os
from collections import defaultdict

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "structs.npz"))
SEEDS = sorted({k.split("_")[1] for k in GOLD.files if k.startswith("graph_")})


def edge_mix(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """mix(source, sink) as the library computes it (SplitMix64 finaliser of
    source << 32 | sink)."""
    with np.errstate(over="ignore"):
        z = (a.astype(np.uint64) << np.uint64(32) | b.astype(np.uint64)) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


@pytest.mark.parametrize("seed", SEEDS)
def test_graph_fixture_is_edges_in_order(seed):
    """The reference's serial build: each source's links are its edges' sinks
    in edge order, and the nodes are the distinct endpoints."""
    e = GOLD[f"graph_{seed}_edges"]
    keys, sinks, start = GOLD[f"graph_{seed}_keys"], GOLD[f"graph_{seed}_sinks"], GOLD[f"graph_{seed}_start"]
    d = defaultdict(list)
    for a, b in e:
        d[int(a)].append(int(b))
    np.testing.assert_array_equal(keys, np.unique(e))
    for i, k in enumerate(keys):
        assert sinks[start[i]:start[i + 1]].tolist() == d.get(int(k), [])


def test_edge_mix_matches_library():
    from kma_b200 import graph
    a = np.array([0, 1, 0xFFFFFFFF, 12345], np.uint32)
    b = np.array([0, 2, 7, 0xFFFFFFFF], np.uint32)
    assert [graph.edge_mix(int(x), int(y)) for x, y in zip(a, b)] == edge_mix(a, b).tolist()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", SEEDS)
def test_gpu_graph_serial_equals_reference(seed):
    from kma_b200 import Heap, graph
    sblocks = int(GOLD[f"graph_{seed}_cfg"][0])
    e = GOLD[f"graph_{seed}_edges"].astype(np.uint32)
    with Heap(sblocks, 12) as h:
        st, (keys, offs, sinks, start) = graph.build(h, e, threads=1, free_after=True, export=True)
        np.testing.assert_array_equal(keys, GOLD[f"graph_{seed}_keys"])
        np.testing.assert_array_equal(offs, GOLD[f"graph_{seed}_offs"])
        np.testing.assert_array_equal(sinks, GOLD[f"graph_{seed}_sinks"])
        np.testing.assert_array_equal(start, GOLD[f"graph_{seed}_start"])
        assert st["lost_adds"] == 0 and st["nulls"] == 0 and st["err"] == 0 and st["sorted"] == 1
        from kma_b200 import inspect as ins
        assert ins.check_canonical_empty(h.snapshot(), h.bitmaps()) == []


@pytest.mark.gpu
@pytest.mark.parametrize("threads", [4096, 65536])
def test_gpu_graph_concurrent_conserves_edges(threads):
    from kma_b200 import Heap, graph
    from kma_b200 import inspect as ins
    e = graph.synth_edges(77, 200_000, 20_000)
    with Heap(4096, 14) as h:
        st, _ = graph.build(h, e, threads=threads, free_after=True)
        m = edge_mix(e[:, 0], e[:, 1])
        assert st["err"] == 0 and st["nulls"] == 0 and st["sorted"] == 1
        assert st["nodes"] == len(np.unique(e))
        assert st["links"] == len(e)
        assert st["edge_xor"] == int(np.bitwise_xor.reduce(m))
        assert st["edge_sum"] == int(m.sum(dtype=np.uint64))
        assert st["lost_adds"] > 0  # threads raced to add the same key and the losers freed their node
        assert ins.check_canonical_empty(h.snapshot(), h.bitmaps()) == []
        assert h.error_flags() == 0
