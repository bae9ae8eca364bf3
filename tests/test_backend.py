"""Program composition (include/kma_backend.cuh): the same kernels compiled
for either heap, as the reference composes a program with kma.cl or pma.cl
(test/tb_clArrayList.c:170-173, 221-223; test/tb_clTree.c:441-446,
478-480).

The serial replay of both heaps is one kernel template (kma_k_heap_replay)
instantiated for kma_backend_kma (kma_replay_host) and kma_backend_pma
(kma_pma_replay_host); the graph build is one set of kernel templates
instantiated for both (kma_graph_build, kma_graph_build_pma).  Each
instantiation is checked against fixtures the reference's own kma.cl and
pma.cl produced."""
import glob
import os

import numpy as np
import pytest
from test_graph import edge_mix

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD_DIR = os.path.join(ROOT, "tests", "golden")
GOLD = np.load(os.path.join(GOLD_DIR, "structs.npz"))
REPLAYS = sorted(glob.glob(os.path.join(GOLD_DIR, "replay_12_*.npz")))
PMA_CASES = sorted(k[:-4] for k in GOLD.files if k.startswith(("pma_", "pmaedge_")) and k.endswith("_ops"))
GRAPH_SEEDS = sorted({k.split("_")[1] for k in GOLD.files if k.startswith("graphpma_")})


def test_pma_graph_fixtures_match_the_kma_ones():
    """Over either heap the reference builds the same graph (keys and the
    links of every node); only where the nodes live differs."""
    assert GRAPH_SEEDS
    for s in GRAPH_SEEDS:
        for f in ("keys", "sinks", "start"):
            np.testing.assert_array_equal(GOLD[f"graphpma_{s}_{f}"], GOLD[f"graph_{s}_{f}"])
        offs = GOLD[f"graphpma_{s}_offs"]
        assert len(np.unique(offs)) == len(offs) and (offs % 8 == 0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("path", REPLAYS, ids=[os.path.basename(p) for p in REPLAYS])
def test_gpu_replay_template_on_kma_equals_reference(path):
    from kma_b200 import MODE_PLAIN, Heap
    z = np.load(path)
    with Heap(int(z["sblocks"]), 12) as h:
        np.testing.assert_array_equal(h.replay(z["ops"], MODE_PLAIN), z["out"])
        assert h.error_flags() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("case", PMA_CASES)
def test_gpu_replay_template_on_pma_equals_reference(case):
    from kma_b200.structs import Pma
    with Pma(int(GOLD[f"{case}_bytes"][0])) as p:
        np.testing.assert_array_equal(p.replay(GOLD[f"{case}_ops"]), GOLD[f"{case}_out"])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", GRAPH_SEEDS)
def test_gpu_graph_build_on_pma_equals_reference(seed):
    """One work-item, as the reference's driver: the same tree, the same
    links in the same order, every node in the reference's PMA block."""
    from kma_b200 import graph
    from kma_b200.structs import Pma
    e = GOLD[f"graph_{seed}_edges"].astype(np.uint32)
    with Pma(int(GOLD[f"graphpma_{seed}_cfg"][0])) as p:
        st, (keys, offs, sinks, start) = graph.build(p, e, threads=1, export=True)
        for name, got in (("keys", keys), ("offs", offs), ("sinks", sinks), ("start", start)):
            np.testing.assert_array_equal(got, GOLD[f"graphpma_{seed}_{name}"], err_msg=name)
        assert st["lost_adds"] == 0 and st["nulls"] == 0 and st["err"] == 0 and st["sorted"] == 1


@pytest.mark.gpu
def test_gpu_graph_build_on_pma_conserves_edges():
    """Many threads on the PMA heap: every edge found once; a node that lost
    its add is not freed (PMA frees nothing), so the heap head counts it."""
    from kma_b200 import graph
    from kma_b200.structs import Pma
    e = graph.synth_edges(78, 200_000, 20_000)
    with Pma(64 << 20) as p:
        st, _ = graph.build(p, e, threads=65536)
        m = edge_mix(e[:, 0], e[:, 1])
        assert st["edge_xor"] == int(np.bitwise_xor.reduce(m))
        assert st["edge_sum"] == int(m.sum(dtype=np.uint64))
        assert st["err"] == 0 and st["nulls"] == 0 and st["sorted"] == 1
        assert st["nodes"] == len(np.unique(e)) and st["links"] == len(e)
        assert p.head() == 40 * (st["nodes"] + st["lost_adds"]) + 16 * len(e)
