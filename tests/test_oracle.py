"""The oracle itself: the C restatement (kma_port.c) must reproduce the
unmodified reference bit for bit under serial replay -- offsets, decoded
end state and the superblock bytes -- before it is trusted as a checker."""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle
from opstream import drain_stream, make_stream

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REPLAYS = sorted(glob.glob(os.path.join(GOLD, "replay_*.npz")))
WORKLOADS = json.load(open(os.path.join(GOLD, "workloads.json")))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def canon_equal(a, b):
    for k in ("cls", "sb_size", "sb_slots", "sb_free", "freelist"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


@pytest.mark.parametrize("path", REPLAYS, ids=os.path.basename)
def test_port_matches_golden_replay(path):
    g = np.load(path)
    log2 = int(os.path.basename(path).split("_")[1])
    with oracle.Port(int(g["sblocks"]), log2) as p:
        out = p.replay(g["ops"])
        assert np.array_equal(out, g["out"])
        canon_equal(p.decode(), g)
        assert digest(p.region()) == str(g["region_sha256"])


@pytest.mark.parametrize("log2,sblocks", [(12, 40), (12, 200), (14, 16), (16, 9), (12, 3), (12, 2)])
@pytest.mark.parametrize("seed", [11, 12, 13])
def test_port_matches_reference_live(log2, sblocks, seed):
    if not oracle.ref_available(log2):
        pytest.skip("reference build not present")
    ops = drain_stream(make_stream(seed * 7 + log2, 1500, log2))
    with oracle.Ref(sblocks, log2) as r, oracle.Port(sblocks, log2) as p:
        a, b = r.replay(ops), p.replay(ops)
        assert np.array_equal(a, b)
        canon_equal(r.decode(), p.decode())
        assert np.array_equal(r.region(), p.region())


@pytest.mark.parametrize("name", sorted(WORKLOADS))
def test_port_workloads_match_golden(name):
    w = WORKLOADS[name]
    with oracle.Port(w["sblocks"], w["sb_size_log2"]) as p:
        st = p.run_workload(w["program"], w["items"], w["rounds"], w["seed"], w["round_major"])
        d = p.decode()
    st.pop("seconds")
    assert st == w["stats"]
    assert len(d["freelist"]) == w["freelist_len"]
    assert digest(d["freelist"]) == w["freelist_sha256"]


def test_port_beyond_reference_index_limit():
    # 70 000 superblocks do not fit the reference's 16-bit queue index
    # (clIndexedQueue.cl:170); the widened port fills every usable
    # superblock (two 2040-byte blocks each), returns NULL once only the
    # free list's dummy is left, and drains back to the canonical state.
    sblocks = 70000
    n = 2 * sblocks
    ops = np.zeros((2 * n, 2), np.int64)
    ops[:n, 0], ops[:n, 1] = 0, 2000
    ops[n:, 0], ops[n:, 1] = 1, np.arange(n)
    with oracle.Port(sblocks, 12) as p:
        out = p.replay(ops)
        d = p.decode()
    usable = 2 * (sblocks - 2)
    assert np.all(out[:usable] >= 0) and np.all(out[usable:n] == -1)
    assert int(out[:usable].max()) // 4096 == sblocks - 3
    assert len(d["freelist"]) == sblocks - 1 and np.all(d["cls"] == -1)
