"""The lock-free structures and the PMA heap (include/kma_structs.h).

CPU: the committed fixtures equal the reference's own results (when the
reference build is present) and the sequential models used for the
concurrent checks agree with them.  GPU: one-thread replays equal the
fixtures exactly; concurrent runs conserve their contents."""
import os

import numpy as np
import pytest

import struct_streams as ss

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "structs.npz"))


def cases(prefix):
    return sorted({k.split("_")[1] for k in GOLD.files if k.startswith(prefix + "_")})


# ---------------------------------------------------------------- models
def queue_model(ops, dummy: bool):
    """FIFO semantics of clQueue (dummy=False) / clIndexedQueue (dummy=True:
    item 0 starts as the dummy, dequeue returns the old dummy)."""
    q = [0] if dummy else []
    out = []
    for kind, arg in ops:
        if kind == 0:
            q.append(int(arg))
            out.append(1)
        elif len(q) > (1 if dummy else 0):
            out.append(q.pop(0))
        else:
            out.append(-1)
    return np.array(out, np.int64), q


def tree_model(ops):
    """clTree add/get plus the logical remove: (results, live keys sorted).
    get returns the op index of the node holding the key."""
    node, live, out = {}, {}, []
    for i, (kind, key) in enumerate(ops):
        key = int(key)
        if kind == 0:
            if key not in node:
                node[key], live[key] = i, True
                out.append(1)
            elif live[key]:
                out.append(0)
            else:
                live[key] = True
                out.append(2)
        elif kind == 1:
            out.append(node[key] if key in node and live[key] else -1)
        else:
            if key in node and live[key]:
                live[key] = False
                out.append(1)
            else:
                out.append(0)
    return np.array(out, np.int64), np.array(sorted(k for k, v in live.items() if v), np.int64)


# ------------------------------------------------------------- CPU tests
def test_fixtures_are_the_references_results():
    from oracle import structs
    if not structs.available():
        pytest.skip("reference build not present")
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "mgs", os.path.join(ROOT, "tests", "golden", "make_golden_structs.py"))
    mgs = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mgs)
    fresh = mgs.cases()
    assert set(fresh) == set(GOLD.files)
    for k, v in fresh.items():
        np.testing.assert_array_equal(v, GOLD[k], err_msg=k)


@pytest.mark.parametrize("seed", cases("clq"))
def test_clqueue_fixture_is_fifo(seed):
    ops = GOLD[f"clq_{seed}_ops"]
    out, q = queue_model(ops, dummy=False)
    np.testing.assert_array_equal(out, GOLD[f"clq_{seed}_out"])
    fin = GOLD[f"clq_{seed}_fin"]
    assert fin[0] == (q[0] if q else -1) and fin[1] == (q[-1] if q else -1)
    for a, b in zip(q, q[1:]):  # the links walk the queue in order
        assert fin[2 + a] == b


@pytest.mark.parametrize("seed", cases("iq"))
def test_iqueue_fixture_returns_old_dummy(seed):
    ops = GOLD[f"iq_{seed}_ops"]
    out, q = queue_model(ops, dummy=True)
    np.testing.assert_array_equal(out, GOLD[f"iq_{seed}_out"])
    fin = GOLD[f"iq_{seed}_fin"]
    assert fin[0] == q[0] and fin[1] == q[-1]


@pytest.mark.parametrize("seed", cases("tree"))
def test_tree_fixture_matches_model(seed):
    ops = GOLD[f"tree_{seed}_ops"]
    out, keys = tree_model(ops)
    np.testing.assert_array_equal(out, GOLD[f"tree_{seed}_out"])
    np.testing.assert_array_equal(keys, GOLD[f"tree_{seed}_keys"])


def test_pma_fixture_is_a_bump_heap():
    keys = [k for k in GOLD.files if k.endswith("_ops") and k.startswith("pma")]
    for k in keys:
        ops, ref = GOLD[k], GOLD[k.replace("_ops", "_out")]
        nb = int(GOLD[k.replace("_ops", "_bytes")][0])
        head, out = 0, []
        for kind, arg in ops:
            if kind == 0:
                ret, head = head, head + int(arg)
                out.append(ret if ret + arg <= nb + 24 else -1)
            else:
                out.append(0)
        np.testing.assert_array_equal(out, ref, err_msg=k)


# ------------------------------------------------------------- GPU tests
@pytest.mark.gpu
@pytest.mark.parametrize("seed", cases("clq"))
def test_gpu_clqueue_replay_equals_reference(seed):
    from kma_b200 import structs
    n = int(GOLD[f"clq_{seed}_n"][0])
    out, fin = structs.clqueue_replay(n, GOLD[f"clq_{seed}_ops"])
    np.testing.assert_array_equal(out, GOLD[f"clq_{seed}_out"])
    np.testing.assert_array_equal(fin, GOLD[f"clq_{seed}_fin"])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", cases("iq"))
def test_gpu_iqueue_replay_equals_reference(seed):
    from kma_b200 import structs
    n = int(GOLD[f"iq_{seed}_n"][0])
    out, fin = structs.iqueue_replay(n, 4, GOLD[f"iq_{seed}_ops"])
    np.testing.assert_array_equal(out, GOLD[f"iq_{seed}_out"])
    np.testing.assert_array_equal(fin, GOLD[f"iq_{seed}_fin"])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", cases("tree"))
def test_gpu_tree_replay_equals_reference(seed):
    from kma_b200 import structs
    out, keys = structs.cltree_replay(GOLD[f"tree_{seed}_ops"])
    np.testing.assert_array_equal(out, GOLD[f"tree_{seed}_out"])
    np.testing.assert_array_equal(keys, GOLD[f"tree_{seed}_keys"])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [61, 62])
def test_gpu_tree_remove_matches_model(seed):
    from kma_b200 import structs
    ops = ss.tree_stream(seed, 3000, 300, remove=True)
    out, keys = structs.cltree_replay(ops)
    mout, mkeys = tree_model(ops)
    np.testing.assert_array_equal(out, mout)
    np.testing.assert_array_equal(keys, mkeys)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", cases("al"))
def test_gpu_arraylist_replay_equals_reference(seed):
    from kma_b200 import Heap, structs
    sblocks, osz = (int(x) for x in GOLD[f"al_{seed}_cfg"])
    with Heap(sblocks, 12) as h:
        out = structs.clarraylist_replay(osz, GOLD[f"al_{seed}_ops"], heap=h)
    np.testing.assert_array_equal(out, GOLD[f"al_{seed}_out"])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", cases("alg"))
def test_gpu_arraylist_group_equals_reference(seed):
    from kma_b200 import Heap, structs
    sblocks, osz = (int(x) for x in GOLD[f"alg_{seed}_cfg"])
    objs = GOLD[f"alg_{seed}_objs"]
    with Heap(sblocks, 12) as h:
        out = structs.clarraylist_group(osz, objs, mode=0, heap=h)
    np.testing.assert_array_equal(out, GOLD[f"alg_{seed}_out"])
    if len(objs) <= 32:  # one warp: the warp form gives the same page and slices
        with Heap(sblocks, 12) as h:
            outw = structs.clarraylist_group(osz, objs, mode=1, heap=h)
        np.testing.assert_array_equal(outw, GOLD[f"alg_{seed}_out"])


@pytest.mark.gpu
def test_gpu_arraylist_group_block_of_many_warps():
    """A 1000-thread block shares one page; each warp form gets its own."""
    from kma_b200 import Heap, structs
    rng = np.random.default_rng(7)
    objs = rng.integers(0, 3, size=1000).astype(np.uint32)
    with Heap(256, 14) as h:
        out = structs.clarraylist_group(4, objs, mode=0, heap=h)
    live = objs > 0
    assert np.all(out[~live] == -1) and np.all(out[live] >= 0)
    excl = np.concatenate([[0], np.cumsum(objs)[:-1]]) * 4
    base = out[live][0] - excl[live][0]
    np.testing.assert_array_equal(out[live], base + excl[live])
    with Heap(256, 14) as h:
        outw = structs.clarraylist_group(4, objs, mode=1, heap=h)
    for w in range(0, 1000, 32):
        o, k = outw[w:w + 32], objs[w:w + 32]
        lv = k > 0
        if lv.any():
            ex = np.concatenate([[0], np.cumsum(k)[:-1]]) * 4
            np.testing.assert_array_equal(o[lv], o[lv][0] - ex[lv][0] + ex[lv])


@pytest.mark.gpu
@pytest.mark.parametrize("key", [k[:-4] for k in GOLD.files if k.startswith("pma") and k.endswith("_ops")])
def test_gpu_pma_replay_equals_reference(key):
    from kma_b200 import structs
    nb = int(GOLD[f"{key}_bytes"][0])
    with structs.Pma(nb) as p:
        out = p.replay(GOLD[f"{key}_ops"])
    np.testing.assert_array_equal(out, GOLD[f"{key}_out"])


@pytest.mark.gpu
def test_gpu_arraylist_on_pma_is_a_bump_sequence():
    """The PMA backend (the reference's source-concatenation switch): pages
    are consecutive bump allocations of objs*size + 24 bytes."""
    from kma_b200 import structs
    ops = ss.arraylist_stream(71, 200, 9)
    with structs.Pma(1 << 20) as p:
        out = structs.clarraylist_replay(8, ops, pma=p)
    head, pages = 0, []  # (start offset of the objects, count)
    for (kind, arg), r in zip(ops, out):
        if kind == 0:
            assert r == head + 24
            pages.append((head + 24, int(arg)))
            head += int(arg) * 8 + 24
        elif kind == 1:
            i = int(arg)
            for start, cnt in pages:
                if i < cnt:
                    assert r == start + i * 8
                    break
                i -= cnt
        else:
            pages = []


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1], ids=["clqueue", "iqueue"])
@pytest.mark.parametrize("form,shards,threads,per", [
    ("thread", 1, 4096, 16), ("thread", 64, 4096, 16),
    ("warp", 1, 4096, 16), ("warp", 64, 4096, 16), ("warp", 1, 1000, 7),
    ("block", 1, 4096, 16), ("block", 1, 1000, 7), ("block", 1, 1 << 16, 64),
])
def test_gpu_c3_queue_conserves_payloads(kind, form, shards, threads, per):
    """Every payload enqueued is dequeued once (per-thread calls, the warp
    forms with their chain log, and the block forms, whose holds take
    several chains), and the queue's links end consistent with its tail;
    thread counts that leave partial warps and blocks included."""
    from kma_b200 import structs
    flag = {"thread": 0, "warp": structs.C3_WARP, "block": structs.C3_BLOCK}[form]
    st = structs.c3_queue(kind | flag, threads, per, shards, seed=0xC3)
    if form != "thread" and shards == 1:
        assert st["log_chains"] > 0  # (over 64 shards a warp's lanes name different queues: no chains)
    n = threads * per
    assert st["err"] == 0 and st["walk_ok"] == 1
    assert st["enqueued"] == n
    assert st["out_count"] == n
    assert st["out_xor"] == st["in_xor"] and st["out_sum"] == st["in_sum"]
    assert st["in_sum"] == n * (n - 1) // 2  # the payloads are a permutation of 0..n-1
    assert st["in_xor"] == int(np.bitwise_xor.reduce(np.arange(n, dtype=np.uint64)))


@pytest.mark.gpu
@pytest.mark.parametrize("kind,state", [(0, 0), (0, 1), (1, 0)],
                         ids=["clqueue_head_held", "clqueue_append_unlinked", "iqueue_head_held"])
def test_gpu_stuck_queue_dequeue_gives_up_and_flags(kind, state):
    """On the device, a dequeue on a queue nothing will ever free (a holder
    that is gone, an append that never linked) ends after its spin limit,
    returns NULL and raises the timeout flag: no hang, no fault."""
    import ctypes
    from kma_b200 import KMA_FLAG_TIMEOUT
    from kma_b200._lib import lib
    taken, flags = ctypes.c_int64(0), ctypes.c_uint32(0)
    assert lib().kma_debug_queue_stuck_dequeue(kind, state, 4096, -1, ctypes.byref(taken),
                                               ctypes.byref(flags)) == 0
    assert taken.value == -1
    assert flags.value & KMA_FLAG_TIMEOUT


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1], ids=["clqueue", "iqueue"])
@pytest.mark.parametrize("tpb,calls", [(256, 4), (512, 3), (64, 8)])
def test_gpu_block_form_keeps_fifo_order(kind, tpb, calls):
    """Warps append their chains one after another (warp forms, chain log),
    then the block takes them back with the block form: each call returns
    exactly the next tpb items in queue order, and the lanes of a warp get
    consecutive items (the indexed queue hands out its initial dummy first,
    as the reference's does)."""
    import ctypes
    from kma_b200._lib import lib
    out = np.zeros(tpb * calls, np.int64)
    err = ctypes.c_uint32(0)
    assert lib().kma_debug_queue_block_fifo(kind, tpb, calls, -1, out.ctypes.data, ctypes.byref(err)) == 0
    assert err.value == 0
    pos = out.copy() if kind == 0 else np.where(out == -2, 0, out + 1)  # queue positions
    assert (out != -1).all()
    pos = pos.reshape(calls, tpb)
    for c in range(calls):
        np.testing.assert_array_equal(np.sort(pos[c]), np.arange(c * tpb, (c + 1) * tpb))
        warps = pos[c].reshape(-1, 32)
        np.testing.assert_array_equal(warps - warps[:, :1], np.tile(np.arange(32), (tpb // 32, 1)))


@pytest.mark.gpu
def test_gpu_c3_tree_equals_sequential_replay():
    from kma_b200 import structs
    rng = np.random.default_rng(0xC3)
    n = 1 << 16
    kinds = rng.choice(3, size=n, p=(0.5, 0.3, 0.2)).astype(np.uint8)
    keys = rng.integers(0, 1 << 14, size=n).astype(np.uint32)  # repeats, so ops interact
    res, st = structs.c3_tree(kinds, keys, threads=2048)
    mout, mkeys = tree_model(np.stack([kinds, keys], 1))
    expect = np.where(kinds == 1, (mout >= 0).astype(np.int64), mout)
    np.testing.assert_array_equal(res.astype(np.int64), expect)
    assert st["err"] == 0 and st["sorted"] == 1
    assert st["live_keys"] == len(mkeys)
    assert st["keys_sum"] == int(mkeys.sum())
    x = 0
    for k in mkeys:
        x ^= int(k)
    assert st["keys_xor"] == x
