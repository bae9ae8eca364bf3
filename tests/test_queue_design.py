"""The queue algorithms of include/kma_queue_algo.cuh on host threads (no GPU).

oracle/queue_harness runs the same algorithm text the GPU runs, bound to
host atomics: producers append chains (a warp's items) and single items,
consumers take batches and re-append some of what they take (items leave
and re-enter the queue), and an append sometimes sleeps between its
exchange of the tail and its link -- the window in which its chain is not
reachable yet.  Every run must conserve every append, keep each appender's
order, end with a consistent head/tail, and never run out a wait.

The second test plants one mistake at a time in a scratch copy of the
algorithm (never in the product) and checks the harness reports it, so a
passing run means something.
"""
import json
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
HARNESS = os.path.join(ORACLE, "queue_harness")
ALGO = os.path.join(ROOT, "include", "kma_queue_algo.cuh")

# threads chains max_chain deq_batch delay_prob seed producers recycle log_records [phased]
# (a negative max_chain / deq_batch: every chain / batch exactly that long;
# phased: consumers start when the producers are done, as config 3 runs)
CONFIGS = [
    "8 20000 1 1 0.01 1 1 0.5 0",      # single items, one producer: the queue is mostly empty
    "8 20000 4 4 0.01 2 2 0.5 0",
    "8 5000 32 32 0.02 3 4 0.5 0",     # warp-sized chains and batches, many delayed appends
    "8 3000 32 32 0.002 4 4 0.9 0",
    "8 40000 32 32 0.0005 5 4 0 0",    # no recycling: plain producer/consumer
    "3 20000 8 8 0.01 6 1 0.5 0",
    # with a chain log: large (records outlive their chains), and small
    # (records overwritten while their chains are queued: stale records)
    "8 5000 32 32 0.02 7 4 0.5 65536",
    "8 5000 32 32 0.02 8 4 0.5 8",
    "8 20000 8 8 0.01 9 2 0.5 2",
    "8 40000 32 32 0.0005 10 4 0 1024",
    # batches larger than a chain: one hold takes several logged chains
    # (the block forms), with long and short chains, large and stale logs
    "8 5000 32 128 0.02 11 4 0.5 65536",
    "8 5000 32 256 0.02 12 4 0.5 8",
    "8 20000 8 64 0.01 13 2 0.5 1024",
    "8 40000 32 256 0.0005 14 4 0 1024",
    # warp-sized chains taken by block-sized batches from a full queue:
    # several whole chains per hold, each reached over its marked link
    "8 5000 -32 -256 0.02 15 4 0.5 65536 1",
    "8 5000 -32 -256 0.02 16 4 0.5 16 1",
    "8 5000 -8 -64 0.01 17 2 0.5 1024 1",
    "8 5000 32 -256 0.02 19 4 0.5 65536 1",
]

# block-sized batches (256) over whole warp chains (32): every chain must
# come out of its record, eight to a hold of the head, not by walking
LOG_PATH_CFG = "8 5000 -32 -256 0 15 4 0 65536 1"


def log_path_use(binary, kind):
    """(share of chains taken from their records, chains per dequeue call)"""
    rc, st = run(binary, kind, LOG_PATH_CFG)
    assert rc == 0 and st.get("ok"), st
    return st["log_chains"] / (st["appended"] / 32), st["log_chains"] / st["dequeue_calls"]


@pytest.mark.parametrize("kind", ["clq", "iq"])
def test_block_batches_take_whole_chains_from_the_log(harness, kind):
    share, per_call = log_path_use(harness, kind)
    assert share > 0.9 and per_call > 6

def test_log_path_check_sees_a_wrong_record_number(harness, tmp_path):
    """Plant a wrong record number on the path that reads it from the link
    into a chain: those records never match, so each hold stops after its
    first chain, and the chains-per-call figure above collapses (the check
    above would catch it)."""
    src = open(ALGO).read()
    old = "((via_into ? into : l1) >> PTR_BITS) & 0x3FFFu"
    assert src.count(old) == 1
    d = tmp_path / "into"
    d.mkdir()
    (d / "kma_queue_algo.cuh").write_text(src.replace(old, "((via_into ? into + (1ull << PTR_BITS) : l1) >> PTR_BITS) & 0x3FFFu"))
    binary = str(d / "h")
    subprocess.run([os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-pthread", f"-I{d}", "-o", binary,
                    os.path.join(ORACLE, "queue_harness.cpp")], check=True)
    assert log_path_use(binary, "clq")[1] < 2


def have_compiler() -> bool:
    return shutil.which(os.environ.get("CXX", "g++")) is not None


def run(binary, kind, cfg, timeout=300):
    r = subprocess.run([binary, kind, *cfg.split()], capture_output=True, text=True, timeout=timeout)
    line = r.stdout.strip().splitlines()[-1] if r.stdout.strip() else "{}"
    return r.returncode, json.loads(line) if line.startswith("{") else {}


@pytest.fixture(scope="module")
def harness():
    if not have_compiler():
        pytest.skip("no C++ compiler")
    subprocess.run(["make", "-s", "-C", ORACLE, "queue_harness"], check=True)
    return HARNESS


@pytest.mark.parametrize("kind", ["clq", "iq"])
@pytest.mark.parametrize("cfg", CONFIGS)
def test_queue_algorithm_conserves_and_keeps_order(harness, kind, cfg):
    rc, st = run(harness, kind, cfg)
    assert rc == 0 and st.get("ok"), st
    assert st["taken"] + st["left"] >= st["appended"] > 0
    assert st["conservation_faults"] == 0 and st["order_faults"] == 0 and st["timeouts"] == 0


def test_stuck_queues_end_every_wait(harness):
    """A dequeuer that died holding the head, and an append that exchanged
    the tail but never linked: a dequeue on such a queue gives up after
    `limit` tries in which the head did not move, reports the expiry and
    leaves the queue as it found it."""
    r = subprocess.run([harness, "stuck"], capture_output=True, text=True, timeout=60)
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    assert r.returncode == 0 and lines[-1] == {"stuck_ok": True}, r.stdout
    assert {x["case"] for x in lines[:-1]} == {"clq_head_held", "clq_append_unlinked", "iq_head_held"}
    assert all(x["timed_out"] and x["taken"] == 0 for x in lines[:-1])


# Each mutant breaks one step the algorithm depends on.
MUTANTS = {
    # link after the previous tail with a plain store: a dequeuer's hold
    # of that link (POISON) is overwritten, and its restore then cuts the chain
    "append_link_store": ("clq", "8 20000 1 1 0.01 1 1 0.5",
                          "const u64 old = O::cas(pl, 0ull, first | into);",
                          "const u64 old = 0; O::st(pl, first | into);"),
    # no check that the held item is still the head (ABA after recycling)
    "no_head_recheck": ("clq", "8 20000 4 4 0.01 2 2 0.5",
                        "\t\tif (O::ld(headw) != h) {\n\t\t\tO::st(hl, nx);",
                        "\t\tif (false) {\n\t\t\tO::st(hl, nx);"),
    # take the last linked item without checking the tail: an append in
    # its window is lost
    "last_item_no_tail_cas": ("clq", "8 20000 1 1 0.01 1 1 0.5",
                              "\t\tif (O::cas(tailw, hp, 0ull) == hp) {",
                              "\t\tif (true) { O::st(tailw, 0ull);"),
    # take the indexed queue's head hold with a plain store: two dequeuers
    # hold it at once and take the same items
    # a hold that takes several chains forgets to return the later ones
    # (shows that batches larger than a chain do take several chains)
    "multi_chain_dropped": ("clq", "8 5000 32 128 0.02 11 4 0.5 65536",
                            "\t\t\t\tm += m2;\n",
                            "\t\t\t\t(void)m2;\n"),
    "iq_multi_chain_dropped": ("iq", "8 5000 32 128 0.02 11 4 0.5 65536",
                               "\t\t\t\tr += r2;\n",
                               "\t\t\t\t(void)r2;\n"),
    "iq_hold_store": ("iq", "8 20000 4 4 0.01 2 2 0.5",
                      "\t\tif (O::cas(headw, hd, tw_make(tw_tag(hd) + 1u, cur)) != hd) {",
                      "\t\tO::st(headw, tw_make(tw_tag(hd) + 1u, cur));\n\t\tif (false) {"),
}


@pytest.mark.parametrize("name", sorted(MUTANTS))
def test_harness_detects_planted_mistakes(harness, tmp_path, name):
    kind, cfg, old, new = MUTANTS[name]
    src = open(ALGO).read()
    assert src.count(old) == 1, f"mutation site of {name} not found once"
    d = tmp_path / name
    d.mkdir()
    (d / "kma_queue_algo.cuh").write_text(src.replace(old, new))
    binary = str(d / "h")
    subprocess.run([os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-pthread", f"-I{d}", "-o", binary,
                    os.path.join(ORACLE, "queue_harness.cpp")], check=True)
    # a fault shows up in most runs, not all: up to four seeds, the first
    # detection is enough
    st = {}
    for seed in range(4):
        args = cfg.split()
        args[5] = str(int(args[5]) + 100 * seed)
        try:
            rc, st = run(binary, kind, " ".join(args), timeout=120)
        except subprocess.TimeoutExpired:
            return  # a wait that never ends is a detection too
        if rc != 0:
            return
    raise AssertionError(f"mutant {name} passed unnoticed: {st}")
