#!/usr/bin/env python
"""Throughput of the KMA device heap on the fragmentation stress workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): config 2 -- a 1 GiB heap of 16 KiB superblocks, 148 x
2048 work-items, 64 rounds; each round every item mallocs 8 << U{0..8}
bytes, tags every word of the block with its id, then frees a seeded 50%
of its live blocks after verifying their tags; after the last round the
live set is drained.  A step is reset + seed + rounds + drain on a heap
resident in HBM.  op = one malloc call or one free call.

Our arm times K steps with CUDA events on the launching stream (L2 flushed
between steps, outside the timed events), max over ranks; N > 1 runs
independent per-GPU heap replicas (weak scaling: the heap does not shard
and has no exchange step).  It also reports the plain per-thread kernel on
the same GPU, the roofline of the dominant kernel, the CPU baseline, the
end-to-end figure through the host-buffer C ABI call, the invariant check
of one extra step, and (under "forms") the other configurations: the
lock-free structures (config 3: one clQueue and one indexed queue at full
size through the warp and block forms, and the tree), the autotuned
batched form (config 4) and the served form's p50/p99 latency at swept
arrival rates (config 5), each beside the plain per-thread calls on the
same work, with PMA arms where the PMA heap applies, and the graph build
of the reference's tree driver.  The reference arm times the reference's
own kma.cl built as host C (oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "M malloc+free ops/s on 1 B200 (0 heap-invariant faults); p99 serving latency"
UNIT = "Mops/s"
ITEMS = 148 * 2048
ROUNDS = 64
SBLOCKS = 65536
SB_LOG2 = 14
SEED = 0xC2
MEAN_REQ = (8 + 16 + 32 + 64 + 128 + 256 + 512 + 1024 + 2048) / 9.0
WORKLOAD = ("C2 fragmentation stress: 1 GiB heap of 16 KiB superblocks, 148x2048 items, 64 rounds, "
            "malloc 8<<U{0..8} B per round, seeded 50% frees of the live set, every word tagged and "
            "verified; step = reset + seed + rounds + drain")
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "c2_rounds_warp_traffic.json")


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "src": "measured"}
    except Exception:  # noqa: BLE001 - file absent: the recipe's fallback
        return {"hbm_gbs": 6650.0, "src": "fallback"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The largest x over all ranks: a replicated job takes as long as its
    slowest replica.  Every rank must call it (a collective when world > 1)."""
    if world == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, ops_per_rank_step: int, steps: int, total_ms: float) -> float:
    """Whole-job M ops/s: every rank's ops over the slowest rank's time."""
    return world * ops_per_rank_step * steps / (total_ms / 1e3) / 1e6


# ---------------------------------------------------------------- CPU legs
def cpu_run(kind_pref: str, items: int, threads: int, timeout: float) -> dict:
    """Run the reference's kma.cl (oracle/_ref; the C restatement when the
    reference build is absent) on `threads` host threads over `items`
    work-items of the workload, in a child process with a time limit."""
    code = f"""
import json, sys
sys.path.insert(0, {ROOT!r})
from oracle import oracle
kind = "reference" if oracle.ref_available({SB_LOG2}) and {kind_pref!r} == "reference" else "port"
H = oracle.Ref if kind == "reference" else oracle.Port
with H({SBLOCKS}, {SB_LOG2}) as h:
    st = h.run_workload(2, {items}, {ROUNDS}, {SEED}, 2, {threads})
st["kind"] = kind
print(json.dumps(st))
"""
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            return {"error": r.stderr.strip().splitlines()[-1:]}
        return json.loads(r.stdout.strip().splitlines()[-1])
    except subprocess.TimeoutExpired:
        return {"error": f"timed out after {timeout:.0f} s"}


def cpu_sample(items: int, threads: int, kind: str) -> str:
    what = ("kma.cl+clIndexedQueue.cl built unmodified as host C" if kind == "reference"
            else "C restatement of kma.cl")
    return (f"{items} of the {ITEMS} work-items x {ROUNDS} rounds per step (1 GiB heap, 16 KiB "
            f"superblocks), work-items round-robin on {threads} pthread{'s' if threads != 1 else ''}, "
            f"each to completion; {what}")


def run_reference(args) -> int:
    """The reference arm: the reference's own kma.cl as host C on all host
    threads, every step the whole config-2 program (all work-items)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    items = ITEMS
    vals = []
    last = None
    for k in range(args.warmup + args.steps):
        st = cpu_run("reference", items, threads, timeout=300)
        if "error" in st:
            print(json.dumps({"impl": "reference", "unavailable": f"CPU run failed: {st['error']}"}))
            return 0
        if k >= args.warmup:
            vals.append((st["mallocs"] + st["frees"]) / st["seconds"] / 1e6)
            last = st
    v = statistics.median(vals)
    kind = last["kind"]
    line = {"metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * last["seconds"], 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "items": items, "rounds": ROUNDS,
                       "heap_bytes": SBLOCKS << SB_LOG2, "sb_size": 1 << SB_LOG2,
                       "ops_per_step": int(last["mallocs"] + last["frees"]), "threads": threads,
                       "invariant_faults": int(last["bad_tags"]), "nulls": int(last["nulls"])},
            "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": cpu_sample(items, threads, kind)},
            "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------ other forms (rank 0)
def tree_expected(kinds, keys):
    """Sequential results of the config-3 tree ops (1 inserted / 0 exists /
    2 revived; lookup 1 found / 0; remove 1 / 0): keys seen once are decided
    in bulk, repeated keys replayed in op order."""
    import numpy as np
    res = np.where(kinds == 0, 1, 0).astype(np.int8)
    uniq, inv, cnt = np.unique(keys, return_inverse=True, return_counts=True)
    rep = np.nonzero(cnt[inv] > 1)[0]
    live, seen = {}, set()
    for j in rep:
        k, kind = int(keys[j]), int(kinds[j])
        if kind == 0:
            res[j] = 1 if k not in seen else (0 if live[k] else 2)
            seen.add(k)
            live[k] = True
        elif kind == 1:
            res[j] = 1 if live.get(k, False) else 0
        else:
            res[j] = 1 if live.get(k, False) else 0
            if k in live:
                live[k] = False
    n_live = int(np.sum((cnt[inv] == 1) & (kinds == 0))) + sum(1 for v in live.values() if v)
    return res, n_live


def c3_line(kind: int, threads: int, per: int, shards: int) -> dict:
    """One config-3 queue run: enqueue / dequeue rates and conservation."""
    from kma_b200 import structs
    st = structs.c3_queue(kind, threads, per, shards, seed=0xC3)
    n = threads * per
    ok = (st["out_count"] == n and st["out_xor"] == st["in_xor"] and st["out_sum"] == st["in_sum"]
          and st["walk_ok"] == 1 and st["err"] == 0)
    t = (st["enqueue_ms"] + st["dequeue_ms"]) / 1e3
    form = "block" if kind & structs.C3_BLOCK else ("warp" if kind & structs.C3_WARP else "thread")
    return {"payloads": n, "threads": threads, "shards": shards, "calls": form,
            "conserved": bool(ok), "enqueue_mops": round(n / st["enqueue_ms"] / 1e3, 2),
            "dequeue_mops": round(n / st["dequeue_ms"] / 1e3, 2), "mops": round(2 * n / t / 1e6, 2)}


def time_batch(b, block_dim: int, depth: int, reps: int = 2) -> tuple[float, dict]:
    """Mean device ms of a captured batch run (CUDA events on the capture
    stream, one warm-up launch) and the counters of the last run."""
    import torch
    stream = torch.cuda.Stream()
    b.capture(block_dim, depth, stream)
    b.launch(stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        b.launch(stream)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps, b.stats(stream)


def measure_forms(quick: bool = False) -> dict:
    """Config 3 (structures), 4 (batched, autotuned) and 5 (served) on this
    GPU: each its own workload at its configured size, timed on the device,
    beside the plain per-thread calls on the same work and the PMA heap."""
    import numpy as np
    from kma_b200 import MODE_PLAIN, Heap, structs
    from kma_b200.batch import Batch, autotune, c4_jobs
    from kma_b200.serve import Server, c5_requests
    out = {}
    # config 3: one clQueue and one clIndexedQueue (the reference's single
    # structures), 2^24 payloads by 2^18 threads x 64, through the warp
    # forms and through the block forms (warp-chained enqueues, dequeues
    # combined per block of 256); the per-thread calls on one queue at 2^16
    # payloads (at full size their waits on the one head run out); 4096
    # independent shards as an extra
    c3 = {}
    big = (1 << 18, 64) if not quick else (1 << 14, 64)
    for name, kind in (("clqueue", structs.C3_CLQUEUE), ("iqueue", structs.C3_IQUEUE)):
        c3[f"{name}_single"] = c3_line(kind | structs.C3_WARP, big[0], big[1], 1)
        c3[f"{name}_single_block"] = c3_line(kind | structs.C3_BLOCK, big[0], big[1], 1)
        c3[f"{name}_single_per_thread_small"] = c3_line(kind, 1 << 12, 16, 1)
        c3[f"{name}_shards4096"] = c3_line(kind, big[0], big[1], 4096)
        c3[f"{name}_shards4096_warp"] = c3_line(kind | structs.C3_WARP, big[0], big[1], 4096)
    rng = np.random.default_rng(0xC3)
    nt = 1 << 22
    kinds = rng.choice(3, size=nt, p=(0.5, 0.3, 0.2)).astype(np.uint8)
    keys = rng.integers(0, 1 << 32, size=nt, dtype=np.uint64).astype(np.uint32)
    res, st = structs.c3_tree(kinds, keys, threads=1 << 18)
    exp, n_live = tree_expected(kinds, keys)
    c3["tree"] = {"ops": nt, "mops": round(nt / st["ms"] / 1e3, 1),
                  "equals_sequential": bool(np.array_equal(res, exp) and st["live_keys"] == n_live
                                            and st["sorted"] == 1 and st["err"] == 0)}
    out["structures_c3"] = c3
    # config 4: 64 jobs of 1k..1M threads, 16 GiB heap, autotuned over the
    # geometries that serve every size the jobs draw; then the same jobs
    # with plain per-thread calls, and on a PMA heap
    t, sd = c4_jobs()
    grid = dict(sb_log2s=(12, 14, 16), block_dims=(128, 256, 512), depths=(0, 2, 4)) if not quick else \
        dict(sb_log2s=(12, 14), block_dims=(256,), depths=(0, 4))
    entries, best = autotune(t, sd, rounds=16, heap_bytes=16 << 30, warmup=1, reps=2, **grid)
    b = entries[best]

    def nulls(e):
        return {"null_frac": round(e["nulls"] / e["mallocs"], 4), "refused": e["refused"],
                "exhausted": e["nulls"] - e["refused"]}
    c4 = {"jobs": 64, "work_items": int(t.sum()), "rounds": 16, "heap_bytes": 16 << 30,
          "best": {"sb_size": b["sb_size"], "block_dim": b["block_dim"], "cache_depth": b["cache_depth"],
                   "mops": b["mops"], "ms_per_launch": b["ms"], **nulls(b), "bad_tags": b["bad_tags"],
                   # algorithmic payload bytes (tag fill + verify, counted by the kernel) per launch
                   "payload_gbs": round((b["fill_bytes"] + b["verify_bytes"]) / b["ms"] / 1e6, 1),
                   "hbm_frac": round((b["fill_bytes"] + b["verify_bytes"]) / b["ms"] / 1e6 / peaks()["hbm_gbs"], 4)},
          "grid": [[e["sb_size"], e["block_dim"], e["cache_depth"], e["mops"], e["serves_all"],
                    round(e["nulls"] / e["mallocs"], 4), e["refused"]] for e in entries],
          "grid_cols": ["sb_size", "block_dim", "cache_depth", "mops", "serves_all", "null_frac", "refused"],
          "launch": "one CUDA graph per configuration: heap reset + job seeding + one persistent kernel"}
    lg = b["sb_size"].bit_length() - 1
    with Heap((16 << 30) >> lg, lg) as h, Batch(h, t, sd, rounds=16, mode=MODE_PLAIN) as pb:
        ms, stp = time_batch(pb, b["block_dim"], 0)
    plain_mops = (stp["mallocs"] + stp["frees"]) / ms / 1e3
    c4["plain_same_workload"] = {"sb_size": b["sb_size"], "block_dim": b["block_dim"], "mops": round(plain_mops, 1),
                                 "ms_per_launch": round(ms, 3), **nulls(stp), "bad_tags": stp["bad_tags"],
                                 "calls": "kma_malloc / kma_free per thread"}
    c4["batched_over_plain_same_workload"] = round(b["mops"] / plain_mops, 3)
    pma = {}
    with structs.Pma(32 << 30) as p:
        for mname, mode in (("warp", 1), ("plain", MODE_PLAIN)):
            with Batch(p, t, sd, rounds=16, mode=mode) as pb:
                ms, stp = time_batch(pb, b["block_dim"], 0)
            pma[mname] = {"mops": round((stp["mallocs"] + stp["frees"]) / ms / 1e3, 1),
                          "ms_per_launch": round(ms, 3), **nulls(stp), "bad_tags": stp["bad_tags"]}
    c4["pma_32GiB"] = pma
    out["batched_c4"] = c4
    # config 5: 64 GiB resident heap, Poisson arrivals at swept rates, warp
    # calls; the all-at-once load again with plain per-thread calls; and a
    # 1 GiB heap with 64 slots, where the 85% occupancy admission, not the
    # slots, bounds how many requests run at once
    served = []

    def load(srv, rate, nreq=300, seed=0xC5, heap_bytes=64 << 30, calls="warp"):
        nv, seeds, arr = c5_requests(seed, nreq, rate=rate if rate else 1.0)
        res_s, summ = srv.run(nv, seeds, arr if rate else None, realtime=bool(rate))
        ok = [r for r in res_s if r["status"] == "ok"]
        lat = np.array([r["latency_s"] for r in ok]) if ok else np.zeros(1)
        return {"rate_per_s": rate or "all at once", "heap_bytes": heap_bytes, "calls": calls,
                "requests": len(res_s), "ok": len(ok),
                "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
                "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3),
                "mops": round(summ["ops"] / summ["wall_s"] / 1e6, 1),
                "requests_per_s": round(len(res_s) / summ["wall_s"], 1),
                "max_running": summ["max_running"], "max_occupancy": round(summ["max_occupancy"], 4),
                "max_reserved": round(summ["max_reserved"], 4), "admit_waits_for_room": summ["admit_waits"]}
    with Heap((64 << 30) >> 14, 14) as h:
        with Server(h, slots=16) as srv:
            for rate in ((200, 3200, 0) if not quick else (3200, 0)):
                served.append(load(srv, rate))
        with Server(h, slots=16, mode=MODE_PLAIN) as srv:
            served.append(load(srv, 0, calls="plain"))
        flags = h.error_flags()
    with Heap((1 << 30) >> 14, 14) as h, Server(h, slots=64, max_vertices=4_000_000) as srv:
        served.append(load(srv, 0, nreq=200, seed=0xC55, heap_bytes=1 << 30))
        flags |= h.error_flags()
    warp_all = next(x for x in served if x["rate_per_s"] == "all at once" and x["calls"] == "warp"
                    and x["heap_bytes"] == 64 << 30)
    plain_all = next(x for x in served if x["calls"] == "plain")
    out["served_c5"] = {"heap_bytes": 64 << 30, "slots": 16, "occupancy_limit": 0.85,
                        "graph": "N log-uniform 1k..4M vertices, degrees ~ d^-2.1 on 1..4096",
                        "heap_error_flags": flags, "loads": served,
                        "served_over_plain_same_workload": round(warp_all["mops"] / plain_all["mops"], 3)
                        if plain_all["mops"] else None}
    out["graph_build"] = measure_graph_build(quick)
    return out


def edge_mix(a, b):
    """mix(source, sink) as the library computes it (SplitMix64 finaliser
    of source << 32 | sink), vectorised."""
    import numpy as np
    with np.errstate(over="ignore"):
        z = (a.astype(np.uint64) << np.uint64(32) | b.astype(np.uint64)) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def measure_graph_build(quick: bool = False) -> dict:
    """The tree driver's graph build (nodes in a clTree, a clQueue of links
    per node, every node and link a heap block) on synthetic edges: each
    build is followed by the teardown that frees every block, and must give
    the edge multiset back and leave the heap canonically empty.  Two rank
    distributions: Zipf(1.1), where the hottest vertex's one link queue
    takes a large share of all enqueues, and uniform.  The same kernels
    also run on a PMA heap (which frees nothing; reset between builds)."""
    import statistics
    import numpy as np
    from kma_b200 import Heap, graph, structs
    from kma_b200 import inspect as ins
    n_e, n_v = (1 << 22, 1 << 20) if not quick else (1 << 18, 1 << 16)
    threads = 148 * 1024
    out = {"edges": n_e, "vertices_drawn_from": n_v, "threads": threads, "heap_bytes": 1 << 30,
           "sb_size": 1 << 14, "keys": "distinct random u32 per vertex rank"}
    for name, skew in (("zipf1.1", 1.1), ("uniform", 0.0)):
        e = graph.synth_edges(0x6A, n_e, n_v, skew=skew)
        m = edge_mix(e[:, 0], e[:, 1])
        want = dict(nodes=len(np.unique(e)), links=n_e, edge_xor=int(np.bitwise_xor.reduce(m)),
                    edge_sum=int(m.sum(dtype=np.uint64)))
        max_out = int(np.unique(e[:, 0], return_counts=True)[1].max())
        ms, ok, lost = [], True, 0
        with Heap((1 << 30) >> 14, 14) as h:
            for _ in range(3):
                st, _ = graph.build(h, e, threads=threads, free_after=True)
                ms.append(float(st["build_ms"]))
                lost = int(st["lost_adds"])
                ok = ok and all(int(st[k]) == v for k, v in want.items()) and \
                    st["err"] == 0 and st["nulls"] == 0 and st["sorted"] == 1
            empty = ins.check_canonical_empty(h.snapshot(), h.bitmaps()) == []
            flags = h.error_flags()
        t = statistics.median(ms)
        pms, pok = [], True
        with structs.Pma(1 << 30) as p:
            for _ in range(3):
                p.reset()
                st, _ = graph.build(p, e, threads=threads)
                pms.append(float(st["build_ms"]))
                pok = pok and all(int(st[k]) == v for k, v in want.items()) and \
                    st["err"] == 0 and st["nulls"] == 0 and st["sorted"] == 1
        tp = statistics.median(pms)
        out[name] = {"nodes": want["nodes"], "max_out_degree": max_out, "build_ms": round(t, 3),
                     "medges_per_s": round(n_e / t / 1e3, 2), "lost_adds": lost,
                     "edges_conserved": bool(ok), "empty_after_teardown": bool(empty),
                     "heap_error_flags": flags,
                     "pma": {"build_ms": round(tp, 3), "medges_per_s": round(n_e / tp / 1e3, 2),
                             "edges_conserved": bool(pok)}}
    return out


def measure_cpu_baseline(items: int | None = None) -> dict:
    """The reference's kma.cl as host C on this host's cores, over the same
    sample on all hardware threads (the reported baseline) and on one
    thread (the reference's CPU throughput falls as threads are added, so
    both are given).  The sample is the whole config-2 program unless
    `items` names fewer work-items."""
    threads = os.cpu_count() or 1
    items = ITEMS if items is None else items
    c = cpu_run("reference", items, threads, timeout=300)
    if "error" in c:
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"unavailable: {c['error']}"}
    cpu = {"value": round((c["mallocs"] + c["frees"]) / c["seconds"] / 1e6, 3),
           "unit": UNIT, "cores": threads, "kind": c["kind"],
           "sample": cpu_sample(items, threads, c["kind"]) + f"; its own tag faults: {c['bad_tags']}"}
    c1 = cpu_run("reference", items, 1, timeout=300)
    if "error" not in c1:
        cpu["one_thread"] = {"value": round((c1["mallocs"] + c1["frees"]) / c1["seconds"] / 1e6, 3),
                             "unit": UNIT, "cores": 1,
                             "sample": cpu_sample(items, 1, c1["kind"]) + f"; its own tag faults: {c1['bad_tags']}"}
    else:
        cpu["one_thread"] = {"value": None, "unit": UNIT, "cores": 1, "sample": f"unavailable: {c1['error']}"}
    return cpu


# ---------------------------------------------------------------- GPU arm
def run_ours(args) -> int:
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from kma_b200 import MODE_PLAIN, MODE_WARP, WL_C2, Heap, Workload, bench_atomics
    from kma_b200 import inspect as ins

    mode = MODE_WARP if args.mode == "warp" else MODE_PLAIN
    stream = torch.cuda.current_stream()
    # the warp heap's waits are bounded at 2^18 iterations (well under a
    # second; legitimate waits here last microseconds), so a wait that
    # cannot be met shows as a flagged NULL in its step instead of a long
    # stall; the per-thread heap on the reference's single structures keeps
    # the default 2^22, its threads legitimately wait far longer
    SPIN = 0 if mode == MODE_PLAIN else 1 << 18
    heap = Heap(SBLOCKS, SB_LOG2, stream=stream, compat=(mode == MODE_PLAIN), shards=args.shards,
                spin_limit=SPIN)
    wl = Workload(heap, WL_C2, ITEMS)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step(hp, w, m, ev=None):
        if ev:
            ev[0].record(stream)
        hp.reset(stream)
        w.begin(SEED, stream)
        if ev:
            ev[1].record(stream)
        w.rounds(ROUNDS, m, stream=stream)
        if ev:
            ev[2].record(stream)
        w.drain(m, stream=stream)
        if ev:
            ev[3].record(stream)

    def timed(hp, w, m, steps, warmup, sampler=None):
        for _ in range(warmup):
            step(hp, w, m)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
        flags = torch.zeros(steps, dtype=torch.int32).pin_memory()
        if sampler:
            sampler.start()
        for k in range(steps):
            flush.zero_()  # > L2, outside the timed events
            step(hp, w, m, evs[k])
            hp.error_flags_async(flags.data_ptr() + 4 * k, stream)  # after the step's events
        torch.cuda.synchronize()
        timed.step_flags = [int(f) & 0xffffffff for f in flags.tolist()]
        clocks = sampler.stop() if sampler else None
        if world > 1:
            torch.distributed.barrier()
        step_ms = [e[0].elapsed_time(e[3]) for e in evs]
        rounds_ms = [e[1].elapsed_time(e[2]) for e in evs]
        return step_ms, rounds_ms, clocks

    sampler = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0])
                           if os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0].isdigit()
                           else local)
    step_ms, rounds_ms, clocks = timed(heap, wl, mode, args.steps, args.warmup,
                                       None if args.only_timed else sampler)
    step_flags = list(timed.step_flags)
    st = wl.stats(stream)
    if args.only_timed:
        if rank == 0:
            print(json.dumps({"items": ITEMS, "rounds": ROUNDS, "sblocks": SBLOCKS, "mode": args.mode,
                              "step_ms": [round(x, 3) for x in step_ms],
                              "rounds_ms": [round(x, 3) for x in rounds_ms],
                              "ops_per_step": st["mallocs"] + st["frees"], "nulls": st["nulls"],
                              "bad_tags": st["bad_tags"], "step_error_flags": step_flags,
                              "rounds_launch_bytes_per_step": None}))
        wl.close()
        heap.close()
        return 0
    ops_step = st["mallocs"] + st["frees"]
    total_ms = max_over_ranks(sum(step_ms), world)
    value = job_rate(world, ops_step, args.steps, total_ms)

    # end to end through the host-buffer C ABI call, on every rank (pinned seeds in,
    # per-item hashes + counters out)
    g = np.arange(ITEMS, dtype=np.uint64)
    seeds_np = np.uint64(SEED) ^ (g * np.uint64(0x9E3779B97F4A7C15))
    seeds = torch.from_numpy(seeds_np.view(np.int64)).pin_memory()
    hashes = torch.empty(ITEMS, dtype=torch.int64).pin_memory()
    wl.run_host(seeds.data_ptr(), ROUNDS, mode, hashes.data_ptr(), stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        st_e = wl.run_host(seeds.data_ptr(), ROUNDS, mode, hashes.data_ptr(), stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world) / args.steps
    e2e = {"value": round(job_rate(world, st_e["mallocs"] + st_e["frees"], 1, e2e_ms), 3),
           "unit": UNIT, "h2d_bytes_per_step": ITEMS * 8,
           "d2h_bytes_per_step": ITEMS * 8 + 56,
           "ms_per_step": round(e2e_ms, 3),
           "call": "kma_wl_run_host (host seeds in, host hashes + counters out)"}

    out = None
    if rank == 0:
        # bytes of the rounds launch (deterministic when no malloc returns NULL)
        heap.reset(stream)
        wl.begin(SEED, stream)
        wl.rounds(ROUNDS, mode, stream=stream)
        st_r = wl.stats(stream)
        # one checked step: live-block invariants, then drain to canonical empty
        nlive, off, size = wl.live(stream)
        sel = np.arange(off.shape[0])[:, None] < nlive[None, :]
        res = ins.check_live_blocks(heap.snapshot(stream=stream), off[sel], size[sel],
                                    heap.bitmaps(stream))
        wl.drain(mode, stream=stream)
        st_d = wl.stats(stream)
        empty = ins.check_canonical_empty(heap.snapshot(stream=stream), heap.bitmaps(stream))
        faults = ins.violations(res) + len(empty) + int(st_d["bad_tags"]) + int(st["bad_tags"])
        flags = heap.error_flags(clear=True, stream=stream)

        # one untimed step with per-phase cycle counters (a separate kernel
        # instantiation): where the rounds kernel spends its warps' time
        heap.reset(stream)
        wl.begin(SEED, stream)
        wl.rounds(ROUNDS, mode | 2, stream=stream)
        cyc = wl.phase_cycles(stream)
        tally = wl.tally(stream)
        tot = sum(cyc) or 1
        phase_share = {k: round(v / tot, 4) for k, v in zip(("malloc", "fill", "verify", "free"), cyc)}
        rounds_bytes = st_r["fill_bytes"] + st_r["verify_bytes"]
        rounds_ops = st_r["mallocs"] + st_r["frees"]
        mean_rounds_s = statistics.mean(rounds_ms) / 1e3
        pk = peaks()
        achieved = rounds_bytes / mean_rounds_s / 1e9
        traffic = None
        if os.path.exists(PROFILE_TRAFFIC):
            try:
                traffic = json.load(open(PROFILE_TRAFFIC)).get("traffic_bytes_per_launch")
            except Exception:  # noqa: BLE001
                traffic = None
        # measured L2 atomic peak (distinct 128-byte lines, returning atomicAdd)
        n_at = 148 * 2048
        at_ms = bench_atomics(True, n_at, 64, 32, stream=stream)
        p_atom = n_at * 64 / (at_ms / 1e3)
        at_same_ms = bench_atomics(False, 148 * 256, 16, 32, stream=stream)
        p_same = 148 * 256 * 16 / (at_same_ms / 1e3)
        op_rate = rounds_ops / mean_rounds_s

        # plain per-thread kernel on the same GPU (the >=5x denominator):
        # the reference's algorithm and structures (one class table,
        # tagged-CAS MS-queue free list), and the same per-thread calls on
        # the default (sharded, ticket-ring) heap
        plain = plain_default = None
        if not args.no_plain and mode != MODE_PLAIN:
            with Heap(SBLOCKS, SB_LOG2, stream=stream, compat=True) as hc, \
                    Workload(hc, WL_C2, ITEMS) as wc:
                p_ms, _, _ = timed(hc, wc, MODE_PLAIN, 2, 1)
                st_p = wc.stats(stream)
                plain = (st_p["mallocs"] + st_p["frees"]) / (statistics.mean(p_ms) / 1e3) / 1e6
            p_ms, _, _ = timed(heap, wl, MODE_PLAIN, 2, 1)
            st_p = wl.stats(stream)
            plain_default = (st_p["mallocs"] + st_p["frees"]) / (statistics.mean(p_ms) / 1e3) / 1e6


        cpu = None if args.no_cpu_baseline else measure_cpu_baseline()

        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "mode": args.mode, "items": ITEMS, "rounds": ROUNDS,
                       "heap_bytes": SBLOCKS << SB_LOG2, "sb_size": 1 << SB_LOG2,
                       "ops_per_step": ops_step, "nulls": int(st["nulls"]),
                       "step_ms_min": round(min(step_ms), 3), "step_ms_max": round(max(step_ms), 3),
                       "step_error_flags": sorted({f for f in step_flags if f}),
                       "spin_limit": SPIN or (1 << 22),
                       "invariant_faults": faults, "heap_error_flags": flags,
                       "l2": "inputs larger than L2 (1 GiB heap) and a 256 MiB write between "
                             "steps, outside the timed events",
                       "parallelism": f"replicas x{world}",
                       "plain_mops": round(plain, 3) if plain else None,
                       "plain_default_heap_mops": round(plain_default, 3) if plain_default else None,
                       "class_shards": heap.cls_shards,
                       "rounds_phase_share": phase_share,
                       "malloc_tally": tally,
                       "warp_over_plain": round(value / world / plain, 2) if plain else None,
                       "warp_over_plain_default_heap":
                           round(value / world / plain_default, 2) if plain_default else None},
            "roofline": {"bound": "hbm", "kernel": "k_wl_rounds<warp>",
                         "achieved": round(achieved, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / pk["hbm_gbs"], 4), "traffic": traffic,
                         "peak_src": pk["src"],
                         "algorithmic_bytes_per_launch": rounds_bytes,
                         "launch_ms": round(1e3 * mean_rounds_s, 3)},
            "l2_atomic": {"achieved": round(op_rate / 1e9, 3), "peak": round(p_atom / 1e9, 3),
                          "unit": "G atomics/s", "frac": round(op_rate / p_atom, 4),
                          "same_address_peak": round(p_same / 1e9, 3),
                          "note": "algorithmic 2 L2 atomics per malloc+free pair = 1 per op; "
                                  "peak = returning atomicAdd on distinct 128-B lines, all SMs"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 4 * args.steps, "clocks": clocks,
        }
        if not args.no_forms:
            out["forms"] = measure_forms()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    wl.close()
    heap.close()
    if out is not None:
        print(json.dumps(out))
    return 0


def main(argv=None) -> int:
    global ITEMS, ROUNDS, SBLOCKS, SB_LOG2
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["warp", "plain"], default="warp")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-kernel comparison")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--items", type=int, default=ITEMS, help="work-items (a smaller case for ncu)")
    ap.add_argument("--rounds", type=int, default=ROUNDS)
    ap.add_argument("--sblocks", type=int, default=SBLOCKS, help="superblocks in the heap")
    ap.add_argument("--sb-log2", type=int, default=SB_LOG2, help="superblock size (experiments)")
    ap.add_argument("--shards", type=int, default=0, help="most class-table shards per class")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the structure, batched and served measurements")
    ap.add_argument("--only-timed", action="store_true",
                    help="run the timed steps only and print a short line (profiling)")
    args = ap.parse_args(argv)
    ITEMS, ROUNDS, SBLOCKS, SB_LOG2 = args.items, args.rounds, args.sblocks, args.sb_log2
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
