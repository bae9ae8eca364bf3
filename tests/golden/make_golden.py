"""Generate the golden fixtures under tests/golden/ from the reference.

Runs the UNMODIFIED reference sources (kma.cl, clIndexedQueue.cl) built by
oracle/Makefile into oracle/_ref/ (needs the reference tree, so this runs
where it is mounted; the fixtures it writes are committed and the tests only
read them):

    python tests/golden/make_golden.py

Writes
  tables.json          size/slot/class tables for 4, 16 and 64 KiB superblocks
  replay_<log2>_<seed>.npz   op stream, the reference's offsets and decoded end state
  workloads.json       C1/C2 serial-run counters and hashes
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle  # noqa: E402
from opstream import drain_stream, make_stream  # noqa: E402

REPLAYS = [  # (sb_size_log2, sblocks, seed, n_ops)
    (12, 48, 1, 3000),
    (12, 48, 2, 3000),
    (12, 6, 3, 400),
    (14, 20, 4, 2000),
    (16, 8, 5, 1500),
]

WORKLOADS = [  # (name, program, sb_log2, sblocks, items, rounds, seed, round_major)
    ("c1_item", 1, 12, 4096, 256, 16, 0xC1, 0),
    ("c1_round", 1, 12, 4096, 256, 16, 0xC1, 1),
    ("c2_round_small", 2, 14, 65536, 2048, 64, 0xC2, 1),
    ("c2_item_small", 2, 14, 65536, 1024, 64, 0xC2, 0),
]


def region_digest(region: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(region).tobytes()).hexdigest()


def tables() -> dict:
    out = {}
    for log2 in (12, 14, 16):
        sizes, slots, sbid = oracle.ref_tables(log2)
        trans = [[0, int(sbid[0])]]
        for n in range(1, len(sbid)):
            if sbid[n] != sbid[n - 1]:
                trans.append([n, int(sbid[n])])
        out[str(log2)] = {"size_by_sbid": sizes, "slots_by_size": slots, "sbid_transitions": trans}
    return out


def main() -> int:
    if not oracle.ref_available(12):
        oracle.build()
    if not oracle.ref_available(12):
        print("reference build unavailable (oracle/_ref missing)", file=sys.stderr)
        return 1
    with open(os.path.join(HERE, "tables.json"), "w") as f:
        json.dump(tables(), f, indent=1)
    for log2, sblocks, seed, n in REPLAYS:
        ops = drain_stream(make_stream(seed, n, log2))
        with oracle.Ref(sblocks, log2) as r:
            out = r.replay(ops)
            d = r.decode()
            reg = r.region()
        np.savez_compressed(os.path.join(HERE, f"replay_{log2}_{seed}.npz"), ops=ops, out=out,
                            cls=d["cls"], sb_size=d["sb_size"], sb_slots=d["sb_slots"],
                            sb_free=d["sb_free"], freelist=d["freelist"],
                            region_sha256=np.array(region_digest(reg)), sblocks=sblocks)
        print(f"replay log2={log2} seed={seed}: {len(ops)} ops, "
              f"{int(np.sum((ops[:, 0] == 0) & (out < 0)))} NULL")
    wl = {}
    for name, prog, log2, sblocks, items, rounds, seed, rm in WORKLOADS:
        with oracle.Ref(sblocks, log2) as r:
            st = r.run_workload(prog, items, rounds, seed, rm)
            d = r.decode()
        st.pop("seconds")
        wl[name] = {"program": prog, "sb_size_log2": log2, "sblocks": sblocks, "items": items,
                    "rounds": rounds, "seed": seed, "round_major": rm,
                    "stats": {k: int(v) for k, v in st.items()},
                    "freelist_sha256": hashlib.sha256(d["freelist"].tobytes()).hexdigest(),
                    "freelist_len": int(len(d["freelist"]))}
        print(name, wl[name]["stats"])
    with open(os.path.join(HERE, "workloads.json"), "w") as f:
        json.dump(wl, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
