"""Seeded malloc/free op streams for serial-replay parity tests.

An op stream is an (n, 2) int64 array of (kind, arg): kind 0 = malloc(arg
bytes), kind 1 = free(the block returned by op `arg`; -1 = free(NULL)).
Streams mix the sizes the reference's size classes care about (tiny, class
boundaries, C1 sizes, the largest request, oversize) with frees of random
live blocks, sized to run the heap into exhaustion so that NULL returns,
refills, detaches and superblock recycling are all exercised.

The reference spins forever on a second live block of a class whose
superblock holds one slot (kma.cl:203-204), so a stream never holds two
such blocks at once.
"""
from __future__ import annotations

import numpy as np


def class_sizes(sb_size_log2: int) -> list[int]:
    """Block sizes per class (kma.cl:55-90), restated for stream generation."""
    sb = 1 << sb_size_log2
    out = []
    for b in range(sb_size_log2 - 1):
        blk = b + 2
        if blk <= (sb_size_log2 >> 1):
            out.append(1 << blk)
            continue
        items = sb // (1 << blk)
        ab = (items >> 3) + (1 if items & 7 else 0)
        ab += (4 - (ab & 3)) if ab & 3 else 0
        out.append(((sb - (12 + ab)) // items) & ~3)
    return out


def make_stream(seed: int, n_ops: int, sb_size_log2: int = 12, p_free: float = 0.42,
                p_null_free: float = 0.01) -> np.ndarray:
    rng = np.random.default_rng(seed)
    sizes = class_sizes(sb_size_log2)
    max_req = (1 << sb_size_log2) - 16
    one_slot_lo = sizes[-2] + 1  # sizes in (sizes[-2], sizes[-1]] use the 1-slot class
    live: list[int] = []
    one_slot_live: set[int] = set()
    ops = np.zeros((n_ops, 2), np.int64)
    for i in range(n_ops):
        r = rng.random()
        if live and r < p_free:
            j = int(rng.integers(len(live)))
            live[j], live[-1] = live[-1], live[j]
            k = live.pop()
            one_slot_live.discard(k)
            ops[i] = (1, k)
            continue
        if r < p_free + p_null_free:
            ops[i] = (1, -1)
            continue
        u = rng.random()
        if u < 0.45:
            n = int(rng.choice([8, 16, 32, 64, 128, 256]))
        elif u < 0.60:
            n = int(rng.integers(0, 17))
        elif u < 0.75:
            c = int(rng.integers(len(sizes)))
            n = sizes[c] + int(rng.integers(-1, 2))
        elif u < 0.97:
            n = int(rng.integers(1, max_req + 1))
        else:
            n = max_req + int(rng.integers(1, 64))
        n = max(n, 0)
        if one_slot_lo <= n <= max_req and one_slot_live:
            n = int(rng.integers(1, 65))
        ops[i] = (0, n)
        if n <= max_req:
            live.append(i)
            if n >= one_slot_lo:
                one_slot_live.add(i)
    return ops


def drain_stream(ops: np.ndarray) -> np.ndarray:
    """The stream followed by a free of every block still live at its end."""
    ops = np.asarray(ops, np.int64)
    freed = set(int(a) for k, a in ops if k == 1 and a >= 0)
    tail = [(1, i) for i, (k, _) in enumerate(ops) if k == 0 and i not in freed]
    if not tail:
        return ops.copy()
    return np.concatenate([ops, np.asarray(tail, np.int64)])
