"""Seeded op streams for the structure replays (shared by the fixture
generator and the tests).  Each stream is an (n, 2) int64 array of
(kind, arg) rows in the encoding of include/kma_structs.h, and never asks
for something the reference cannot do (enqueue an item that is already
queued, get past the end of a list, remove from the reference tree)."""
from __future__ import annotations

import numpy as np


def clqueue_stream(seed: int, n_items: int, n_ops: int) -> np.ndarray:
    """Enqueue free items / dequeue, with runs that empty and refill the
    queue (the head == tail transitions)."""
    rng = np.random.default_rng(seed)
    queued: list[int] = []
    free = list(range(n_items))
    ops = []
    for i in range(n_ops):
        phase = (i // 50) % 3  # fill, drain, mixed
        p_enq = (0.8, 0.2, 0.5)[phase]
        if free and (rng.random() < p_enq or not queued):
            k = int(rng.integers(len(free)))
            it = free.pop(k)
            queued.append(it)
            ops.append((0, it))
        else:
            ops.append((1, 0))
            if queued:
                free.append(queued.pop(0))
    return np.array(ops, np.int64)


def iqueue_stream(seed: int, n_items: int, n_ops: int) -> np.ndarray:
    """As clqueue_stream, for the indexed queue's semantics: item 0 starts
    as the dummy, dequeue hands out the old dummy and needs one item behind
    it, so the queue always holds at least one item."""
    rng = np.random.default_rng(seed)
    queued = [0]
    free = list(range(1, n_items))
    ops = []
    for i in range(n_ops):
        phase = (i // 40) % 3
        p_enq = (0.8, 0.2, 0.5)[phase]
        if free and (rng.random() < p_enq or len(queued) < 2):
            k = int(rng.integers(len(free)))
            it = free.pop(k)
            queued.append(it)
            ops.append((0, it))
        else:
            ops.append((1, 0))
            if len(queued) >= 2:
                free.append(queued.pop(0))
    return np.array(ops, np.int64)


def tree_stream(seed: int, n_ops: int, key_space: int, remove: bool) -> np.ndarray:
    """Adds and gets (and removes when `remove`) over a small key space, so
    keys repeat; kind 0 add, 1 get, 2 remove."""
    rng = np.random.default_rng(seed)
    kinds = rng.choice(3 if remove else 2, size=n_ops, p=(0.5, 0.3, 0.2) if remove else (0.6, 0.4))
    keys = rng.integers(0, key_space, size=n_ops)
    return np.stack([kinds, keys], axis=1).astype(np.int64)


def arraylist_stream(seed: int, n_ops: int, max_objs: int, gets: bool = True) -> np.ndarray:
    """grow(objs) / get(i < count) / clear; kind 0 grow, 1 get, 2 clear.
    With gets, the case's heap must hold every grow (the reference's get
    past the end returns an uninitialised value); without, grows may run
    the heap out (NULL pages)."""
    rng = np.random.default_rng(seed)
    count = 0
    ops = []
    for _ in range(n_ops):
        r = rng.random()
        if r < 0.45 or not gets:
            objs = int(rng.integers(1, max_objs + 1))
            ops.append((0, objs))
            count += objs
        elif r < 0.97 and count:
            ops.append((1, int(rng.integers(count))))
        else:
            ops.append((2, 0))
            count = 0
    return np.array(ops, np.int64)


def pma_stream(seed: int, n_ops: int, nbytes: int) -> np.ndarray:
    """Mallocs of mixed sizes (some larger than what is left), frees of
    earlier results; runs past the limit so NULLs and the header slack show."""
    rng = np.random.default_rng(seed)
    ops = []
    mean = max(8, nbytes // max(1, n_ops // 2))
    for i in range(n_ops):
        if i and rng.random() < 0.2:
            ops.append((1, int(rng.integers(i))))
        else:
            r = rng.random()
            size = int(rng.integers(1, 2 * mean)) if r < 0.9 else int(rng.integers(nbytes // 4, nbytes))
            ops.append((0, size))
    return np.array(ops, np.int64)


def pma_edge_stream(nbytes: int) -> np.ndarray:
    """The limit exactly: fill to nbytes, then the 24-byte slack the
    reference's check allows, then one more byte (refused)."""
    return np.array([(0, nbytes), (0, 24), (0, 1), (0, 0)], np.int64)
