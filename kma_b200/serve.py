"""The served form (include/kma_serve.h): a request loop over one
device-resident heap with continuous batching, FIFO admission by free slot
and heap occupancy, and per-request latency.  No counterpart in the
reference; every allocation goes through the device heap."""
from __future__ import annotations

from ctypes import byref, c_void_p

import numpy as np

from ._lib import KmaServeCfg, KmaServeReq, KmaServeResult, KmaServeSummary, check, lib
from .heap import Heap

STATUS = {0: "ok", 1: "nomem", 2: "mismatch", 3: "too_big"}


def c5_requests(seed: int, n: int, rate: float, nmin: int = 1000, nmax: int = 4_000_000):
    """Poisson arrivals at `rate` per second, N log-uniform in [nmin, nmax],
    one seed per request: (n_vertices, seeds, arrival_s)."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    nv = np.exp(rng.uniform(np.log(nmin), np.log(nmax), n)).astype(np.int64)
    seeds = rng.integers(0, 2**63, n)
    return nv, seeds, arrivals


class Server:
    def __init__(self, heap: Heap, slots: int = 8, max_vertices: int = 4_000_000, deg_max: int = 4096,
                 gamma: float = 2.1, occupancy_limit: float = 0.85, block_dim: int = 256, mode: int | None = None):
        """mode: MODE_WARP (default, warp-collaborative page mallocs and
        frees) or MODE_PLAIN (every vertex's thread calls malloc / free)."""
        self.heap = heap
        self.cfg = KmaServeCfg(slots, max_vertices, deg_max, block_dim, gamma, occupancy_limit)
        s = c_void_p()
        check(lib().kma_serve_create(heap.handle, byref(self.cfg), byref(s)), "kma_serve_create")
        self._s = s
        if mode is not None:
            check(lib().kma_serve_set_mode(s, mode), "kma_serve_set_mode")

    def close(self) -> None:
        s = getattr(self, "_s", None)
        if s is not None:
            self._s = None
            check(lib().kma_serve_destroy(s), "kma_serve_destroy")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def estimate(self, n_vertices: int) -> int:
        return int(lib().kma_serve_estimate(self._s, n_vertices))

    def run(self, n_vertices, seeds, arrivals=None, realtime: bool = False):
        """Serve the requests; returns (per-request dicts, summary dict)."""
        n = len(n_vertices)
        reqs = (KmaServeReq * n)()
        arr = np.zeros(n) if arrivals is None else np.asarray(arrivals, float)
        for i in range(n):
            reqs[i].n_vertices = int(n_vertices[i])
            reqs[i].seed = int(seeds[i]) & (2**64 - 1)
            reqs[i].arrival_s = float(arr[i])
        res = (KmaServeResult * n)()
        summ = KmaServeSummary()
        check(lib().kma_serve_run(self._s, reqs, n, int(realtime), res, byref(summ)), "kma_serve_run")
        out = []
        for i, r in enumerate(res):
            d = {k: getattr(r, k) for k, _ in KmaServeResult._fields_}
            d["status"] = STATUS.get(r.status, str(r.status))
            d["latency_s"] = r.done_s - float(arr[i])
            out.append(d)
        return out, {k: getattr(summ, k) for k, _ in KmaServeSummary._fields_}


# ---------------------------------------------------------------- model
_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix(state: np.ndarray):
    state += np.uint64(0x9E3779B97F4A7C15)
    z = state.copy()
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def degree_thresholds(deg_max: int, gamma: float) -> np.ndarray:
    """The degree law's cumulative thresholds of 2^32, as the server builds them."""
    g = float(np.float32(gamma))
    pd = np.power(np.arange(1, deg_max + 1, dtype=np.float64), -g)
    tot = np.cumsum(pd)[-1]
    run = np.cumsum(pd)
    t = run / tot * 4294967296.0
    out = np.minimum(t, 4294967295.0).astype(np.uint64).astype(np.uint32)
    out[-1] = 0xFFFFFFFF
    return out


def expected_result(seed: int, n: int, deg_max: int = 4096, gamma: float = 2.1):
    """(checksum, edges) of request (seed, n), computed on the host from the
    same draws the device uses -- independent of the heap."""
    with np.errstate(over="ignore"):
        cdf = degree_thresholds(deg_max, gamma)
        v = np.arange(n, dtype=np.uint64)
        rng = np.uint64(seed) ^ ((v + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15))
        u = (_splitmix(rng) >> np.uint64(32)).astype(np.uint32)
        deg = np.searchsorted(cdf, u, side="left").astype(np.int64) + 1
        h = ((v + np.uint64(1)) * np.uint64(0xD6E8FEB86659FD93)) ^ deg.astype(np.uint64)
        for k in range(int(deg.max())):
            m = deg > k
            nb = ((_splitmix(rng) >> np.uint64(32)) * np.uint64(n)) >> np.uint64(32)
            hk = (h ^ nb) * np.uint64(0x9E3779B97F4A7C15)
            hk = hk ^ (hk >> np.uint64(29))
            h = np.where(m, hk, h)
        return int(h.sum(dtype=np.uint64)), int(deg.sum())
