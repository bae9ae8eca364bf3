"""The served form (include/kma_serve.h): requests build and verify their
graphs through the device heap while others run, each result equals the
host model's and is the same alone and in the mix, admission keeps the
reserved bytes under the occupancy limit, and the heap ends empty."""
import numpy as np
import pytest

from kma_b200 import inspect as ins
from kma_b200.serve import c5_requests, degree_thresholds, expected_result


def test_c5_requests_shapes():
    nv, seeds, arr = c5_requests(5, 200, rate=100.0)
    assert len(nv) == len(seeds) == len(arr) == 200
    assert nv.min() >= 1000 and nv.max() <= 4_000_000
    assert np.all(np.diff(arr) >= 0)
    assert 1.0 < arr[-1] < 3.5  # 200 arrivals at 100/s


def test_degree_law_is_a_power_law():
    cdf = degree_thresholds(4096, 2.1).astype(np.float64)
    p = np.diff(np.concatenate([[0.0], cdf])) / 2**32
    assert abs(p.sum() - 1) < 1e-6
    # P(d) ~ d^-2.1: the ratio of P(1) to P(2) is 2^2.1
    assert abs(p[0] / p[1] - 2 ** 2.1) < 1e-3


def test_model_is_deterministic():
    a = expected_result(123, 5000)
    b = expected_result(123, 5000)
    c = expected_result(124, 5000)
    assert a == b and a != c and a[1] >= 5000


def _empty(h):
    assert ins.check_canonical_empty(h.snapshot(), h.bitmaps()) == []
    assert h.error_flags() == 0


@pytest.mark.gpu
def test_gpu_serve_results_equal_model_and_overlap():
    from kma_b200 import Heap
    from kma_b200.serve import Server
    nv, seeds, _ = c5_requests(11, 12, rate=0, nmin=1000, nmax=100_000)
    with Heap(65536, 14) as h, Server(h, slots=4, max_vertices=200_000) as s:
        res, summ = s.run(nv, seeds)
        for r, n, sd in zip(res, nv, seeds):
            assert r["status"] == "ok", r
            assert (r["checksum"], r["edges"]) == expected_result(int(sd), int(n))
            assert r["mallocs"] == r["frees"] and r["nulls"] == 0
            assert r["done_s"] >= r["admit_s"] >= 0
        assert summ["max_running"] > 1  # requests were on the device together
        assert summ["ops"] == sum(r["mallocs"] + r["frees"] for r in res)
        _empty(h)


@pytest.mark.gpu
def test_gpu_serve_alone_equals_mix():
    from kma_b200 import Heap
    from kma_b200.serve import Server
    nv, seeds, _ = c5_requests(12, 10, rate=0, nmin=2000, nmax=150_000)
    with Heap(65536, 14) as h, Server(h, slots=6, max_vertices=200_000) as s:
        mix, summ = s.run(nv, seeds)
        assert summ["max_running"] > 1
        for i in (0, 4, 9):
            alone, _ = s.run(nv[i:i + 1], seeds[i:i + 1])
            assert alone[0]["status"] == mix[i]["status"] == "ok"
            assert alone[0]["checksum"] == mix[i]["checksum"]  # exact: tolerance 0
            assert alone[0]["edges"] == mix[i]["edges"]
        _empty(h)


@pytest.mark.gpu
def test_gpu_serve_realtime_poisson():
    from kma_b200 import Heap
    from kma_b200.serve import Server
    nv, seeds, arr = c5_requests(13, 40, rate=400.0, nmin=1000, nmax=60_000)
    with Heap(65536, 14) as h, Server(h, slots=8, max_vertices=100_000) as s:
        res, summ = s.run(nv, seeds, arr, realtime=True)
        for r, a in zip(res, arr):
            assert r["status"] == "ok"
            assert r["admit_s"] >= a - 1e-3 and r["done_s"] > r["admit_s"]
            assert r["latency_s"] > 0
        assert summ["wall_s"] > 0
        _empty(h)


@pytest.mark.gpu
def test_gpu_serve_admission_respects_occupancy():
    """A heap that fits only a few requests at once: reservations never pass
    the limit, too-large requests are refused, the rest all complete."""
    from kma_b200 import Heap
    from kma_b200.serve import Server
    with Heap(4096, 14) as h, Server(h, slots=8, max_vertices=400_000, occupancy_limit=0.85) as s:
        limit = 0.85 * 4096 * 16384
        # the estimate is linear in the vertex count: size requests so that
        # three fit at once and a fourth does not
        slope = (s.estimate(200_000) - s.estimate(0)) / 200_000
        n_ok = int((limit / 3 - s.estimate(0)) / slope) - 1
        assert 1000 < n_ok <= 400_000 and 3 * s.estimate(n_ok) <= limit < 4 * s.estimate(n_ok)
        nv = [n_ok] * 6 + [400_000]
        est_big = s.estimate(400_000)
        seeds = list(range(100, 107))
        res, summ = s.run(nv, seeds)
        for r in res[:6]:
            assert r["status"] == "ok"
            assert r["reserved_bytes"] == s.estimate(n_ok)
        assert res[6]["status"] == ("too_big" if est_big > limit else "ok")
        assert summ["max_running"] * s.estimate(n_ok) <= limit
        # the heap room, not the 8 slots, held requests back
        assert summ["max_running"] <= 3 and summ["admit_waits"] > 0
        assert summ["max_reserved"] <= 0.85 + 1e-9
        assert summ["max_reserved"] == pytest.approx(summ["max_running"] * s.estimate(n_ok) / (4096 * 16384))
        _empty(h)


@pytest.mark.gpu
def test_gpu_serve_plain_calls_equal_warp_calls():
    """The same requests with every vertex's thread calling kma_malloc /
    kma_free itself give the same results as the warp-collaborative calls
    (results do not depend on where the blocks landed), and empty the heap."""
    from kma_b200 import MODE_PLAIN, Heap
    from kma_b200.serve import Server
    nv, seeds, _ = c5_requests(13, 8, rate=0, nmin=1000, nmax=80_000)
    with Heap(65536, 14) as h:
        with Server(h, slots=4, max_vertices=100_000) as s:
            warp, _ = s.run(nv, seeds)
        with Server(h, slots=4, max_vertices=100_000, mode=MODE_PLAIN) as s:
            plain, _ = s.run(nv, seeds)
        for a, b in zip(warp, plain):
            assert a["status"] == b["status"] == "ok"
            assert (a["checksum"], a["edges"], a["mallocs"]) == (b["checksum"], b["edges"], b["mallocs"])
        _empty(h)
