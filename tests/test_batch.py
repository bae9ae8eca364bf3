"""The batched form (include/kma_batch.h): uneven jobs in one persistent
launch keep every tag intact, balance mallocs and frees, and leave the heap
canonically empty -- run directly, through a captured CUDA graph, and with
the per-warp cache; the autotuner reports every configuration."""
import numpy as np
import pytest

from kma_b200 import inspect as ins

SMALL_THREADS = [3000, 1000, 12345, 700, 40000, 2048, 5, 33]


def _check_empty(h):
    img = h.snapshot()
    assert ins.check_canonical_empty(img, h.bitmaps()) == []
    assert h.error_flags() == 0


def test_c4_jobs_are_log_uniform():
    from kma_b200.batch import c4_jobs
    t, s = c4_jobs()
    assert len(t) == 64 and t.min() >= 1000 and t.max() <= 1_000_000
    assert len(set(s.tolist())) == 64
    # log-uniform: the median thread count is near sqrt(1e3 * 1e6)
    assert 3e3 < np.median(t) < 3e5


@pytest.mark.gpu
@pytest.mark.parametrize("depth", [0, 4])
@pytest.mark.parametrize("sb_log2", [12, 14, 16])
def test_gpu_batch_run_invariants(sb_log2, depth):
    from kma_b200 import Heap
    from kma_b200.batch import Batch
    seeds = list(range(101, 101 + len(SMALL_THREADS)))
    # a 64 KiB-superblock heap needs more superblocks than 256 MiB holds: each
    # of its 15 classes keeps current superblocks pinned in many shards
    heap_bytes = (1 << 30) if sb_log2 == 16 else (256 << 20)
    with Heap(heap_bytes >> sb_log2, sb_log2) as h, Batch(h, SMALL_THREADS, seeds, rounds=12) as b:
        b.run(block_dim=256, cache_depth=depth)
        st = b.stats()
        items = sum(SMALL_THREADS)
        assert b.items == items
        assert st["bad_tags"] == 0
        assert st["mallocs"] == items * 12
        assert st["frees"] == st["mallocs"] - st["nulls"]
        if sb_log2 > 12:
            assert st["nulls"] == 0 and st["refused"] == 0
        else:
            # 4 KiB superblocks serve at most 4080 bytes: the jobs' 4088 and
            # 4096-byte draws are refused, and those are all the NULLs here
            assert st["refused"] == st["nulls"] > 0
        if depth:
            assert st["cache_hits"] > 0 and st["cache_puts"] >= st["cache_hits"]
        else:
            assert st["cache_hits"] == 0 and st["cache_puts"] == 0
        _check_empty(h)


@pytest.mark.gpu
@pytest.mark.parametrize("block_dim", [128, 512])
def test_gpu_batch_graph_replays(block_dim):
    import torch
    from kma_b200 import Heap
    from kma_b200.batch import Batch
    stream = torch.cuda.Stream()
    with Heap((256 << 20) >> 14, 14, stream=stream) as h, \
            Batch(h, SMALL_THREADS, list(range(7, 7 + len(SMALL_THREADS))), rounds=8) as b:
        b.capture(block_dim, 2, stream)
        for _ in range(3):  # every replay resets the heap and reseeds the jobs
            b.launch(stream)
            st = b.stats(stream)
            assert st["bad_tags"] == 0 and st["nulls"] == 0
            assert st["mallocs"] == sum(SMALL_THREADS) * 8 and st["frees"] == st["mallocs"]
        torch.cuda.synchronize()
        _check_empty(h)


@pytest.mark.gpu
def test_gpu_batch_autotune_reports_every_config():
    from kma_b200.batch import autotune
    entries, best = autotune(SMALL_THREADS, list(range(len(SMALL_THREADS))), rounds=6,
                             heap_bytes=128 << 20, sb_log2s=(12, 14), block_dims=(128, 256),
                             depths=(0, 2), warmup=1, reps=1)
    assert len(entries) == 8 and best is not None and 0 <= best < 8
    assert all(e["bad_tags"] == 0 and e["ms"] > 0 for e in entries)
    assert {(e["sb_size"], e["block_dim"], e["cache_depth"]) for e in entries} == \
        {(s, b, d) for s in (4096, 16384) for b in (128, 256) for d in (0, 2)}
    # a geometry that refuses sizes the jobs draw never wins, however fast
    assert all(e["serves_all"] == (e["sb_size"] > 4096) for e in entries)
    assert entries[best]["serves_all"] and entries[best]["refused"] == 0
    rate = [(e["mallocs"] - e["nulls"] + e["frees"]) / e["ms"] if e["serves_all"] else 0 for e in entries]
    assert rate[best] == max(rate)


@pytest.mark.gpu
@pytest.mark.parametrize("sb_log2", [12, 14])
def test_gpu_batch_plain_calls_invariants(sb_log2):
    """The same jobs with every thread calling kma_malloc / kma_free itself
    (the reference's per-work-item calls): tags intact, every block freed,
    the heap canonically empty."""
    from kma_b200 import MODE_PLAIN, Heap
    from kma_b200.batch import Batch
    seeds = list(range(201, 201 + len(SMALL_THREADS)))
    with Heap((256 << 20) >> sb_log2, sb_log2) as h, \
            Batch(h, SMALL_THREADS, seeds, rounds=10, mode=MODE_PLAIN) as b:
        b.run(block_dim=256, cache_depth=0)
        st = b.stats()
        assert st["bad_tags"] == 0 and st["mallocs"] == sum(SMALL_THREADS) * 10
        assert st["frees"] == st["mallocs"] - st["nulls"]
        assert st["nulls"] == st["refused"]  # only the sizes 4 KiB superblocks cannot serve
        _check_empty(h)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "warp"])
def test_gpu_batch_on_pma(mode):
    """The batch kernel compiled for the bump heap: every tag intact, and
    the heap head is exactly the bytes handed out (frees do nothing)."""
    from kma_b200.batch import Batch
    from kma_b200.structs import Pma
    seeds = list(range(301, 301 + len(SMALL_THREADS)))
    with Pma(1 << 30) as p, Batch(p, SMALL_THREADS, seeds, rounds=10, mode=mode) as b:
        b.run(block_dim=256, cache_depth=0)
        st = b.stats()
        assert st["bad_tags"] == 0 and st["nulls"] == 0 and st["refused"] == 0
        assert st["mallocs"] == sum(SMALL_THREADS) * 10 and st["frees"] == st["mallocs"]
        assert p.head() == st["fill_bytes"]
        with pytest.raises(Exception):
            b.run(block_dim=256, cache_depth=2)  # the warp cache needs KMA size classes
