"""The replicated bench path on CPU: with one process per GPU, the job's time
is its slowest rank's (a MAX all-reduce every rank joins) and its rate
counts every rank's operations; the reference arm runs on rank 0 alone.
Two gloo ranks on 127.0.0.1 stand in for the NCCL ranks of a GPU node."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(times[rank], world, device="cpu")
        out[rank] = (t, bench.job_rate(world, 1000, 10, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    world, times = 2, [12.5, 20.0]
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(rank_main, args=(world, free_port(), times, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    t, rate = res[0]
    assert t == max(times)
    # 2 ranks x 1000 ops x 10 steps in the slowest rank's 20 ms
    assert abs(rate - 2 * 1000 * 10 / 0.020 / 1e6) < 1e-9


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_rate(1, 500, 4, 2.0) == 1.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
