"""The N > 1 host logic of bench.py on CPU: two gloo ranks (one process each)
take the maximum of their timings and report the whole-job rate, and the
reference arm runs on rank 0 only.  The replicas share no data, so the timing
reduction is the only collective."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        # Rank r "took" 10 * (r + 1) ms for 1000 units.
        ms = bench.max_over_ranks(dist, 10.0 * (rank + 1))
        value = bench.whole_job_rate(world, 1000.0, ms / 1e3)
        queue.put((rank, ms, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    queue = ctx.SimpleQueue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    results = sorted(queue.get() for _ in range(world))
    for rank, ms, value in results:
        assert ms == 20.0, (rank, ms)                       # max over ranks
        assert value == pytest.approx(2 * 1000 / 0.020)     # all ranks' units / slowest time


def test_max_over_ranks_without_a_group_is_identity():
    assert bench.max_over_ranks(None, 3.5) == 3.5
    assert bench.whole_job_rate(1, 100.0, 2.0) == 50.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
