"""The multi-GPU path is replicas (each rank runs the whole step on its own
GPU; no data-path collective): the timing's only collective, the maximum
over ranks, and the whole-job value, checked with two gloo ranks on CPU."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, times, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(times[rank], dist, "cpu")
        value = bench.replicas_value(world, 1e12, 4, ms)
        out.put((rank, ms, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_the_slowest_rank_times_the_job(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    times = [40.0 + 7.5 * r for r in range(world)]
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, world, port, times, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(out.get(timeout=10) for _ in range(world))
    slowest = max(times)
    for rank, ms, value in got:
        assert ms == slowest
        # world ranks x 4 steps x 1 TFLOP in the slowest rank's time.
        assert value == pytest.approx(world * 4 * 1e12 / (slowest / 1e3) / 1e12)


def test_one_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.replicas_value(1, 2e12, 10, 1000.0) == pytest.approx(20.0)
