"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): every rank
runs an independent solve sequence, the job's time is the slowest rank's and
its throughput counts the units of all ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    ms = [120.0, 80.0][rank]          # this rank's device time of the timed region
    bench.barrier(world)
    ms_max = bench.max_over_ranks(ms, world)
    out[rank] = (ms_max, bench.job_rate(100, world, ms_max))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_sum_the_work():
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        ms_max, rate = out[r]
        assert ms_max == pytest.approx(120.0)
        assert rate == pytest.approx(2 * 100 / 0.120)


def test_single_rank_rate():
    import bench

    assert bench.job_rate(1000, 1, 500.0) == pytest.approx(2000.0)
    assert bench.max_over_ranks(3.5, 1) == 3.5
