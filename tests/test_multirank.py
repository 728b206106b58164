"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the
independent solves are sharded over the ranks by bench.shard_instances, each
rank solves its shard (here with the CPU oracle on a small grid), the union
of the shards equals a single-rank run, the job's time is the slowest rank's
and its throughput counts the units of all ranks."""
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


SHARD_GRID = (18, 18, 16, 1.0 / 14.0, 2, 6)
N_INSTANCES = 7


def _instance_density(i):
    """Instance i of the sharded list: the smooth test field rotated by i zones
    and scaled, so that every instance has a different potential."""
    import numpy as np

    from tests.helpers import smooth_density

    numr, numz, numphi, dr, isym, _ = SHARD_GRID
    rho = smooth_density(numr, numz, numphi, dr, isym)
    return np.asfortranarray(np.roll(rho, i, axis=2) * (1.0 + 0.1 * i))


def _solve_instances(ids):
    from oracle import oracle as O

    o = O.Oracle(*SHARD_GRID)
    out = {i: o.potential_solver(_instance_density(i), 0) for i in ids}
    o.close()
    return out


def _shard_worker(rank, world, port, out):
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    mine = bench.shard_instances(N_INSTANCES, world, rank)
    solved = _solve_instances(mine)
    gathered = [None] * world
    dist.all_gather_object(gathered, {i: p.tobytes() for i, p in solved.items()})
    count = torch.tensor([len(solved)], dtype=torch.int64)
    dist.all_reduce(count)                      # units solved by the whole job
    ms_max = bench.max_over_ranks([30.0, 45.0][rank], world)
    out[rank] = (list(mine), gathered, int(count.item()), ms_max,
                 bench.job_rate(len(solved), world, ms_max))
    dist.barrier()
    dist.destroy_process_group()


def test_shards_cover_every_instance_once():
    import bench

    for n in (1, 2, 7, 96, 256):
        for world in (1, 2, 3, 8):
            parts = [list(bench.shard_instances(n, world, r)) for r in range(world)]
            flat = [i for p in parts for i in p]
            assert sorted(flat) == list(range(n)), (n, world)
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1


def test_two_ranks_solve_their_shards_and_the_union_equals_one_rank():
    import numpy as np

    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    shards = [out[r][0] for r in range(world)]
    assert shards == [[0, 1, 2, 3], [4, 5, 6]]
    union = {}
    for part in out[0][1]:
        for i, b in part.items():
            assert i not in union
            union[i] = np.frombuffer(b, dtype=np.float64)
    assert sorted(union) == list(range(N_INSTANCES))
    single = _solve_instances(range(N_INSTANCES))   # the same instances on one rank
    for i in range(N_INSTANCES):
        assert np.array_equal(union[i], np.frombuffer(single[i].tobytes(), dtype=np.float64)), i
    for r in range(world):
        _, gathered, count, ms_max, rate = out[r]
        assert count == N_INSTANCES
        assert ms_max == pytest.approx(45.0)
        assert rate == pytest.approx(world * len(shards[r]) / 0.045)


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
