"""The bench's multi-rank aggregation on CPU: two gloo ranks (replicas).

bench.py --gpus N runs one frame stream per rank and reports the whole-job
value as (path samples summed over ranks) / (the slowest rank's time); the
ranks meet only in allreduce / barrier.  This runs those helpers with
world_size 2 over gloo on 127.0.0.1, each rank with a different time and
sample count, and checks the aggregate each rank sees.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        secs = [0.5, 0.8][rank]          # rank 1 is the slower replica
        samples = [1.0e9, 1.2e9][rank]
        bench.barrier(world)
        secs_max, = bench.allreduce([secs], "max", world)
        samples_sum, rays_sum = bench.allreduce([samples, 2 * samples], "sum", world)
        bench.barrier(world)
        out.put((rank, secs_max, samples_sum, rays_sum, samples_sum / secs_max))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_is_sum_over_slowest():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, secs_max, samples_sum, rays_sum, value in got:
        assert secs_max == pytest.approx(0.8)
        assert samples_sum == pytest.approx(2.2e9)
        assert rays_sum == pytest.approx(4.4e9)
        assert value == pytest.approx(2.2e9 / 0.8)


def test_single_rank_helpers_are_identity():
    import bench
    assert bench.allreduce([1.5, 2.0], "max", 1) == [1.5, 2.0]
    bench.barrier(1)
