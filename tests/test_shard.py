"""Multi-GPU batch splitting and the bench's own rank launch, on CPU.

* ``raymotion_b200.shard.partition`` gives every image of a batch to exactly
  one rank, balanced by estimated cost.
* Two gloo ranks on 127.0.0.1 each take their subset of the batched workload's
  64 images (as bench.py's batch measurement does), see together every image
  exactly once, and aggregate a whole-job value as the sum of their samples
  over the slowest rank's time.
* ``bench.py --gpus 2`` started without a launcher starts its two ranks itself
  (torch.distributed.run); a WORLD_SIZE that disagrees with --gpus is an error.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

from raymotion_b200.scenes import batch_workload
from raymotion_b200.shard import image_cost, partition, rank_items

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n_ranks", [1, 2, 3, 8])
def test_partition_covers_every_image_once_and_balances(n_ranks):
    specs = batch_workload(seed=3, n_scenes=64)
    costs = [image_cost(**s) for s in specs]
    parts = partition(costs, n_ranks)
    assert len(parts) == n_ranks
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(specs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    # greedy LPT: no rank exceeds the mean load by more than the largest single image
    assert max(loads) <= sum(costs) / n_ranks + max(costs) + 1e-6
    assert partition(costs, n_ranks) == parts  # deterministic


def test_partition_edge_cases():
    assert partition([], 4) == [[], [], [], []]
    assert partition([5.0], 3) == [[0], [], []]
    assert partition([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition([1.0], 0)


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        specs = batch_workload(seed=3, n_scenes=64)
        mine = rank_items(specs, rank, world)
        everyone = [None] * world
        dist.all_gather_object(everyone, mine)
        # stand-ins for a rank's measurement: its path samples and a time proportional to its cost
        samples = float(sum(specs[i]["width"] * specs[i]["height"] * specs[i]["spp"] for i in mine))
        secs = sum(image_cost(**specs[i]) for i in mine) * 1e-12
        bench.barrier(world)
        secs_max, = bench.allreduce([secs], "max", world)
        samples_sum, = bench.allreduce([samples], "sum", world)
        out.put((rank, everyone, secs, secs_max, samples_sum))
    finally:
        dist.destroy_process_group()


def test_two_ranks_render_disjoint_subsets_that_cover_the_batch():
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
    specs = batch_workload(seed=3, n_scenes=64)
    total = float(sum(s["width"] * s["height"] * s["spp"] for s in specs))
    (_, ev0, s0, m0, n0), (_, ev1, s1, m1, n1) = got
    assert ev0 == ev1
    a, b = ev0
    assert not set(a) & set(b) and sorted(a + b) == list(range(64))
    assert m0 == m1 == max(s0, s1)
    assert n0 == n1 == total
    # balanced: the slowest rank carries close to half the work
    assert max(s0, s1) / (s0 + s1) < 0.55


def test_bench_rejects_a_rank_count_that_disagrees_with_gpus():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--impl", "reference"],
                       capture_output=True, text=True, timeout=120, env=env, cwd=ROOT)
    assert r.returncode == 2
    assert "WORLD_SIZE=1" in r.stderr


def test_bench_launch_command():
    import bench
    cmd = bench.rank_launch_command(["--gpus", "4", "--steps", "2"], 4, 29511)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--master-addr=127.0.0.1" in cmd and "--master-port=29511" in cmd
    assert cmd[-4:] == ["--gpus", "4", "--steps", "2"]


def test_bench_starts_its_own_ranks():
    """The reference arm on the Cornell box with two ranks: rank 0 alone
    measures and prints one JSON line; the launcher returns its status."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_PORT")}
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--impl", "reference", "--workload",
                        "cornell", "--steps", "1", "--warmup", "0", "--ref-step-seconds", "0.3"],
                       capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2 and lines[0]["value"] > 0
