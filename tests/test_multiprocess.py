"""The multi-GPU plumbing of bench.py on CPU: gloo ranks, max-over-ranks timing, the LPT partition of one
global batch over the ranks and the one-process-per-rank relaunch."""

import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, per_rank, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        vals = bench.max_over_ranks([1.0 + rank, 10.0 - rank])
        total, shards, load = bench.shard_plan(0, per_rank, world)
        mine = shards[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, [int(i) for i in mine])
        dist.barrier()
        out[rank] = (vals, total, gathered, load.tolist())
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_ranks_take_the_max_and_partition_one_batch():
    """Two gloo ranks: the timing max is the slowest rank's, and the ranks' shards partition the global batch
    (every instance exactly once) with LPT's balance bound: the heaviest shard exceeds the lightest by at most
    the cost of one instance (vertices x colors)."""
    import bench

    world, per_rank = 2, 24
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, per_rank, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert res[0][0] == [2.0, 10.0] and res[1][0] == [2.0, 10.0]
    total = res[0][1]
    assert total == world * per_rank
    shards = res[0][2]
    assert shards == res[1][2]  # both ranks hold the same plan
    allidx = sorted(i for s in shards for i in s)
    assert allidx == list(range(total))
    assert all(s == sorted(s) for s in shards)
    sides = bench.instance_params(0, total)[0]
    tpl = bench.templates(sides)
    cost = np.array([float(n) ** 2 * len(tpl[int(n)]._color_groups) for n in sides])
    load = np.array([cost[s].sum() for s in shards])
    assert np.allclose(load, res[0][3])
    assert load.max() - load.min() <= cost.max()


def test_lpt_partition_properties():
    """LPT on random costs: a partition, shards in increasing index order, and the greedy balance bound."""
    import bench

    rng = np.random.default_rng(3)
    for parts in (1, 2, 3, 8):
        costs = rng.integers(16, 129, size=200).astype(np.float64) ** 2
        shards, load = bench.lpt_partition(costs, parts)
        assert sorted(np.concatenate(shards).tolist()) == list(range(200))
        assert all(np.all(np.diff(s) > 0) for s in shards)
        assert np.allclose([costs[s].sum() for s in shards], load)
        assert load.max() - load.min() <= costs.max()
    one, _ = bench.lpt_partition(np.ones(5), 1)
    assert one[0].tolist() == [0, 1, 2, 3, 4]


def test_single_process_max_is_identity():
    import bench

    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert torch.distributed.is_available()


@pytest.mark.timeout(600)
def test_bench_relaunches_one_process_per_rank():
    """`bench.py --gpus 2` without WORLD_SIZE relaunches itself under torchrun; the reference arm (CPU) then
    runs on rank 0 alone and reports both ranks."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--instances", "4", "--cpu-seconds", "0.5"]  # fmt: skip
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=540)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["impl"] == "reference" and line["value"] > 0
