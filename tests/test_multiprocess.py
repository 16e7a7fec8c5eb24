"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks, max-over-ranks timing and per-rank batches."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        vals = bench.max_over_ranks([1.0 + rank, 10.0 - rank])
        sides, E, bend, pins = bench.instance_params(bench.rank_seed(0, rank), 8)
        dist.barrier()
        out[rank] = (vals, [int(x) for x in sides])
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_ranks_take_the_max_and_own_batches():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert res[0][0] == [2.0, 10.0] and res[1][0] == [2.0, 10.0]
    assert res[0][1] != res[1][1]  # each rank simulates its own batch


def test_single_process_max_is_identity():
    import bench

    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert torch.distributed.is_available()
