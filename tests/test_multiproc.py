"""Frame-parallel sharding of bench.py across ranks (world size 2, gloo on CPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = bench.frame_seeds(rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        timing = bench.max_over_ranks([10.0 + rank, 5.0 - rank], world)
        out[rank] = (gathered, timing)
    finally:
        dist.destroy_process_group()


def test_frame_sharding_two_ranks():
    world, port = 2, _free_port()
    manager = mp.Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    gathered, timing = out[0]
    flat = [s for seeds in gathered for s in seeds]
    assert len(flat) == len(set(flat)) == 4          # every rank owns distinct frames
    assert out[1][0] == gathered                      # every rank sees the same assignment
    assert timing == [11.0, 5.0] and out[1][1] == timing  # max over ranks on both ranks


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks([1.5, 2.5], 1) == [1.5, 2.5]
    assert bench.frame_seeds(0, 1) == [7000, 7001]
