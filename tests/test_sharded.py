"""Z-slab sharding of one frame (cuda_ultrasound_toolkit_b200/sharded.py) without a GPU: the slab
bounds, and the all-gather of slabs over world-size-2 and -3 gloo process groups on CPU tensors that
stand in for each rank's beamformed slab."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from cuda_ultrasound_toolkit_b200.sharded import gather_slabs, slab_bounds


@pytest.mark.parametrize("Z,depth,world", [(256, 16, 2), (256, 16, 3), (250, 16, 4), (40, 32, 3), (17, 16, 2),
                                           (128, 16, 8), (16, 16, 2)])
def test_slab_bounds_cover_the_volume_in_whole_tiles(Z, depth, world):
    b = slab_bounds(Z, depth, world)
    assert len(b) == world
    assert b[0][0] == 0 and b[-1][1] == Z
    for (z0, z1), (n0, _) in zip(b, b[1:]):
        assert z1 == n0                                   # contiguous, disjoint
    for z0, z1 in b:
        assert z0 <= z1 and z0 % depth == 0 and (z1 % depth == 0 or z1 == Z)
    sizes = [z1 - z0 for z0, z1 in b]
    tiles = [-(-s // depth) for s in sizes]
    assert max(tiles) - min(tiles) <= 1                   # as even as the tile count allows


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _volume(Z, Y, X):
    z = torch.arange(Z, dtype=torch.float32)[:, None, None]
    y = torch.arange(Y, dtype=torch.float32)[None, :, None]
    x = torch.arange(X, dtype=torch.float32)[None, None, :]
    return torch.complex(z * 1000 + y * 10 + x, -z)


def _worker(rank, world, port, Z, depth, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bounds = slab_bounds(Z, depth, world)
        z0, z1 = bounds[rank]
        slab = _volume(Z, 3, 5)[z0:z1].contiguous()       # this rank's slab of the volume
        out[rank] = gather_slabs(slab, bounds, Z)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,Z,depth", [(2, 48, 16), (3, 40, 16)])
def test_gathered_slabs_are_the_whole_volume_on_every_rank(world, Z, depth):
    port = _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_worker, args=(world, port, Z, depth, out), nprocs=world, start_method="spawn", join=True)
    want = _volume(Z, 3, 5)
    for r in range(world):
        assert torch.equal(out[r], want)
