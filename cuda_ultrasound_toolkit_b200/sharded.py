"""One large frame beamformed by several GPUs: z-slabs of the volume, one process per GPU.

Upstream beamforms on one GPU only (cuda_toolkit/src/rf_processing/rf_processor.cpp:47 hard-codes
device 0). Frames are independent, so the usual multi-GPU form is one frame per GPU (bench.py
--gpus N). A single frame too slow for one GPU splits by voxel depth instead, with one exchange
step on each side:
  1. the raw frame is broadcast from rank 0 (NCCL, into every GPU's HBM);
  2. every rank decodes and transforms the whole frame (about 0.4 ms of the ~84 ms step);
  3. every rank beamforms its own slab of z-planes (cutb_das_zslab: the same tiles the whole-frame
     launch would run, so the slabs side by side equal the single-GPU volume bit for bit);
  4. the slabs are all-gathered into the whole volume on every rank.
Slabs are whole tiles of the delay-and-sum (the tile depth from cutb_plan_das_tile_shape), dealt
as evenly as the tile count allows, and padded to one size for the collective.
"""
import torch

from .api import Plan


def slab_bounds(Z, tile_depth, world):
    """[(z0, z1)] per rank: contiguous slabs of whole tiles (the last one may end inside a tile at Z);
    a rank gets an empty slab (z0 == z1) when there are fewer tiles than ranks."""
    tiles = -(-Z // tile_depth)
    out = []
    for r in range(world):
        t0, t1 = tiles * r // world, tiles * (r + 1) // world
        out.append((min(t0 * tile_depth, Z), min(t1 * tile_depth, Z)))
    return out


def gather_slabs(slab, bounds, Z, group=None):
    """All-gather every rank's slab [(z1 - z0)][Y][X] into the whole volume [Z][Y][X] on every rank.
    Slabs are padded to the largest one so that one all_gather_into_tensor carries them."""
    import torch.distributed as dist
    depth = max(z1 - z0 for z0, z1 in bounds)
    y, x = slab.shape[1], slab.shape[2]
    padded = torch.zeros((depth, y, x), dtype=slab.dtype, device=slab.device)
    padded[:slab.shape[0]] = slab
    world = len(bounds)
    allv = torch.empty((world * depth, y, x), dtype=slab.dtype, device=slab.device)
    if slab.dtype.is_complex:  # collectives on the real view (gloo and NCCL both carry float32)
        dist.all_gather_into_tensor(torch.view_as_real(allv), torch.view_as_real(padded), group=group)
    else:
        dist.all_gather_into_tensor(allv, padded, group=group)
    vol = torch.empty((Z, y, x), dtype=slab.dtype, device=slab.device)
    for r, (z0, z1) in enumerate(bounds):
        vol[z0:z1] = allv[r * depth:r * depth + (z1 - z0)]
    return vol


class ShardedFrame:
    """A plan on this rank's GPU and its slab of the volume."""

    def __init__(self, bp, rank, world, **plan_options):
        self.plan = Plan(bp, **plan_options)
        self.rank, self.world = rank, world
        self.Z = int(bp.output_points[2])
        tile_depth = self.plan.tile_shape[2]
        self.bounds = slab_bounds(self.Z, tile_depth, world)
        self.dec = self.plan.empty_decoded()
        self.iq = self.plan.empty_iq()

    def slab(self, d_raw, stream=None):
        """Decode + Hilbert of the whole frame, delay-and-sum of this rank's slab."""
        z0, z1 = self.bounds[self.rank]
        self.plan.decode(d_raw, out=self.dec, stream=stream)
        self.plan.hilbert(self.dec, out=self.iq, stream=stream)
        if z1 == z0:
            z, y, x = self.plan.bp.volume_shape
            return torch.empty((0, y, x), dtype=torch.complex64, device="cuda")
        return self.plan.das_zslab(self.iq, z0, z1, stream=stream)

    def beamform(self, d_raw, group=None, src=0):
        """The whole volume on every rank: broadcast of rank src's raw frame, this rank's slab,
        all-gather of the slabs."""
        import torch.distributed as dist
        dist.broadcast(d_raw, src=src, group=group)
        return gather_slabs(self.slab(d_raw), self.bounds, self.Z, group)
