"""Z-slabs of one frame on the GPU (cutb_das_zslab, sharded.ShardedFrame). One GPU stands in for
the ranks: each rank's slab is computed in turn, and the slabs side by side must equal the
whole-frame delay-and-sum bit for bit (the same tiles run, only their output planes move)."""
import numpy as np
import pytest
import torch

from cuda_ultrasound_toolkit_b200 import CutbError, Plan, SequenceId, synth
from cuda_ultrasound_toolkit_b200.sharded import ShardedFrame

pytestmark = pytest.mark.gpu


def frame(kind):
    if kind == "small":
        return synth.frame("small")
    w = synth.Workload(kind, 16, 32, 1024, 24, 12, 70, 8, cubic=True, cf=1.0, filter_taps=16,
                       z_range=(5e-3, 15e-3), box_xy=2e-3)
    raw, cmap, _, _ = synth.synth_frame(w, 5)
    bp = synth.make_params(w, channel_map=cmap)
    if kind == "forces":
        bp.das_shader_id = int(SequenceId.FORCES)
        bp.tx_orientation = bp.rx_orientation
    return raw, bp


@pytest.mark.parametrize("kind", ["small", "odd", "forces"])  # odd: 70 planes, a partial last tile
@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_slabs_equal_the_whole_frame(kind, world):
    raw, bp = frame(kind)
    d_raw = torch.from_numpy(raw).cuda()
    whole = Plan(bp, das_schedule=1)
    ref = whole.beamform(d_raw)
    whole.check()
    Z = int(bp.output_points[2])
    parts = []
    for r in range(world):
        sf = ShardedFrame(bp, r, world, das_schedule=1)
        parts.append(sf.slab(d_raw))
        sf.plan.check()
    vol = torch.cat(parts, dim=0)
    assert vol.shape[0] == Z
    assert torch.equal(vol, ref)


def test_zslab_rejects_misaligned_planes():
    raw, bp = frame("small")
    plan = Plan(bp)
    iq = plan.hilbert(plan.decode(torch.from_numpy(raw).cuda()))
    depth = plan.tile_shape[2]
    with pytest.raises(CutbError):
        plan.das_zslab(iq, 1, depth)
    with pytest.raises(CutbError):
        plan.das_zslab(iq, 0, depth + 1)
    with pytest.raises(CutbError):
        plan.das_zslab(iq, depth, depth)
    assert np.isfinite(plan.das_zslab(iq, 0, depth).abs().sum().item())
