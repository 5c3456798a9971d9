"""Receive channels per staged delay-and-sum stage (cutb_options.das_rows_per_stage, 1..8).

With one READI sub-signal a stage of fewer rows keeps the order in which every voxel sums its
(transmit, channel) rows, so with one CTA per tile the volume must equal the default 8-row form bit
for bit. With sub-signals, or with the tiles' stages split over CTAs, the order of the sums
changes and the volume agrees within FP32 rounding."""
import numpy as np
import pytest
import torch

from cuda_ultrasound_toolkit_b200 import CutbError, Plan, SequenceId, synth

pytestmark = pytest.mark.gpu


def params(kind):
    w = synth.Workload(kind, 16, 24, 1024, 24, 16, 48, 0, cubic=True, cf=1.0, z_range=(5e-3, 15e-3), box_xy=2e-3)
    bp = synth.make_params(w)
    if kind == "forces":
        bp.das_shader_id = int(SequenceId.FORCES)
        bp.tx_orientation = bp.rx_orientation
    elif kind == "readi":
        bp.readi_group_count, bp.readi_group_id = 2, 1
    elif kind == "tpw":  # plane waves over y on a grid fine enough for the staged windows
        bp.das_shader_id = int(SequenceId.RCA_TPW)
        bp.output_min_coordinate[0], bp.output_max_coordinate[0] = -0.8e-3, 0.8e-3
        bp.output_min_coordinate[2], bp.output_max_coordinate[2] = 4e-3, 6e-3
        bp.fn_rx = 1.0
        for t, a in enumerate(np.linspace(-0.2, 0.2, 16)):
            bp.foci[3 * t + 2] = float(a)
    return bp


def random_iq(plan, seed):
    g = torch.Generator().manual_seed(seed)
    shape = plan.empty_iq().shape
    return torch.complex(torch.randn(shape, generator=g), torch.randn(shape, generator=g)).cuda()


def volume(bp, iq, **opts):
    plan = Plan(bp, **opts)
    v = plan.das(iq)
    plan.check()
    return v


@pytest.mark.parametrize("rows", [1, 3, 4, 5, 7])
@pytest.mark.parametrize("kind,tile", [("hercules", 1), ("hercules", 2), ("forces", 0), ("tpw", 2)])
def test_fewer_rows_per_stage_is_bit_identical(kind, tile, rows):
    bp = params(kind)
    iq = random_iq(Plan(bp), 11)
    ref = volume(bp, iq, das_tile=tile, das_schedule=1)
    got = volume(bp, iq, das_tile=tile, das_schedule=1, das_rows_per_stage=rows)
    assert torch.equal(got, ref)


@pytest.mark.parametrize("kind,schedule", [("readi", 1), ("forces", 0), ("tpw", 0)])
def test_fewer_rows_per_stage_with_reordered_sums(kind, schedule):
    bp = params(kind)
    iq = random_iq(Plan(bp), 12)
    ref = volume(bp, iq, das_schedule=schedule).cpu().numpy()
    got = volume(bp, iq, das_schedule=schedule, das_rows_per_stage=4).cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6


@pytest.mark.parametrize("rows", [-1, 9])
def test_rows_per_stage_out_of_range_is_rejected(rows):
    with pytest.raises(CutbError):
        Plan(params("hercules"), das_rows_per_stage=rows)
