"""The bounded device-side waits of the staged delay-and-sum, made to run out on purpose.

The kernel's only device-side waits are the mbarrier waits for the bulk copies of a stage
(cuda_ultrasound_toolkit_b200/csrc/das.cu). The test hook cutb_debug_das_skip_stage keeps one
stage from ever being issued, so the wait for it gives up after a short limit: the CTA must then
stop, let the copies it had already issued land, leave, and report CUTB_ERR_TIMEOUT through
cutb_plan_check. A normal call on the same plan afterwards must succeed and give the same volume
as before. No GPU fault is involved: the missing stage is a flag nothing sets, and every wait is
bounded.
"""
import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200 import CutbError, EncodingMatrix, Plan, SequenceId, synth

pytestmark = pytest.mark.gpu

CUTB_ERR_TIMEOUT = 6
WAIT_LIMIT = 2_000_000  # cycles, about 1 ms


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def params(kind):
    S, C, T = 1024, 16, 16
    cubic = kind not in ("linear", "linear_apo")
    w = synth.Workload(kind, T, C, S, 16, 8, 32, 0, cubic=cubic, cf=1.0 if kind != "linear" else 0.0,
                       encoding=EncodingMatrix.HADAMARD, z_range=(5e-3, 15e-3), box_xy=2e-3)
    bp = synth.make_params(w)
    if kind in ("apo", "linear_apo"):
        bp.fn_rx = 1.5
    if kind == "forces":
        bp.das_shader_id = int(SequenceId.FORCES)
        bp.tx_orientation = bp.rx_orientation
    if kind in ("tpw_xz", "tpw_yz"):
        bp.das_shader_id = int(SequenceId.RCA_TPW)
        if kind == "tpw_xz":
            bp.tx_orientation = bp.rx_orientation
        for t, ang in enumerate(np.linspace(-0.2, 0.2, T)):
            bp.foci[3 * t + 2] = float(ang)
    if kind == "uforces":
        bp.das_shader_id = int(SequenceId.UFORCES)
        bp.tx_orientation = bp.rx_orientation
        bp.foci[2] = 10e-3
        for t in range(T):
            bp.sparse_elements[t] = t
    return bp


# default: short tile with double-buffered coefficients; long: 4 x 8 x 32 tile, one coefficient
# buffer; apo: apodized cubic (scalar row pass); linear: packed linear coefficients; linear_apo:
# raw taps, no coefficients; forces: the y-invariant sequence; tpw_xz / tpw_yz: tilted plane waves
# (y-invariant, and over y); uforces: sparse transmit elements after a flash.
CASES = [("default", 0), ("long", 1), ("apo", 0), ("linear", 0), ("linear_apo", 0), ("forces", 0),
         ("tpw_xz", 2), ("tpw_yz", 2), ("uforces", 2)]  # tile 2: the staged engine on this coarse grid


@pytest.mark.parametrize("kind,tile", CASES)
@pytest.mark.parametrize("where", ["first", "middle", "last"])
def test_missing_stage_times_out_and_plan_recovers(torch, kind, tile, where):
    bp = params(kind)
    plan = Plan(bp, das_tile=tile)
    S, C, T = bp.dims
    stages = (T - (kind == "uforces")) * ((C + 7) // 8)  # UFORCES: transmit row 0 is the flash
    stage = {"first": 0, "middle": stages // 2 + 1, "last": stages - 1}[where]
    g = torch.Generator(device="cuda").manual_seed(5)
    iq = torch.complex(torch.randn(T, C, S, device="cuda", generator=g),
                       torch.randn(T, C, S, device="cuda", generator=g))
    ref = plan.das(iq)
    plan.check()

    plan.debug_skip_stage(stage, WAIT_LIMIT)
    vol = plan.das(iq)
    with pytest.raises(CutbError) as err:
        plan.check()
    assert err.value.code == CUTB_ERR_TIMEOUT
    plan.check()  # the flag was cleared by the report

    plan.debug_skip_stage(-1)
    plan.das(iq, out=vol)
    plan.check()
    assert torch.equal(vol, ref)


def test_skip_stage_rejects_kernels_without_waits(torch):
    bp = params("default")
    bp.das_shader_id = int(SequenceId.RCA_TPW)
    bp.tx_orientation = bp.rx_orientation
    plan = Plan(bp, das_tile=3)  # one thread per voxel: no staged copies, no waits
    with pytest.raises(CutbError):
        plan.debug_skip_stage(0, WAIT_LIMIT)


def test_skip_stage_argument_checks(torch):
    plan = Plan(params("default"))
    with pytest.raises(CutbError):
        plan.debug_skip_stage(-2)
    with pytest.raises(CutbError):
        plan.debug_skip_stage(0, -1)
    assert np.isfinite(plan.das(torch.zeros(16, 16, 1024, dtype=torch.complex64, device="cuda"))
                       .abs().sum().item())
