"""The int8 tensor-core decode (hi/lo byte split, tcgen05 kind::i8) against the exact oracle.

Every raw int16 sample is 256 * hi + lo, so the two int8 products combine exactly in int32 and the
result must equal upstream's FP32 GEMM bit for bit (the oracle's exact restatement), like the FWHT
decode. At the precision configuration's full size (256 x 256 x 8192) the two GPU paths are
compared with each other (bit-exact), which needs no CPU oracle.
"""
import numpy as np
import pytest
import torch

from cuda_ultrasound_toolkit_b200 import CutbError, EncodingMatrix, Plan, synth

pytestmark = pytest.mark.gpu


def params(S, C, T, R0, R1, decode, cmap):
    w = synth.Workload("t", T, C, S, 8, 8, 8, 0, cubic=True, cf=0.0, encoding=decode)
    bp = synth.make_params(w, channel_map=cmap)
    bp.rf_raw_dim[0] = R0
    bp.rf_raw_dim[1] = R1
    return bp


CASES = [
    # (T, ordering, S, C, padding, extra raw channels)
    (32, 1, 256, 3, 0, 0), (32, 2, 200, 5, 8, 2), (64, 1, 128, 4, 0, 1), (96, 1, 64, 3, 0, 0),
    (128, 1, 512, 6, 16, 3), (128, 2, 136, 4, 0, 0), (160, 2, 64, 2, 0, 0), (256, 1, 384, 3, 0, 0),
    (256, 2, 72, 2, 8, 1),
]


@pytest.mark.parametrize("T,ordering,S,C,pad,extra", CASES)
@pytest.mark.parametrize("out_stride", [1, 2])
def test_tc_decode_bit_exact(orc, T, ordering, S, C, pad, extra, out_stride):
    rng = np.random.default_rng(T * 100 + S + ordering)
    R0, R1 = T * S + pad, C + extra
    raw = rng.integers(-32768, 32768, size=(R1, R0), dtype=np.int16)
    cmap = rng.permutation(R1)[:C]
    bp = params(S, C, T, R0, R1, ordering, cmap)
    plan = Plan(bp, decode_tc=True)
    out = plan.decode(torch.from_numpy(raw).cuda(), out_stride=out_stride)
    plan.check()
    got = out.cpu().numpy().reshape(T, C, S, out_stride)
    assert np.array_equal(got[..., 0], orc.decode_i16(raw, bp))
    if out_stride == 2:
        assert not got[..., 1].any()


def test_tc_decode_extreme_values(orc):
    """All-minimum and all-maximum samples: the largest sums the split must carry exactly."""
    T, S, C = 256, 64, 2
    for v in (-32768, 32767):
        raw = np.full((C, T * S), v, dtype=np.int16)
        raw[1, ::3] = -32768 if v > 0 else 32767
        bp = params(S, C, T, T * S, C, EncodingMatrix.HADAMARD, np.arange(C))
        got = Plan(bp, decode_tc=True).decode(torch.from_numpy(raw).cuda()).cpu().numpy()
        assert np.array_equal(got, orc.decode_i16(raw, bp))


def test_tc_decode_precision_config_matches_fwht():
    """Precision configuration (256 transmits x 256 channels x 8192 samples, 1 GiB of int16)."""
    T, C, S = 256, 256, 8192
    g = torch.Generator(device="cuda").manual_seed(1)
    raw = torch.randint(-32768, 32768, (C, T * S), dtype=torch.int32, device="cuda", generator=g).to(torch.int16)
    bp = params(S, C, T, T * S, C, EncodingMatrix.HADAMARD, np.random.default_rng(0).permutation(C))
    a = Plan(bp).decode(raw)
    b = Plan(bp, decode_tc=True).decode(raw)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_tc_decode_rejects_unsupported():
    with pytest.raises(CutbError):
        Plan(params(64, 2, 16, 16 * 64, 2, 1, np.arange(2)), decode_tc=True)      # 16 transmits
    with pytest.raises(CutbError):
        Plan(params(60, 2, 32, 32 * 60, 2, 1, np.arange(2)), decode_tc=True)      # 60 samples
