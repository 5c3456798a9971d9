"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

Bars: the convert + reorder + decode stage is bit-exact against the oracle's exact
restatement of the upstream FP32 result; the analytic signal and the volume are compared
with the FP64 oracle by relative L2 error (tolerances stated per test).
"""
import ctypes
import math

import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200 import (ApoType, CutbError, EncodingMatrix, InputDataTypes, Plan, RfSession,
                                          SequenceId, beamform, beamform_f32, beamform_i16, synth)
from cuda_ultrasound_toolkit_b200.params import CudaBeamformerParameters

pytestmark = pytest.mark.gpu

# Relative L2 tolerances (GPU FP32 vs oracle FP64).
TOL_HILBERT = 2e-6          # FP32 shared-memory FFT, twiddles rounded once from FP64
TOL_DAS_RANDOM = 2e-4       # random analytic rows: FP32 delay rounding (~1e-4 sample) x signal slope
TOL_DAS_APO = 2e-3          # Hann / sine apodization in FP32 (__cosf, sinf) and 0.1-threshold flips
TOL_VOLUME = 1e-5           # phantom volume (coherent sum) through the whole pipeline


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def base_params(S, C, T, X=16, Y=8, Z=24, R0=None, R1=None, decode=EncodingMatrix.HADAMARD, cmap=None,
                data_type=InputDataTypes.TYPE_I16):
    w = synth.Workload("t", T, C, S, X, Y, Z, 0, cubic=True, cf=0.0, encoding=decode)
    bp = synth.make_params(w, data_type=data_type, channel_map=cmap)
    if R0 is not None:
        bp.rf_raw_dim[0] = R0
    if R1 is not None:
        bp.rf_raw_dim[1] = R1
    return bp


# ---------------------------------------------------------------------------------------------
# convert + reorder + decode
# ---------------------------------------------------------------------------------------------
DECODE_CASES = [
    # (T, ordering, S, C, padding, extra raw channels)
    (1, 1, 64, 3, 0, 0), (2, 1, 64, 3, 0, 0), (8, 2, 64, 5, 7, 2), (16, 1, 128, 4, 0, 0), (32, 2, 64, 3, 0, 1),
    (64, 1, 256, 6, 0, 0), (128, 1, 64, 4, 16, 3), (128, 2, 64, 4, 0, 0), (256, 1, 32, 3, 0, 0),
    (512, 2, 32, 2, 0, 0), (1024, 1, 16, 2, 0, 0),
    (12, 1, 64, 3, 0, 0), (24, 2, 64, 3, 4, 1), (96, 1, 32, 3, 0, 0), (768, 1, 16, 2, 0, 0),
    (20, 1, 64, 3, 0, 0), (40, 2, 32, 3, 0, 0), (640, 1, 16, 2, 0, 0),
    (64, 0, 64, 4, 3, 1),  # decode == NONE
    (16, 1, 34, 3, 0, 0),  # sample count not a multiple of 4: scalar-load path
    (20, 1, 30, 3, 1, 0),  # idem for the base-20 kernel
]


@pytest.mark.parametrize("T,ordering,S,C,pad,extra", DECODE_CASES)
@pytest.mark.parametrize("out_stride", [1, 2])
def test_decode_bit_exact_int16(torch, orc, T, ordering, S, C, pad, extra, out_stride):
    rng = np.random.default_rng(T * 1000 + S + ordering)
    R0, R1 = T * S + pad, C + extra
    raw = rng.integers(-32768, 32768, size=(R1, R0), dtype=np.int16)
    cmap = rng.permutation(R1)[:C]
    bp = base_params(S, C, T, R0=R0, R1=R1, decode=ordering, cmap=cmap)
    plan = Plan(bp)
    out = plan.decode(torch.from_numpy(raw).cuda(), out_stride=out_stride)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(T, C, S, out_stride)
    ref = orc.decode_i16(raw, bp)
    assert np.array_equal(got[..., 0], ref)
    if out_stride == 2:
        assert not got[..., 1].any()
    assert plan.launches == 1


def test_decode_f32_integer_valued_bit_exact(torch, orc):
    rng = np.random.default_rng(2)
    S, C, T = 256, 8, 128
    raw16 = rng.integers(-32768, 32768, size=(C, T * S), dtype=np.int16)
    bp = base_params(S, C, T, cmap=rng.permutation(C), data_type=InputDataTypes.TYPE_F32)
    got = Plan(bp).decode(torch.from_numpy(raw16.astype(np.float32)).cuda()).cpu().numpy()
    assert np.array_equal(got, orc.decode_i16(raw16, bp))


def test_decode_f32_general(torch, orc):
    rng = np.random.default_rng(3)
    S, C, T = 128, 4, 96
    raw = rng.normal(size=(C, T * S)).astype(np.float32)
    bp = base_params(S, C, T, cmap=rng.permutation(C), data_type=InputDataTypes.TYPE_F32)
    got = Plan(bp).decode(torch.from_numpy(raw).cuda()).cpu().numpy()
    assert rel_l2(got, orc.decode_f64(raw, bp)) < 1e-6


# ---------------------------------------------------------------------------------------------
# Hilbert
# ---------------------------------------------------------------------------------------------
# Powers of two run at their own length (16384: one row per CTA); other counts as a zero-padded
# transform of at least twice the length (8191: the longest, padded to 16384).
@pytest.mark.parametrize("N", [16, 64, 256, 1024, 2048, 4096, 8192, 16384,
                               8, 100, 127, 1001, 2500, 3072, 6000, 8191])
@pytest.mark.parametrize("taps", [0, 64])
def test_hilbert_vs_fp64(torch, orc, N, taps):
    T, C = 3, 5                                    # 15 rows: odd count exercises the unpaired row
    rng = np.random.default_rng(N + taps)
    rows = rng.normal(size=(T, C, N)).astype(np.float32)
    bp = base_params(N, C, T, decode=EncodingMatrix.NONE)
    h = None
    if taps:
        h = synth.chirp_taps(min(taps, N))
        bp.filter_length = len(h)
        for i, v in enumerate(h):
            bp.rf_filter[i] = float(v)
    plan = Plan(bp)
    got = plan.hilbert(torch.from_numpy(rows).cuda()).cpu().numpy()
    ref = orc.hilbert(rows.astype(np.float64), h)
    assert rel_l2(got, ref) < TOL_HILBERT


# Rows of more than 2^14 transform points: a thread-block cluster of 2, 4 or 8 CTAs per row (the
# exchange arrays spread over their shared memory). 8193 samples pad to 32768 (the oracle's DFT of a
# length that is not a power of two is a direct sum, so that case keeps to one row).
@pytest.mark.parametrize("N,rows,taps", [(32768, 2, 0), (32768, 2, 64), (65536, 2, 64), (131072, 2, 64),
                                         (131072, 1, 0), (8193, 1, 64)])
def test_hilbert_cluster_lengths_vs_fp64(torch, orc, N, rows, taps):
    rng = np.random.default_rng(N + taps + rows)
    x = rng.normal(size=(1, rows, N)).astype(np.float32)
    bp = base_params(N, rows, 1, decode=EncodingMatrix.NONE)
    h = None
    if taps:
        h = synth.chirp_taps(taps)
        bp.filter_length = len(h)
        for i, v in enumerate(h):
            bp.rf_filter[i] = float(v)
    plan = Plan(bp)
    got = plan.hilbert(torch.from_numpy(x).cuda()).cpu().numpy()
    plan.check()
    ref = orc.hilbert(x.astype(np.float64), h)
    assert rel_l2(got, ref) < TOL_HILBERT


def test_hilbert_strided_input_and_known_answer(torch, orc):
    N, T, C = 1024, 2, 2
    n = np.arange(N)
    rows = np.stack([np.cos(2 * np.pi * k * n / N) for k in (1, 5, 100, N // 2)]).reshape(T, C, N)
    cplx = np.zeros((T, C, N, 2), np.float32)
    cplx[..., 0] = rows
    cplx[..., 1] = 123.0                           # the imaginary part must be ignored
    plan = Plan(base_params(N, C, T))
    got = plan.hilbert(torch.from_numpy(cplx).cuda().reshape(T, C, 2 * N), in_stride=2).cpu().numpy()
    expect = np.stack([0.75 * np.exp(2j * np.pi * k * n / N) for k in (1, 5, 100)] + [1.5 * (-1.0) ** n])
    np.testing.assert_allclose(got.reshape(4, N), expect, atol=2e-6)


# ---------------------------------------------------------------------------------------------
# delay and sum
# ---------------------------------------------------------------------------------------------
def das_params(seq=SequenceId.HERCULES, cubic=True, cf=0.0, fn_rx=0.0, fn_tx=0.0, apo=ApoType.RX_HANN,
               readi=0, readi_id=0, decode=EncodingMatrix.HADAMARD, focus_z=math.inf, S=512, C=8, T=8,
               X=20, Y=9, Z=40, z=(4e-3, 26e-3), time_offset=0.0, x=(-3e-3, 3e-3)):
    bp = base_params(S, C, T, X=X, Y=Y, Z=Z, decode=decode)
    bp.das_shader_id = int(seq)
    bp.interpolate = bool(cubic)
    bp.coherency_weighting = cf
    bp.fn_rx, bp.fn_tx = fn_rx, fn_tx
    bp.apo_type = int(apo)
    bp.to_power = 2
    bp.readi_group_count, bp.readi_group_id = readi, readi_id
    bp.foci[2] = focus_z
    bp.output_min_coordinate[0], bp.output_max_coordinate[0] = x
    bp.output_min_coordinate[1] = -1e-3
    bp.output_min_coordinate[2], bp.output_max_coordinate[2] = z
    bp.time_offset = time_offset
    return bp


def analytic_rows(orc, T, C, S, seed):
    """Band-limited analytic rows (Hilbert of random pulses), the kind of data DAS sees."""
    rng = np.random.default_rng(seed)
    x = np.zeros((T, C, S))
    n = np.arange(S)
    for _ in range(12):
        c0 = rng.uniform(20, S - 20)
        x += rng.normal() * np.exp(-0.5 * ((n - c0) / 3.4) ** 2) * np.cos(2 * np.pi * 0.25 * (n - c0))
    x += 0.05 * rng.normal(size=x.shape)
    return orc.hilbert(x)


DAS_CASES = [
    dict(),                                             # HERCULES plane wave, cubic, no CF
    dict(cubic=False),
    dict(cf=1.0),
    dict(cf=0.5, cubic=False),
    dict(focus_z=15e-3),                                # YZ_FOCUS
    dict(time_offset=2e-7),
    dict(z=(0.0, 60e-3)),                               # reaches z = 0 and the clamp at S-2
    dict(z=(0.0, 60e-3), cf=1.0),                       # packed path: clamped and clamp-free stages, CF
    dict(readi=2, readi_id=1),
    dict(readi=4, readi_id=2, decode=EncodingMatrix.WALSH),
    dict(seq=SequenceId.FORCES),
    dict(seq=SequenceId.FORCES, cubic=False, cf=0.3),
    dict(seq=SequenceId.FORCES, readi=2, readi_id=1),
    dict(X=33, Y=3, Z=70),                              # partial tiles in every direction
]
DAS_APO_CASES = [
    dict(fn_rx=1.5),
    dict(apo=ApoType.RX_TO_SIN),
    dict(seq=SequenceId.FORCES, fn_rx=1.0, fn_tx=2.0),
    dict(seq=SequenceId.FORCES, apo=ApoType.RX_TO_SIN),
    dict(seq=SequenceId.FORCES, apo=ApoType.TX_TO_SIN),
    dict(seq=SequenceId.FORCES, apo=ApoType.BOTH_TO_SIN),
]


@pytest.mark.parametrize("case", DAS_CASES + DAS_APO_CASES, ids=lambda c: ",".join(f"{k}={v}" for k, v in c.items()) or "default")
def test_das_vs_fp64(torch, orc, case):
    bp = das_params(**case)
    S, C, T = bp.dims
    iq = analytic_rows(orc, T, C, S, seed=len(str(case)))
    plan = Plan(bp)
    got = plan.das(torch.from_numpy(iq.astype(np.complex64)).cuda()).cpu().numpy()
    ref = orc.das(iq, bp)
    tol = TOL_DAS_APO if case in DAS_APO_CASES else TOL_DAS_RANDOM
    err = rel_l2(got, ref)
    assert err < tol, err
    if bp.das_shader_id == SequenceId.FORCES:      # y-invariant
        assert (got == got[:, :1, :]).all()


TILE_CASES = [dict(), dict(cf=1.0, cubic=False), dict(focus_z=15e-3), dict(X=33, Y=3, Z=70),
              dict(z=(10e-3, 14e-3)), dict(z=(10e-3, 13e-3), cf=1.0, fn_rx=1.5),
              # staged windows with linear interpolation over many stages (C = 64 -> 8 per transmit)
              dict(z=(10e-3, 14e-3), cubic=False, C=64, T=16), dict(z=(10e-3, 14e-3), cubic=False, cf=0.7, C=32),
              # fine grids: the 8x8x16 tile's window bound (4 reach + 8 samples) fits the 80 samples of the
              # double-buffered form; X=25 sits just inside the bound (78.9), X=24 just outside (81.5)
              dict(X=40, Z=48, z=(10e-3, 12e-3)), dict(X=40, Z=48, z=(10e-3, 12e-3), cubic=False, cf=0.7, C=64, T=16),
              dict(X=40, Z=48, z=(0.0, 2e-3), cf=1.0), dict(X=44, Y=11, Z=35, z=(20e-3, 21.5e-3), time_offset=2e-7),
              dict(X=25, Z=40, z=(10e-3, 13e-3)), dict(X=24, Z=40, z=(10e-3, 13e-3))]


@pytest.mark.parametrize("tile", [1, 2], ids=["tile4x8x32", "tile8x8x16"])
@pytest.mark.parametrize("case", TILE_CASES, ids=lambda c: ",".join(f"{k}={v}" for k, v in c.items()) or "default")
def test_das_tile_shapes(torch, orc, case, tile):
    """Both HERCULES tile shapes (staged and direct windows) against the FP64 oracle."""
    bp = das_params(**case)
    S, C, T = bp.dims
    iq = analytic_rows(orc, T, C, S, seed=3 + len(str(case)))
    got = Plan(bp, das_tile=tile).das(torch.from_numpy(iq.astype(np.complex64)).cuda()).cpu().numpy()
    tol = TOL_DAS_APO if "fn_rx" in case else TOL_DAS_RANDOM
    assert rel_l2(got, orc.das(iq, bp)) < tol


@pytest.mark.parametrize("splits", [1, 3, 16])
@pytest.mark.parametrize("tile", [1, 2])
def test_das_tile_list(torch, orc, splits, tile):
    """Listed tiles with split stage slices equal the whole-grid delay-and-sum there; other voxels are 0."""
    bp = das_params(z=(10e-3, 14e-3), C=24, T=8, X=24, Y=16, Z=64)
    S, C, T = bp.dims
    iq = torch.from_numpy(analytic_rows(orc, T, C, S, seed=4).astype(np.complex64)).cuda()
    plan = Plan(bp, das_tile=tile)
    full = plan.das(iq).cpu().numpy()
    tx, ty, tz = plan.tile_shape
    nx, ny, nz = -(-24 // tx), -(-16 // ty), -(-64 // tz)
    ids = np.array(sorted(set([0, nx * ny * nz - 1, 5 % (nx * ny * nz), (nx * ny * nz) // 2])), dtype=np.int32)
    got = plan.das_tiles(iq, ids, splits=splits).cpu().numpy()
    mask = np.zeros(full.shape, bool)
    for i in ids:
        x, y, z = i % nx, (i // nx) % ny, i // (nx * ny)
        mask[z * tz:(z + 1) * tz, y * ty:(y + 1) * ty, x * tx:(x + 1) * tx] = True
    assert np.all(got[~mask] == 0)
    assert rel_l2(got[mask], full[mask]) < 1e-6
    plan.check()


def test_das_tile_list_rejects_bad_ids(torch):
    plan = Plan(das_params(z=(10e-3, 14e-3)))
    iq = plan.empty_iq()
    with pytest.raises(CutbError):
        plan.das_tiles(iq, [-1])
    with pytest.raises(CutbError):
        plan.das_tiles(iq, [10 ** 6])


TPW_UFORCES_CASES = [
    dict(seq=SequenceId.RCA_TPW, angles=np.linspace(-0.2, 0.2, 8), fn_rx=1.0, cf=0.5),          # YZ plane
    dict(seq=SequenceId.RCA_TPW, angles=np.linspace(-0.1, 0.3, 8), same=True, cf=1.0),           # XZ plane
    dict(seq=SequenceId.RCA_TPW, angles=np.linspace(-0.1, 0.1, 8), same=True, cubic=False, cf=0.0),
    dict(seq=SequenceId.UFORCES, elems=[0, 2, 3, 5, 6, 8, 9, 11], same=True, focus_z=20e-3, fn_rx=1.0, cf=0.5),
    dict(seq=SequenceId.UFORCES, elems=list(range(8)), same=True, focus_z=30e-3, cf=1.0, cubic=False),
    dict(seq=SequenceId.UFORCES, elems=list(range(8)), same=True, focus_z=30e-3, cf=0.3, z=(0.0, 30e-3)),  # clamp at 0
    # fine grids: the staged windows fit, so tile 0 takes the staged engine
    dict(seq=SequenceId.RCA_TPW, angles=np.linspace(-0.2, 0.2, 8), same=True, cf=1.0, fn_rx=1.0, X=64, Z=64,
         x=(-1.5e-3, 1.5e-3), z=(4e-3, 7e-3)),
    dict(seq=SequenceId.RCA_TPW, angles=np.linspace(-0.2, 0.2, 8), cf=0.5, X=32, Y=16, Z=48,
         x=(-0.8e-3, 0.8e-3), z=(4e-3, 6e-3)),
    dict(seq=SequenceId.UFORCES, elems=[0, 2, 3, 5, 6, 8, 9, 11], same=True, focus_z=20e-3, fn_rx=1.0, cf=0.5,
         X=64, Z=64, x=(-1.5e-3, 1.5e-3), z=(4e-3, 7e-3)),
]


@pytest.mark.parametrize("case", TPW_UFORCES_CASES, ids=lambda c: f"{int(c['seq'])}-" + "-".join(
    f"{k}" for k in c if k != "seq"))
@pytest.mark.parametrize("bf16", [False, True])
# 0: chosen (one thread per voxel here, the grids are too coarse for the stage buffers); 1, 2: the staged
# engine (TPW over y: 4 x 8 x 32 and 8 x 8 x 16 tiles; rows whose window overflows read global memory);
# 3: one thread per voxel
@pytest.mark.parametrize("tile", [0, 1, 2, 3])
def test_das_tpw_uforces_vs_fp64(torch, orc, case, bf16, tile):
    case = dict(case)
    angles, elems, same = case.pop("angles", None), case.pop("elems", None), case.pop("same", False)
    bp = das_params(**case)
    if same:
        bp.tx_orientation = bp.rx_orientation
    if angles is not None:
        for t, a in enumerate(angles):
            bp.foci[3 * t + 2] = float(a)
    if elems is not None:
        for t, e in enumerate(elems):
            bp.sparse_elements[t] = int(e)
    S, C, T = bp.dims
    iq = analytic_rows(orc, T, C, S, seed=21 + len(str(case)))
    plan = Plan(bp, iq_bf16=bf16, das_tile=tile)
    if bf16:
        d = torch.from_numpy(np.stack([iq.real, iq.imag], -1).astype(np.float32)).cuda().to(torch.bfloat16)
    else:
        d = torch.from_numpy(iq.astype(np.complex64)).cuda()
    got = plan.das(d).cpu().numpy()
    plan.check()
    ref = orc.das(iq, bp)
    assert rel_l2(got, ref) < (2e-2 if bf16 else TOL_DAS_APO)
    if bp.das_shader_id == SequenceId.UFORCES or bp.tx_orientation == bp.rx_orientation:  # y-invariant
        assert (got == got[:, :1, :]).all()


BANDPASS_CASES = [
    # (T, encoding, S, C, taps, f32 input)
    (8, EncodingMatrix.NONE, 256, 6, 0, False), (16, EncodingMatrix.HADAMARD, 512, 4, 31, False),
    (32, EncodingMatrix.WALSH, 128, 3, 8, True), (12, EncodingMatrix.HADAMARD, 300, 5, 64, False),
]


@pytest.mark.parametrize("T,enc,S,C,ntaps,f32", BANDPASS_CASES)
def test_bandpass_front_end_vs_fp64(torch, orc, T, enc, S, C, ntaps, f32):
    """Bandpass IQ pairs: exact transmit decode of the raw pairs, demodulation, time-domain filter."""
    rng = np.random.default_rng(T * 7 + S)
    R0, R1 = 2 * T * S + 4, C + 1
    bp = base_params(S, C, T, R0=R0, R1=R1, decode=enc, cmap=rng.permutation(R1)[:C],
                     data_type=InputDataTypes.TYPE_F32 if f32 else InputDataTypes.TYPE_I16)
    bp.sample_type = 1
    taps = synth.chirp_taps(ntaps) if ntaps else np.zeros(0, np.float32)
    bp.filter_length = ntaps
    for i, v in enumerate(taps):
        bp.rf_filter[i] = float(v)
    raw = rng.integers(-32768, 32768, size=(R1, R0), dtype=np.int16)
    if f32:
        raw = raw.astype(np.float32)
    plan = Plan(bp)
    dec = plan.decode(torch.from_numpy(raw).cuda())
    iq = plan.hilbert(dec).cpu().numpy()
    plan.check()
    ref = orc.convert_demod(raw, bp, taps if ntaps else None)
    assert rel_l2(iq, ref) < 2e-6


def test_bandpass_pipeline_vs_oracle(torch, orc):
    rng = np.random.default_rng(5)
    T, C, S = 16, 8, 512
    bp = das_params(S=S, C=C, T=T, z=(4e-3, 12e-3))
    bp.sample_type = 1
    bp.rf_raw_dim[0] = 2 * T * S
    raw = rng.integers(-3000, 3000, size=(C, 2 * T * S), dtype=np.int16)
    vol = Plan(bp).beamform(torch.from_numpy(raw).cuda()).cpu().numpy()
    iq = orc.convert_demod(raw, bp)
    vox = rng.choice(vol.size, 1024, replace=False)
    assert rel_l2(vol.ravel()[vox], orc.das(iq, bp, vox)) < TOL_DAS_RANDOM


@pytest.mark.parametrize("grid", [dict(), dict(X=40, Z=48, z=(10e-3, 12e-3))], ids=["coarse", "fine"])
def test_das_bf16_storage(torch, orc, grid):
    """BF16 analytic-signal storage; the fine grid's 8x8x16-tile window bound (51 samples) selects
    the double-buffered-coefficient form."""
    bp = das_params(cf=1.0, **grid)
    S, C, T = bp.dims
    iq = analytic_rows(orc, T, C, S, seed=9)
    plan = Plan(bp, iq_bf16=True)
    iq_b = torch.from_numpy(np.stack([iq.real, iq.imag], -1).astype(np.float32)).cuda().to(torch.bfloat16)
    got = plan.das(iq_b).cpu().numpy()
    assert rel_l2(got, orc.das(iq, bp)) < 2e-2     # bf16 keeps 8 bits of mantissa


# ---------------------------------------------------------------------------------------------
# whole pipeline
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def small_frame():
    return synth.frame("small")


def test_pipeline_small_vs_oracle(torch, orc, small_frame):
    raw, bp = small_frame
    plan = Plan(bp)
    d_raw = torch.from_numpy(raw).cuda()
    vol = plan.beamform(d_raw).cpu().numpy()
    assert plan.launches == 3
    dec = plan.decode(d_raw).cpu().numpy()
    assert np.array_equal(dec, orc.decode_i16(raw, bp))
    iq = plan.hilbert(torch.from_numpy(dec).cuda()).cpu().numpy()
    iq_ref = orc.hilbert(dec.astype(np.float64))
    assert rel_l2(iq, iq_ref) < TOL_HILBERT
    rng = np.random.default_rng(0)
    vox = rng.choice(vol.size, 4096, replace=False)
    ref = orc.das(iq_ref, bp, vox)
    assert rel_l2(vol.ravel()[vox], ref) < TOL_VOLUME


@pytest.mark.parametrize("S", [1000, 2500])
def test_pipeline_sample_count_not_power_of_two(torch, orc, S):
    """Whole pipeline with rows whose length is not a power of two (the analytic signal runs as a
    zero-padded transform), against the FP64 oracle's decode -> Hilbert (length-S DFT) -> DAS."""
    w = synth.Workload("np2", 8, 8, S, 16, 8, 32, 4, cubic=True, cf=1.0, filter_taps=16, z_range=(5e-3, 15e-3),
                       box_xy=2e-3)
    raw, cmap, _, _ = synth.synth_frame(w, 9)
    bp = synth.make_params(w, channel_map=cmap)
    plan = Plan(bp)
    vol = plan.beamform(torch.from_numpy(raw).cuda()).cpu().numpy()
    plan.check()
    ref, _, _ = orc.pipeline(raw, bp)
    assert rel_l2(vol, ref) < 1e-4


def test_host_span_entry_points(torch, small_frame):
    raw, bp = small_frame
    ref = Plan(bp).beamform(torch.from_numpy(raw).cuda()).cpu().numpy()
    assert np.array_equal(beamform(raw, bp), ref)
    assert np.array_equal(beamform_i16(raw, bp), ref)
    bpf = bp.copy()
    bpf.data_type = InputDataTypes.TYPE_F32
    assert np.array_equal(beamform_f32(raw.astype(np.float32), bpf), ref)
    with pytest.raises(CutbError):                  # output span too short
        beamform(raw, bp, out=np.empty(10, np.complex64))


def test_buffer_registry_front_end(torch, orc, small_frame):
    raw, bp = small_frame
    S, C, T = bp.dims
    sess = RfSession((int(bp.rf_raw_dim[0]), int(bp.rf_raw_dim[1])), (S, C, T))
    try:
        pad = 64                                            # input offset into the raw buffer
        d_raw = torch.zeros(raw.size + pad // 2, dtype=torch.int16, device="cuda")
        d_raw[pad // 2:] = torch.from_numpy(raw.ravel()).cuda()
        bufs = [torch.full((T, C, S), 7 + 7j, dtype=torch.complex64, device="cuda") for _ in range(2)]
        raw_id = sess.register(d_raw)
        ids = [sess.register(b) for b in bufs]
        sess.register_buffers(ids, raw_id)
        sess.set_channel_mapping(np.ctypeslib.as_array(bp.channel_mapping)[:C])
        taps = synth.chirp_taps(32)
        sess.set_match_filter(taps)
        sess.decode(pad, 0)
        dec = bufs[0].cpu().numpy()
        ref = orc.decode_i16(raw, bp)
        assert np.array_equal(dec.real, ref) and not dec.imag.any()
        sess.hilbert(0, 1)
        iq = bufs[1].cpu().numpy()
        assert rel_l2(iq, orc.hilbert(ref.astype(np.float64), taps)) < TOL_HILBERT
        with pytest.raises(CutbError):
            sess.decode(0, 5)                               # index beyond the registered buffers
    finally:
        sess.close()


# ---------------------------------------------------------------------------------------------
# error contract
# ---------------------------------------------------------------------------------------------
def test_invalid_parameters_are_rejected(torch):
    S, C, T = 64, 4, 8
    bad = []
    bp = base_params(S, C, T, R0=T * S - 1); bad.append((bp, 1))               # rows shorter than T*S
    bp = base_params(S, C, 36); bad.append((bp, 2))                             # unsupported order
    bp = base_params(S, C, T); bp.channel_mapping[1] = 99; bad.append((bp, 1))  # map outside raw channels
    bp = base_params(S, C, T); bp.sample_type = 7; bad.append((bp, 2))          # unknown sample type
    bp = base_params(S, C, T); bp.sample_type = 1; bad.append((bp, 1))          # bandpass: raw rows hold no IQ pairs
    bp = base_params(S, C, T); bp.data_type = 4; bad.append((bp, 2))            # u8 input
    bp = base_params(S, C, T); bp.das_shader_id = SequenceId.RCA_VLS; bad.append((bp, 2))
    bp = base_params(S, C, T); bp.rx_orientation = bp.tx_orientation; bad.append((bp, 2))  # XZ focus for HERCULES
    bp = base_params(S, C, T); bp.readi_group_count = 2; bp.readi_group_id = 5; bad.append((bp, 1))
    bp = base_params(S, C, T); bp.filter_length = S + 1; bad.append((bp, 1))
    for bp, code in bad:
        with pytest.raises(CutbError) as e:
            Plan(bp)
        assert e.value.code == code, e.value
    # decode works, the FFT length does not (not a power of two, and over 65536)
    plan = Plan(base_params(65537, C, T))
    with pytest.raises(CutbError) as e:
        plan.beamform(torch.zeros(65537 * T * C, dtype=torch.int16, device="cuda"))
    assert e.value.code == 2


def test_allocation_failure_injection(torch):
    from cuda_ultrasound_toolkit_b200 import lib
    bp = base_params(64, 4, 8)
    lib().cutb_debug_fail_allocations_after(1)
    try:
        with pytest.raises(CutbError) as e:
            Plan(bp)
        assert e.value.code == 5
    finally:
        lib().cutb_debug_fail_allocations_after(-1)
    Plan(bp)


def test_short_raw_buffer_rejected(torch):
    bp = base_params(64, 4, 8)
    plan = Plan(bp)
    with pytest.raises(CutbError):
        plan.beamform(torch.zeros(10, dtype=torch.int16, device="cuda"))
