"""The benchmark frame end to end against the FP64 oracle, at full size.

Workload "full": 128 transmits x 128 channels x 4096 samples of Hadamard-encoded int16 RF, 64-tap
chirp match filter, HERCULES plane wave, 128 x 128 x 256 volume, cubic interpolation and
coherence-factor weighting: the configuration the benchmark times. The same integer samples are
also sent as float32. Bars: the convert + reorder + decode stage is bit-exact; the volume on a
seeded sample of voxels is within TOL_VOLUME relative L2 of the FP64 oracle's decode -> Hilbert ->
delay-and-sum of the same frame. The 256 x 256 x 8192 frame (linear, no coherence factor, int8
tensor-core decode) is checked the same way.
"""
import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200 import InputDataTypes, Plan, beamform, beamform_f32, synth

pytestmark = pytest.mark.gpu

TOL_VOLUME = 1e-5   # relative L2 of the sampled voxels, GPU FP32 pipeline vs FP64 oracle
N_VOXELS = 16384    # seeded voxel sample of the 4,194,304-voxel volume


def rel_l2(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def full_frame(orc):
    raw, bp = synth.frame("full")
    z, y, x = bp.volume_shape
    vox = np.sort(np.random.default_rng(20).choice(x * y * z, N_VOXELS, replace=False))
    ref, _, _ = orc.pipeline(raw, bp, voxels=vox)
    return raw, bp, vox, ref


def test_full_frame_int16_device(torch, orc, full_frame):
    raw, bp, vox, ref = full_frame
    plan = Plan(bp)
    d_raw = torch.from_numpy(raw).cuda()
    dec = plan.decode(d_raw).cpu().numpy()
    assert np.array_equal(dec, orc.decode_i16(raw, bp))
    vol = plan.beamform(d_raw)
    plan.check()
    got = vol.reshape(-1)[torch.from_numpy(vox).cuda()].cpu().numpy()
    assert rel_l2(got, ref) < TOL_VOLUME


def test_full_frame_f32_device_and_host(torch, orc, full_frame):
    raw, bp, vox, ref = full_frame
    bp32 = bp.copy()
    bp32.data_type = int(InputDataTypes.TYPE_F32)
    raw32 = raw.astype(np.float32)
    plan = Plan(bp32)
    d_raw = torch.from_numpy(raw32).cuda()
    dec = plan.decode(d_raw).cpu().numpy()
    assert np.array_equal(dec, orc.decode_i16(raw, bp))
    vol = plan.beamform(d_raw)
    plan.check()
    got = vol.reshape(-1)[torch.from_numpy(vox).cuda()].cpu().numpy()
    assert rel_l2(got, ref) < TOL_VOLUME
    # the MATLAB entry point and cuda_toolkit::beamform with host buffers give the same volume
    host = beamform_f32(raw32, bp32)
    assert np.array_equal(host, vol.cpu().numpy())
    assert np.array_equal(beamform(raw, bp), host)


def test_precision_frame_vs_fp64(torch, orc):
    """256 x 256 x 8192 (int8 tensor-core decode, linear, no coherence factor), volume on a
    seeded voxel sample against the FP64 oracle."""
    from cuda_ultrasound_toolkit_b200.simulate import Simulator
    w = synth.CONFIGS["precision"]
    rng = np.random.default_rng(3000)
    cmap = rng.permutation(w.C).astype(np.int16)
    scat = synth.phantom(rng, w.scatterers, 0, box_xy=w.box_xy, z_range=w.z_range)
    d_raw, _ = Simulator(w.T, w.C, w.S).run(scat, cmap, 3000)
    bp = synth.make_params(w, channel_map=cmap)
    plan = Plan(bp, decode_tc=True)
    vol = plan.beamform(d_raw)
    plan.check()
    raw = d_raw.cpu().numpy()
    z, y, x = bp.volume_shape
    vox = np.sort(rng.choice(x * y * z, 4096, replace=False))
    ref, _, _ = orc.pipeline(raw, bp, voxels=vox)
    got = vol.reshape(-1)[torch.from_numpy(vox).cuda()].cpu().numpy()
    assert rel_l2(got, ref) < TOL_VOLUME
