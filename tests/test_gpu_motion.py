"""Image correlation and NCC motion detection on the GPU, against upstream's own outputs
(tests/golden/ncc.npz: NPP correlation + CUB candidate sort + peak fit, run on a GPU) and against
the oracle on seeded cases that cover the edges: clipped windows at the image border, grid points
outside the image, zero margins, maps of more than 2048 values, neighbour comparison, flat
windows and templates."""

import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200.params import NccMotionParameters
from tests import ncc_golden as N

pytestmark = pytest.mark.gpu

# The correlation numerator is an FP32 sum like NPP's; measured against upstream <= 4e-6 and
# against the FP64 oracle <= 3e-6 on these images. Motion vectors inherit that error through the
# quadratic fit (sub-pixel offsets are ratios of fit coefficients).
TOL_CORR = 2e-5
TOL_PEAK = 2e-5
TOL_OFFSET = 2e-3


@pytest.fixture(scope="module")
def api(native):
    from cuda_ultrasound_toolkit_b200 import api as A
    return A


def _check_corr(out, ref, what):
    assert out.shape == ref.shape, what
    flat = ref >= N.FLT_MAX
    assert ((out >= N.FLT_MAX) == flat).all(), what
    if (~flat).any():
        err = np.abs(out[~flat] - ref[~flat]).max()
        assert err < TOL_CORR, (what, err)


def _check_maps(out, ref, what):
    assert out.shape == ref.shape, what
    d = np.abs(out - ref)
    assert d[..., 2:].max() < TOL_PEAK, (what, d[..., 2:].max())
    assert d[..., :2].max() < TOL_OFFSET, (what, d[..., :2].max())
    # accepted / rejected classification identical
    assert ((out[..., 2] == -1) == (ref[..., 2] == -1)).all(), what
    assert ((out[..., 2] == -2) == (ref[..., 2] == -2)).all(), what


def _cuda(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_corr_images_device_matches_upstream(api):
    g = N.load()
    for name in N.cases(g, "corr"):
        t, s, ref = N.corr_case(g, name)
        out = api.corr_images_device(_cuda(t), _cuda(s)).cpu().numpy()
        _check_corr(out, ref, name)


def test_corr_images_host_entry_points(api):
    g = N.load()
    t, s, ref = N.corr_case(g, "large")
    a = api.corr_images(t, s)
    b = api.corr_images_f32(t, s)
    _check_corr(a, ref, "cuda_toolkit::corr_images")
    assert np.array_equal(a, b)
    assert np.array_equal(a, api.corr_images_device(_cuda(t), _cuda(s)).cpu().numpy())


@pytest.mark.parametrize("tw,th,sw,sh,kind", [
    (40, 37, 150, 90, "float"),      # several template blocks in x and y
    (1, 1, 17, 13, "u8"),
    (33, 1, 70, 4, "float"),
    (1, 20, 9, 64, "u8"),
    (16, 16, 300, 200, "u8"),        # many output tiles
    (64, 50, 64, 50, "float"),       # one position
    (7, 5, 48, 40, "flat_block"),
])
def test_corr_images_vs_oracle(api, orc, tw, th, sw, sh, kind):
    rng = np.random.default_rng(tw * 1000 + sw)
    if kind == "float":
        s = rng.normal(3.0, 1.5, (sh, sw)).astype(np.float32)
        t = s[sh - th:, :tw] + rng.normal(0, 0.3, (th, tw)).astype(np.float32)
    else:
        s = rng.integers(0, 256, (sh, sw)).astype(np.float32)
        t = rng.integers(0, 256, (th, tw)).astype(np.float32)
        if kind == "flat_block":
            s[10:30, 12:36] = 200.0
    ref = orc.corr_images(t, s)
    out = api.corr_images_device(_cuda(t), _cuda(s)).cpu().numpy()
    _check_corr(out, ref, (tw, th, sw, sh))
    if kind == "flat_block":
        assert (out >= N.FLT_MAX).any()


def test_motion_device_matches_upstream(api):
    g = N.load()
    for name in N.cases(g, "motion"):
        frames, p, ref = N.motion_case(g, name)
        out = api.motion_detection_device(_cuda(frames), p).cpu().numpy()
        _check_maps(out, ref, name)


def test_motion_host_entry_points(api):
    g = N.load()
    frames, p, ref = N.motion_case(g, "neighbour_integer")
    a = api.motion_detection(frames, p)
    b = api.motion_detect_f32(frames, p)
    _check_maps(a, ref, "cuda_toolkit::motion_detection")
    assert np.array_equal(a, b)
    assert np.array_equal(a, api.motion_detection_device(_cuda(frames), p).cpu().numpy())


def _speckle(seed, w, h, shifts):
    from cuda_ultrasound_toolkit_b200.synth import speckle_frames
    return speckle_frames(seed, w, h, shifts).astype(np.float32)


MOTION_CASES = [
    # grid points beyond the image (zero vectors), odd patch, reference = last frame
    dict(image=(70, 50), shifts=[(0, 0), (2.2, 1.1), (-1.4, 0.6)],
         p=dict(patch_size=11, motion_grid_spacing=9, motion_grid_dims=(10, 8), search_margins=(4, 4),
                abs_cor_threshold=0.2, rel_cor_threshold=0.0, min_patch_variance=0.0, use_subpixel=True,
                reference_frame=2, neighbour_compare=False)),
    # zero margins: a one-value map per grid point
    dict(image=(48, 48), shifts=[(0, 0), (0.3, 0.2)],
         p=dict(patch_size=8, motion_grid_spacing=8, motion_grid_dims=(6, 6), search_margins=(0, 0),
                abs_cor_threshold=0.0, rel_cor_threshold=0.0, min_patch_variance=0.0, use_subpixel=True,
                reference_frame=0, neighbour_compare=False)),
    # 32-pixel patches, 49 x 49 maps (more than 2048 values), neighbour comparison on 6 frames
    dict(image=(128, 112), shifts=[(0, 0), (3.5, -2.0), (7.1, -4.2), (10.4, -6.1), (14.0, -8.3), (17.2, -10.0)],
         p=dict(patch_size=32, motion_grid_spacing=24, motion_grid_dims=(5, 4), search_margins=(24, 24),
                abs_cor_threshold=0.3, rel_cor_threshold=0.01, min_patch_variance=0.01, use_subpixel=True,
                reference_frame=3, neighbour_compare=True)),
    # one frame: nothing to compare
    dict(image=(32, 32), shifts=[(0, 0)],
         p=dict(patch_size=8, motion_grid_spacing=8, motion_grid_dims=(4, 4), search_margins=(2, 2),
                abs_cor_threshold=0.1, rel_cor_threshold=0.0, min_patch_variance=0.0, use_subpixel=True,
                reference_frame=0, neighbour_compare=False)),
]


@pytest.mark.parametrize("case", range(len(MOTION_CASES)))
def test_motion_vs_oracle(api, orc, case):
    c = MOTION_CASES[case]
    (w, h), shifts = c["image"], c["shifts"]
    frames = _speckle(100 + case, w, h, shifts)
    p = NccMotionParameters.make(frame_count=len(shifts), image_dims=(w, h), **c["p"])
    ref = orc.motion_detection(frames, p)
    out = api.motion_detection_device(_cuda(frames), p).cpu().numpy()
    _check_maps(out, ref, case)
    if case == 0:
        # grid points whose patch starts past the image keep zero vectors
        assert (out[:, :, 9:] == 0).all() and (out[:, 7:] == 0).all()
        assert (out[2] == 0).all()
    if case == 3:
        assert (out == 0).all()


def test_motion_flat_frames(api, orc):
    """Constant frames: every position is flat (FLT_MAX), so every candidate is rejected."""
    frames = np.full((2, 32, 40), 100.0, dtype=np.float32)
    p = NccMotionParameters.make(frame_count=2, image_dims=(40, 32), patch_size=8, motion_grid_spacing=8,
                                 motion_grid_dims=(4, 3), search_margins=(3, 3), abs_cor_threshold=0.1,
                                 reference_frame=0)
    ref = orc.motion_detection(frames, p)
    out = api.motion_detection_device(_cuda(frames), p).cpu().numpy()
    assert np.array_equal(out, ref)
    assert (out[1, ..., 3] >= N.FLT_MAX).all()


def test_motion_rejects_bad_parameters(api):
    frames = _cuda(np.zeros((2, 16, 16), np.float32))
    p = NccMotionParameters.make(frame_count=2, image_dims=(16, 16), patch_size=4, motion_grid_spacing=4,
                                 motion_grid_dims=(2, 2), search_margins=(1, 1), reference_frame=2)
    with pytest.raises(api.CutbError) as e:
        api.motion_detection_device(frames, p)
    assert e.value.code == 1  # CUTB_ERR_INVALID_ARGUMENT
    big = _cuda(np.zeros((2, 400, 400), np.float32))
    p = NccMotionParameters.make(frame_count=2, image_dims=(400, 400), patch_size=64, motion_grid_spacing=64,
                                 motion_grid_dims=(2, 2), search_margins=(60, 60), reference_frame=0)
    with pytest.raises(api.CutbError) as e:
        api.motion_detection_device(big, p)
    assert e.value.code == 2  # CUTB_ERR_UNSUPPORTED
    # host spans shorter than the parameters say
    p = NccMotionParameters.make(frame_count=3, image_dims=(16, 16), patch_size=4, motion_grid_spacing=4,
                                 motion_grid_dims=(2, 2), search_margins=(1, 1), reference_frame=0)
    with pytest.raises(api.CutbError):
        api.motion_detection(np.zeros((2, 16, 16), np.float32), p)


def test_corr_images_rejects_bad_sizes(api):
    t = np.zeros((8, 8), np.float32)
    s = np.zeros((6, 10), np.float32)
    with pytest.raises(api.CutbError) as e:
        api.corr_images(t, s)
    assert "Template dimensions must be <= source dimensions" in e.value.message
    with pytest.raises(api.CutbError) as e:
        api.corr_images(np.zeros((0, 3), np.float32), s)
    assert "Invalid image dimensions" in e.value.message
    with pytest.raises(api.CutbError) as e:
        api.corr_images(t, np.zeros((20, 20), np.float32), dims=((8, 8), (24, 20)))
    assert "Input image spans are smaller" in e.value.message
    with pytest.raises(api.CutbError):
        api.corr_images_f32(t, s)
