"""The oracle (and the library's host-side encoding tables) against golden vectors produced by the
upstream toolkit's own code (tests/golden/make_golden.py: upstream sources compiled for the CPU).
No GPU needed."""
import os

import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200.params import CudaBeamformerParameters

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# Upstream computes delays in FP32 (~1e-4 sample rounding of ~1000-sample indices); the oracle
# in FP64. Measured oracle-vs-upstream relative L2 on these cases: 1.6e-5 .. 2.5e-5.
TOL_VOLUME_UPSTREAM = 1e-4
TOL_IQ_UPSTREAM = 1e-6   # upstream's FFT runs in the emulation in FP64, rounded to FP32


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


def _params(buf):
    return CudaBeamformerParameters.from_buffer_copy(buf.tobytes())


def test_encoding_matrices_match_upstream(orc, native):
    from cuda_ultrasound_toolkit_b200 import encoding_matrix
    g = _load("encoding_matrices.npz")
    assert len(g.files) == 48
    for key in g.files:
        n, o = (int(v[1:]) for v in key.split("_"))
        assert np.array_equal(orc.encoding_matrix(n, o), g[key]), key
        assert np.array_equal(encoding_matrix(n, o), g[key]), key


def test_frontend_matches_upstream(orc):
    g = _load("frontend.npz")
    names = sorted(k[:-4] for k in g.files if k.endswith(".raw"))
    assert len(names) == 8  # 4 power-of-two and 4 other sample counts
    for n in names:
        bp = _params(g[n + ".params"])
        dec = orc.decode_i16(g[n + ".raw"], bp)
        assert np.array_equal(dec, g[n + ".decoded"]), n
        taps = g[n + ".taps"]
        iq = orc.hilbert(dec.astype(np.float64), taps if len(taps) else None)
        want = g[n + ".iq"]
        assert np.linalg.norm(iq - want) / np.linalg.norm(want) < TOL_IQ_UPSTREAM, n


def test_volumes_match_upstream(orc):
    g = _load("volumes.npz")
    names = sorted(k[:-7] for k in g.files if k.endswith(".params"))
    assert len(names) == 16
    for n in names:
        bp = _params(g[n + ".params"])
        vol, _, _ = orc.pipeline(g["raw"], bp)
        want = g[n + ".volume"]
        assert np.abs(want).max() > 0, n
        err = np.linalg.norm(vol - want) / np.linalg.norm(want)
        assert err < TOL_VOLUME_UPSTREAM, (n, err)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                    "oracle", "_ref", "libcuda_toolkit_ref.so")),
                    reason="upstream CPU build (oracle/Makefile.ref) not present")
def test_golden_files_are_reproducible():
    """When the upstream CPU build is present, it still reproduces the committed fixtures."""
    from oracle import ref
    g = _load("encoding_matrices.npz")
    for key in ("n24_o2", "n640_o2", "n1024_o1"):
        n, o = (int(v[1:]) for v in key.split("_"))
        assert np.array_equal(ref.encoding_matrix(n, o).astype(np.int8), g[key])
    v = _load("volumes.npz")
    bp = _params(v["hercules_readi_walsh.params"])
    assert np.array_equal(ref.beamform(v["raw"], bp), v["hercules_readi_walsh.volume"])


def test_trained_weights_are_committed():
    """The learned path's weights ship with the package and match the network's layout."""
    import os
    from cuda_ultrasound_toolkit_b200 import sparse
    assert os.path.exists(sparse.WEIGHTS)
    d = np.load(sparse.WEIGHTS)
    assert tuple(d["grid"]) == sparse.GRID
    # 11 layers: sum over layers of cout * (27 * cin + 1) in the padded master layout
    specs = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 64), (128, 32), (64, 16), (32, 16),
             (16, 16)]
    assert d["params"].size == sum(co * (27 * ci + 1) for ci, co in specs)
    assert np.all(np.isfinite(d["params"]))


def test_bandpass_front_end_matches_upstream(orc):
    """The oracle's bandpass demodulation + filter against upstream's RfProcessor::convert_demod."""
    g = _load("bandpass.npz")
    names = sorted(k[:-4] for k in g.files if k.endswith(".raw"))
    assert len(names) == 3
    for n in names:
        bp = _params(g[n + ".params"])
        taps = g[n + ".taps"]
        got = orc.convert_demod(g[n + ".raw"], bp, taps if len(taps) else None)
        want = g[n + ".iq"]
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-4, n


# ---- image correlation and NCC motion detection (tests/golden/make_ncc_golden.py, on a GPU) -------
# Upstream's correlation is NPP's FP32 nppiCrossCorrValid_NormLevel_32f_C1R; the oracle forms it in
# FP64. Measured oracle-vs-upstream: correlation values <= 3.6e-6, motion vectors <= 7e-6.
TOL_CORR_UPSTREAM = 2e-5
TOL_MOTION_UPSTREAM = 1e-4


def test_corr_images_oracle_matches_upstream(orc):
    from tests import ncc_golden as N
    g = N.load()
    names = N.cases(g, "corr")
    assert len(names) == 7
    for name in names:
        t, s, ref = N.corr_case(g, name)
        out = orc.corr_images(t, s)
        assert out.shape == ref.shape, name
        flat = ref >= N.FLT_MAX  # zero-variance positions: NPP returns FLT_MAX
        assert ((out >= N.FLT_MAX) == flat).all(), name
        assert np.abs(out[~flat] - ref[~flat]).max(initial=0) < TOL_CORR_UPSTREAM, name
    # the flat cases exercise both zero-variance forms
    assert (N.corr_case(g, "flat_template")[2] >= N.FLT_MAX).all()
    ref = N.corr_case(g, "flat_block")[2]
    assert 0 < (ref >= N.FLT_MAX).sum() < ref.size


def test_motion_oracle_matches_upstream(orc):
    from tests import ncc_golden as N
    g = N.load()
    names = N.cases(g, "motion")
    assert len(names) == 5
    for name in names:
        frames, p, ref = N.motion_case(g, name)
        out = orc.motion_detection(frames, p)
        assert out.shape == ref.shape, name
        assert np.abs(out - ref).max() < TOL_MOTION_UPSTREAM, name
        # the reference frame keeps its cleared map
        assert (out[p.reference_frame] == 0).all()
    # the cases cover accepted vectors, rejected peaks (-1) and sub-pixel offsets
    _, _, m = N.motion_case(g, "tiny_search_strict")
    assert (m[..., 2] == -1).any() and (m[..., 2] > 0).any()
    _, _, m = N.motion_case(g, "subpixel_ref0")
    assert (np.abs(m[..., 0] - np.rint(m[..., 0])) > 0.05).any()
