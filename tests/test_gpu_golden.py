"""The CUDA path (through the C ABI) against golden vectors produced by the upstream toolkit's
own code (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200 import Plan, RfSession, beamform_i16
from cuda_ultrasound_toolkit_b200.params import CudaBeamformerParameters

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_VOLUME_UPSTREAM = 1e-4   # upstream FP32 delays vs this library (see test_golden.py)
TOL_IQ_UPSTREAM = 2e-6


def _params(buf):
    return CudaBeamformerParameters.from_buffer_copy(buf.tobytes())


def test_gl_front_end_matches_upstream():
    import torch
    g = np.load(os.path.join(GOLDEN, "frontend.npz"))
    for n in sorted(k[:-4] for k in g.files if k.endswith(".raw")):
        bp = _params(g[n + ".params"])
        S, C, T = bp.dims
        raw = g[n + ".raw"]
        sess = RfSession((int(bp.rf_raw_dim[0]), int(bp.rf_raw_dim[1])), (S, C, T))
        try:
            d_raw = torch.from_numpy(raw).cuda()
            bufs = [torch.zeros((T, C, S), dtype=torch.complex64, device="cuda") for _ in range(2)]
            rid = sess.register(d_raw)
            ids = [sess.register(b) for b in bufs]
            sess.register_buffers(ids, rid)
            sess.set_channel_mapping(np.ctypeslib.as_array(bp.channel_mapping)[:C])
            sess.set_match_filter(g[n + ".taps"])
            sess.decode(0, 0)
            sess.hilbert(0, 1)
            dec, iq = bufs[0].cpu().numpy(), bufs[1].cpu().numpy()
        finally:
            sess.close()
        assert np.array_equal(dec.real, g[n + ".decoded"]), n
        want = g[n + ".iq"]
        assert np.linalg.norm(iq - want) / np.linalg.norm(want) < TOL_IQ_UPSTREAM, n


def test_volumes_match_upstream():
    import torch
    g = np.load(os.path.join(GOLDEN, "volumes.npz"))
    raw = g["raw"]
    for n in sorted(k[:-7] for k in g.files if k.endswith(".params")):
        bp = _params(g[n + ".params"])
        want = g[n + ".volume"]
        got = Plan(bp).beamform(torch.from_numpy(raw).cuda()).cpu().numpy()
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < TOL_VOLUME_UPSTREAM, (n, err)
        host = beamform_i16(raw, bp)                       # the MATLAB entry point, host spans
        assert np.array_equal(host, got), n


def test_bandpass_front_end_matches_upstream():
    import torch
    g = np.load(os.path.join(GOLDEN, "bandpass.npz"))
    for n in sorted(k[:-4] for k in g.files if k.endswith(".raw")):
        bp = _params(g[n + ".params"])
        plan = Plan(bp)
        iq = plan.hilbert(plan.decode(torch.from_numpy(g[n + ".raw"]).cuda())).cpu().numpy()
        plan.check()
        want = g[n + ".iq"]
        assert np.linalg.norm(iq - want) / np.linalg.norm(want) < 1e-4, n
