"""The out-of-process transfer path on the GPU: requests from the client library
(libcuda_transfer.so) to a cutb_transfer_server process, and to an in-process server, give the
same bytes as the direct host-span entry points."""
import uuid

import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200 import synth
from cuda_ultrasound_toolkit_b200.params import InputDataTypes

pytestmark = pytest.mark.gpu


@pytest.fixture()
def T(native, monkeypatch):
    from cuda_ultrasound_toolkit_b200 import transfer
    name = "cutbg" + uuid.uuid4().hex[:10]
    monkeypatch.setenv("CUDA_TRANSFER_NAME", name)
    transfer.deinit()
    transfer.set_timeout_ms(120000)
    transfer.NAME = name
    yield transfer
    transfer.deinit()


def test_server_process_matches_direct_calls(T):
    from cuda_ultrasound_toolkit_b200 import api
    raw, bp = synth.frame("small")
    direct = api.beamform(raw, bp)
    proc = T.spawn_server(T.NAME, data_bytes=256 << 20, max_commands=4, timeout_ms=120000)
    try:
        vol = T.beamform_i16(raw, bp)
        assert np.array_equal(vol, direct)
        rawf, bpf = synth.frame("small", data_type=InputDataTypes.TYPE_F32)
        assert np.array_equal(T.beamform_f32(rawf, bpf), api.beamform(rawf, bpf))
        frames, p = synth.motion_workload(frames=3, size=96, patch=16, spacing=16, grid=6, margin=6)
        assert np.array_equal(T.motion_detect_f32(frames, p), api.motion_detection(frames, p))
        t, s = frames[0, 20:44, 30:62], frames[1]
        assert np.array_equal(T.corr_images_f32(t, s), api.corr_images(t, s))
        assert proc.wait(60) == 0  # exits after its 4 commands
    finally:
        if proc.poll() is None:
            proc.kill()


def test_in_process_server_builtin_handlers(T):
    from cuda_ultrasound_toolkit_b200 import api
    raw, bp = synth.frame("small")
    with T.Server(T.NAME, 64 << 20) as srv:
        srv.start()
        for _ in range(2):  # the staging buffer and the page-locked segment are reused
            assert np.array_equal(T.beamform_i16(raw, bp), api.beamform(raw, bp))
        # a request the library rejects answers ERR and the server keeps serving
        bad = bp.copy()
        bad.output_points[0] = 0
        with pytest.raises(T.TransferError) as e:
            T.beamform_i16(raw, bad)
        assert e.value.status == 6
        assert np.array_equal(T.beamform_i16(raw, bp), api.beamform(raw, bp))
        assert srv.stop() == 4
