"""The out-of-process transfer protocol on CPU: upstream's message layout, the client library
against an in-process server with replacement handlers (no GPU), and the failure paths: server
errors, client timeouts, servers that are absent, restarted or sent invalid requests."""
import ctypes
import os
import socket
import struct
import subprocess
import time
import uuid

import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200.params import CudaBeamformerParameters, NccMotionParameters

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


@pytest.fixture()
def T(native, monkeypatch):
    from cuda_ultrasound_toolkit_b200 import transfer
    name = "cutbt" + uuid.uuid4().hex[:10]
    monkeypatch.setenv("CUDA_TRANSFER_NAME", name)
    transfer.deinit()
    transfer.set_timeout_ms(20000)
    transfer.NAME = name
    yield transfer
    transfer.deinit()


def test_wire_layout(tmp_path):
    """CommandPipeMessage and SharedMemoryParams have upstream's x86-64 layout, and the ctypes
    mirrors agree with the C header."""
    from cuda_ultrasound_toolkit_b200 import transfer
    src = tmp_path / "w.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "communication_params.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(CommandPipeMessage),\n'
                   ' offsetof(CommandPipeMessage, data_size), offsetof(CommandPipeMessage, frame_count),\n'
                   ' sizeof(SharedMemoryParams), offsetof(SharedMemoryParams, svdParameters),\n'
                   ' offsetof(SharedMemoryParams, nccMotionParameters),\n'
                   ' offsetof(SharedMemoryParams, corrImagesParameters), sizeof(SVDParameters)); return 0; }\n')
    exe = tmp_path / "w"
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    S = transfer.SharedMemoryParams
    assert vals == [24, 8, 16, ctypes.sizeof(S), S.svdParameters.offset, S.nccMotionParameters.offset,
                    S.corrImagesParameters.offset, ctypes.sizeof(transfer.SVDParameters)]
    assert ctypes.sizeof(transfer.CommandPipeMessage) == 24


def _bp(x=4, y=3, z=5, r0=64, r1=8):
    bp = CudaBeamformerParameters()
    bp.rf_raw_dim[0], bp.rf_raw_dim[1] = r0, r1
    bp.output_points[0], bp.output_points[1], bp.output_points[2] = x, y, z
    bp.time_offset = 1.25e-6
    return bp


def _echo(op, params, data):
    """Replacement handler: answers from the request alone, so the test can recompute it."""
    if op == 3:  # BEAMFORM_VOLUME: volume filled with (input byte sum, time_offset)
        bp = params.beamformerParameters
        n = bp.output_points[0] * bp.output_points[1] * bp.output_points[2]
        v = np.empty(2 * n, np.float32)
        v[0::2] = float(data.astype(np.int64).sum())
        v[1::2] = bp.time_offset
        return v.tobytes()
    if op == 5:  # NCC_MOTION_DETECT: per frame, its float sum
        p = params.nccMotionParameters
        f = data.view(np.float32).reshape(p.frame_count, -1)
        cells = p.motion_grid_dims[0] * p.motion_grid_dims[1]
        return np.repeat(f.sum(1), cells * 4).astype(np.float32).tobytes()
    if op == 6:  # CORR_IMAGES: template sum everywhere
        p = params.corrImagesParameters
        nt = p.template_dims[0] * p.template_dims[1]
        nc = (p.source_dims[0] - p.template_dims[0] + 1) * (p.source_dims[1] - p.template_dims[1] + 1)
        return np.full(nc, data.view(np.float32)[:nt].sum(), np.float32).tobytes()
    return None


def test_round_trip_every_request(T):
    rng = np.random.default_rng(1)
    with T.Server(T.NAME, 1 << 20, handler=_echo) as s:
        s.start()
        bp = _bp()
        raw = rng.integers(-3000, 3000, (8, 64)).astype(np.int16)
        vol = T.beamform_i16(raw, bp)
        assert vol.shape == (5, 3, 4)
        assert (vol.real == float(raw.view(np.uint8).astype(np.int64).sum())).all()
        assert (vol.imag == np.float32(1.25e-6)).all()
        rawf = rng.normal(size=(8, 64)).astype(np.float32)
        vol = T.beamform_f32(rawf, bp)
        assert (vol.real == np.float32(rawf.view(np.uint8).astype(np.int64).sum())).all()
        p = NccMotionParameters.make(frame_count=3, image_dims=(10, 6), motion_grid_dims=(2, 4))
        frames = rng.normal(size=(3, 6, 10)).astype(np.float32)
        m = T.motion_detect_f32(frames, p)
        assert m.shape == (3, 4, 2, 4)
        np.testing.assert_allclose(m[:, 0, 0, 0], frames.reshape(3, -1).sum(1), rtol=1e-5)
        t, src = rng.normal(size=(3, 4)).astype(np.float32), rng.normal(size=(7, 9)).astype(np.float32)
        c = T.corr_images_f32(t, src)
        assert c.shape == (5, 6)
        np.testing.assert_allclose(c, t.sum(), rtol=1e-5)
        assert s.stop() == 4


def test_server_error_then_recovery(T):
    calls = []

    def h(op, params, data):
        calls.append(op)
        return None if len(calls) == 1 else _echo(op, params, data)

    with T.Server(T.NAME, 1 << 20, handler=h) as s:
        s.start()
        p = NccMotionParameters.make(frame_count=1, image_dims=(4, 4), motion_grid_dims=(1, 1))
        with pytest.raises(T.TransferError) as e:
            T.motion_detect_f32(np.ones((1, 4, 4), np.float32), p)
        assert e.value.status == 6  # CUDA_TRANSFER_ERR_SERVER
        m = T.motion_detect_f32(np.ones((1, 4, 4), np.float32), p)  # reconnects
        assert m[0, 0, 0, 0] == 16


def test_client_side_validation(T):
    with T.Server(T.NAME, 4096, handler=_echo) as s:
        s.start()
        with pytest.raises(T.TransferError) as e:
            T.corr_images_f32(np.ones((5, 5)), np.ones((4, 9)))
        assert e.value.status == 2
        with pytest.raises(T.TransferError) as e:  # larger than the 4 KiB data segment
            T.beamform_f32(np.ones((8, 256), np.float32), _bp(r0=256))
        assert e.value.status == 2
        assert s.stop() == 0  # nothing reached the server


def test_client_timeout_and_late_answer(T):
    """A request that outlives the client's timeout fails with TIMEOUT; the late answer goes to
    the closed connection and the next request is served normally."""
    def slow(op, params, data):
        time.sleep(1.0)
        return _echo(op, params, data)

    with T.Server(T.NAME, 1 << 20, handler=slow) as s:
        s.start()
        T.set_timeout_ms(200)
        p = NccMotionParameters.make(frame_count=1, image_dims=(4, 4), motion_grid_dims=(1, 1))
        t0 = time.monotonic()
        with pytest.raises(T.TransferError) as e:
            T.motion_detect_f32(np.ones((1, 4, 4), np.float32), p)
        assert e.value.status == 4 and time.monotonic() - t0 < 0.9
        T.set_timeout_ms(5000)
        m = T.motion_detect_f32(np.full((1, 4, 4), 2, np.float32), p)
        assert m[0, 0, 0, 0] == 32


def test_no_server(T):
    t0 = time.monotonic()
    with pytest.raises(T.TransferError) as e:
        T.corr_images_f32(np.ones((2, 2)), np.ones((3, 3)))
    assert e.value.status == 1 and time.monotonic() - t0 < 2


def test_server_restart(T):
    p = NccMotionParameters.make(frame_count=1, image_dims=(4, 4), motion_grid_dims=(1, 1))
    with T.Server(T.NAME, 1 << 20, handler=_echo) as s:
        s.start()
        assert T.motion_detect_f32(np.ones((1, 4, 4), np.float32), p)[0, 0, 0, 0] == 16
    # the server is gone: the client's connection and segments are stale
    with pytest.raises(T.TransferError):
        T.motion_detect_f32(np.ones((1, 4, 4), np.float32), p)
    with T.Server(T.NAME, 1 << 20, handler=_echo) as s:
        s.start()
        assert T.motion_detect_f32(np.full((1, 4, 4), 3, np.float32), p)[0, 0, 0, 0] == 48


def _raw_client(name):
    c = socket.socket(socket.AF_UNIX, socket.SOCK_SEQPACKET)
    c.settimeout(5)
    c.connect("\0" + name + "_command")
    return c


def _msg(op, size):
    return struct.pack("<iIQi4x", op, 0, size, 0)


def _reply(c):
    op, _, size, _ = struct.unpack("<iIQi4x", c.recv(64))
    return op, size


def test_server_rejects_invalid_requests(T):
    """Oversized data, SVD_FILTER and unknown opcodes answer ERR (upstream would end its loop or
    never answer) and the server keeps serving; client-side response opcodes are ignored."""
    with T.Server(T.NAME, 4096, handler=_echo) as s:
        s.start()
        c = _raw_client(T.NAME)
        c.send(_msg(3, 1 << 20))
        assert _reply(c) == (0, 0)
        c.send(_msg(4, 0))
        assert _reply(c) == (0, 0)
        c.send(_msg(42, 0))
        assert _reply(c) == (0, 0)
        c.send(_msg(1, 0))  # ACK from a client: logged, no answer
        c.send(b"short")  # not a message: ignored
        c.send(_msg(6, 0))  # CORR_IMAGES: ACK, then the replacement handler's 1-value map
        assert _reply(c) == (1, 0)
        assert _reply(c) == (2, 4)
        c.close()
        p = NccMotionParameters.make(frame_count=1, image_dims=(4, 4), motion_grid_dims=(1, 1))
        assert T.motion_detect_f32(np.ones((1, 4, 4), np.float32), p)[0, 0, 0, 0] == 16
        assert s.stop() == 6  # the ignored ACK counts as a command


def test_builtin_handler_validation_without_gpu(T):
    """The built-in corr_images handler validates the request before ACK, as upstream
    (test_app.cpp:214-252): a size mismatch answers ERR without ACK."""
    with T.Server(T.NAME, 4096) as s:
        s.start()
        shm = os.path.join("/dev/shm", T.NAME + "_parameters")
        with open(shm, "r+b") as f:
            base = T.SharedMemoryParams.corrImagesParameters.offset
            f.seek(base)
            f.write(struct.pack("<4I", 2, 2, 3, 3))
        c = _raw_client(T.NAME)
        c.send(_msg(6, 4 * 4))  # 4 floats, but 2x2 + 3x3 = 13 are needed
        assert _reply(c) == (0, 0)
        c.close()


def test_second_server_of_the_same_name_is_refused(T):
    """The command socket name acts as the lock: a second server fails to start and leaves the
    running server's shared memory in place."""
    p = NccMotionParameters.make(frame_count=1, image_dims=(4, 4), motion_grid_dims=(1, 1))
    with T.Server(T.NAME, 1 << 20, handler=_echo) as s:
        s.start()
        with pytest.raises(Exception):
            T.Server(T.NAME, 1 << 20, handler=_echo)
        assert T.motion_detect_f32(np.ones((1, 4, 4), np.float32), p)[0, 0, 0, 0] == 16


def test_server_executable_starts_and_times_out(native):
    from cuda_ultrasound_toolkit_b200 import transfer
    name = "cutbt" + uuid.uuid4().hex[:10]
    p = transfer.spawn_server(name, data_bytes=1 << 20, timeout_ms=300)
    assert p.wait(10) == 0
    assert not os.path.exists(os.path.join("/dev/shm", name + "_data"))  # segments removed
