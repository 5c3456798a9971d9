"""Out-of-process transfer path: a Python mirror of the client library (libcuda_transfer.so,
upstream test_app/client_lib/cuda_transfer.c) and control of the server (cutb_server_* in
libcuda_toolkit_b200.so, or the cutb_transfer_server executable).

The client functions keep upstream's contract (void, errors on stderr); these wrappers raise
``TransferError`` with the client's status code instead.
"""
import ctypes
import os
import subprocess
import threading

import numpy as np

from .params import CorrImagesParameters, CudaBeamformerParameters, NccMotionParameters

_HERE = os.path.dirname(os.path.abspath(__file__))
CLIENT_PATH = os.path.join(_HERE, "libcuda_transfer.so")
SERVER_EXE = os.path.join(_HERE, "cutb_transfer_server")

# CudaCommand (communication_params.h)
ERR, ACK, SUCCESS, BEAMFORM_VOLUME, SVD_FILTER, NCC_MOTION_DETECT, CORR_IMAGES = range(7)
STATUS = {0: "ok", 1: "setup", 2: "size", 3: "send", 4: "timeout", 5: "protocol", 6: "server", 7: "disconnected"}


class SVDParameters(ctypes.Structure):
    _fields_ = [("frame_count", ctypes.c_int), ("filter_indicies", ctypes.c_int * 256)]


class SharedMemoryParams(ctypes.Structure):
    _fields_ = [("beamformerParameters", CudaBeamformerParameters), ("svdParameters", SVDParameters),
                ("nccMotionParameters", NccMotionParameters), ("corrImagesParameters", CorrImagesParameters)]


class CommandPipeMessage(ctypes.Structure):
    _fields_ = [("opcode", ctypes.c_int), ("data_size", ctypes.c_ulonglong), ("frame_count", ctypes.c_int)]


class TransferError(RuntimeError):
    def __init__(self, what, status):
        super().__init__(f"{what} failed: {STATUS.get(status, status)} ({status})")
        self.status = status


_client = None


def client():
    """libcuda_transfer.so, loaded once (raises if it has not been built)."""
    global _client
    if _client is None:
        if not os.path.exists(CLIENT_PATH):
            raise RuntimeError(f"{CLIENT_PATH} is missing: build it with `make -C {_HERE}`")
        L = ctypes.CDLL(CLIENT_PATH)
        vp = ctypes.c_void_p
        L.beamform_i16.argtypes = [vp, CudaBeamformerParameters, vp]
        L.beamform_f32.argtypes = [vp, CudaBeamformerParameters, vp]
        L.motion_detect_f32.argtypes = [vp, NccMotionParameters, vp]
        L.corr_images_f32.argtypes = [vp, vp, CorrImagesParameters, vp]
        for f in (L.beamform_i16, L.beamform_f32, L.motion_detect_f32, L.corr_images_f32, L.deinit):
            f.restype = None
        L.deinit.argtypes = []
        L.cuda_transfer_status.restype = ctypes.c_int
        L.cuda_transfer_set_timeout_ms.argtypes = [ctypes.c_uint]
        _client = L
    return _client


def _status(what):
    st = client().cuda_transfer_status()
    if st:
        raise TransferError(what, st)


def set_timeout_ms(ms):
    client().cuda_transfer_set_timeout_ms(int(ms))


def deinit():
    client().deinit()


def beamform_i16(raw, bp, out=None):
    raw = np.ascontiguousarray(raw, dtype=np.int16)
    out = np.empty(bp.volume_shape, np.complex64) if out is None else out
    client().beamform_i16(raw.ctypes.data, bp, out.ctypes.data)
    _status("beamform_i16")
    return out


def beamform_f32(raw, bp, out=None):
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    out = np.empty(bp.volume_shape, np.complex64) if out is None else out
    client().beamform_f32(raw.ctypes.data, bp, out.ctypes.data)
    _status("beamform_f32")
    return out


def motion_detect_f32(frames, params, out=None):
    frames = np.ascontiguousarray(frames, dtype=np.float32)
    shape = (int(params.frame_count), int(params.motion_grid_dims[1]), int(params.motion_grid_dims[0]), 4)
    out = np.zeros(shape, np.float32) if out is None else out
    client().motion_detect_f32(frames.ctypes.data, params, out.ctypes.data)
    _status("motion_detect_f32")
    return out


def corr_images_f32(template, source, out=None):
    t = np.ascontiguousarray(template, dtype=np.float32)
    s = np.ascontiguousarray(source, dtype=np.float32)
    p = CorrImagesParameters()
    p.template_dims[0], p.template_dims[1] = t.shape[1], t.shape[0]
    p.source_dims[0], p.source_dims[1] = s.shape[1], s.shape[0]
    shape = (max(s.shape[0] - t.shape[0] + 1, 0), max(s.shape[1] - t.shape[1] + 1, 0))
    out = np.zeros(shape, np.float32) if out is None else out
    client().corr_images_f32(t.ctypes.data, s.ctypes.data, p, out.ctypes.data)
    _status("corr_images_f32")
    return out


HANDLER = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.POINTER(SharedMemoryParams),
                           ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint8),
                           ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p)


class Server:
    """An in-process server (cutb_server_*) serving on a background thread.

    ``handler(opcode, params, data: np.ndarray[uint8]) -> bytes | None`` replaces the built-in
    GPU handlers when given (None answers ERR); without it the requests run on the GPU."""

    def __init__(self, name, data_bytes=64 << 20, handler=None):
        from .api import lib, _check
        L = lib()
        L.cutb_server_create.argtypes = [ctypes.c_char_p, ctypes.c_uint64]
        L.cutb_server_create.restype = ctypes.c_void_p
        L.cutb_server_set_handler.argtypes = [ctypes.c_void_p, HANDLER, ctypes.c_void_p]
        L.cutb_server_serve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.cutb_server_serve.restype = ctypes.c_int
        L.cutb_server_stop.argtypes = [ctypes.c_void_p]
        L.cutb_server_destroy.argtypes = [ctypes.c_void_p]
        self._L = L
        self.name = name
        self._h = L.cutb_server_create(name.encode(), data_bytes)
        _check(self._h, "cutb_server_create")
        self._cb = None
        if handler is not None:
            def cb(op, params, data, nbytes, out, cap, out_bytes, user):
                try:
                    res = handler(op, params.contents, np.ctypeslib.as_array(data, (nbytes,)).copy() if nbytes else
                                  np.zeros(0, np.uint8))
                except Exception:  # a handler error answers ERR
                    return 1
                if res is None or len(res) > cap:
                    return 1
                ctypes.memmove(out, bytes(res), len(res))
                out_bytes[0] = len(res)
                return 0
            self._cb = HANDLER(cb)
            L.cutb_server_set_handler(self._h, self._cb, None)
        self._thread = None
        self.handled = None

    def start(self, max_commands=0, idle_timeout_ms=0):
        def run():
            self.handled = self._L.cutb_server_serve(self._h, max_commands, idle_timeout_ms)
        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return self

    def stop(self, timeout=10):
        if self._thread is not None:
            self._L.cutb_server_stop(self._h)
            self._thread.join(timeout)
            self._thread = None
        return self.handled

    def close(self):
        self.stop()
        if self._h:
            self._L.cutb_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def spawn_server(name, data_bytes=256 << 20, max_commands=0, timeout_ms=600000):
    """Starts cutb_transfer_server in a child process and waits for its "ready" line."""
    p = subprocess.Popen([SERVER_EXE, "--name", name, "--data-bytes", str(data_bytes), "--max-commands",
                          str(max_commands), "--timeout-ms", str(timeout_ms)], stdout=subprocess.PIPE, text=True)
    line = p.stdout.readline()
    if not line.startswith("ready"):
        p.kill()
        raise RuntimeError(f"cutb_transfer_server did not start: {line!r}")
    return p
