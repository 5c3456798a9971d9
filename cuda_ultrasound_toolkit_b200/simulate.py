"""GPU RF simulator (csrc/simulate.cu): int16 raw frames of point-scatterer phantoms in the
raw layout the pipeline reads, on the device, with a counter-based (Philox4x32-10) noise
stream keyed by the frame seed."""
import ctypes

import numpy as np
import torch

from . import synth
from .api import _check, _stream_handle, lib


class _SimConfig(ctypes.Structure):
    _fields_ = [("transmits", ctypes.c_uint), ("rows_per_transmit", ctypes.c_uint), ("channels", ctypes.c_uint),
                ("samples", ctypes.c_uint), ("pitch", ctypes.c_float), ("sampling_frequency", ctypes.c_float),
                ("center_frequency", ctypes.c_float), ("speed_of_sound", ctypes.c_float),
                ("snr_db", ctypes.c_float), ("encoding", ctypes.c_int), ("array_rows", ctypes.c_uint),
                ("row_stride", ctypes.c_uint), ("row_offset", ctypes.c_uint), ("reserved", ctypes.c_uint * 3)]


_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        vp = ctypes.c_void_p
        sig = {
            "cutb_sim_create": ([ctypes.POINTER(_SimConfig)], vp),
            "cutb_sim_destroy": ([vp], None),
            "cutb_sim_run": ([vp, vp, ctypes.c_uint, ctypes.POINTER(ctypes.c_int16), ctypes.c_ulonglong, vp, vp, vp],
                             ctypes.c_bool),
            "cutb_sim_copy_signal": ([vp, vp, vp], ctypes.c_bool),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _bound = True
    return L


class Simulator:
    """Simulates frames of `transmits` events, `channels` receive columns and `samples` samples
    per event. Event t fires rows t * row_stride + row_offset + k, k < rows_per_transmit, of an
    array of `array_rows` rows (defaults: row_stride = rows_per_transmit, array_rows =
    transmits * row_stride)."""

    def __init__(self, transmits, channels, samples, rows_per_transmit=1, pitch=synth.PITCH, fs=synth.FS,
                 fc=synth.FC, c_sound=synth.C_SOUND, snr_db=40.0, hadamard=True, row_stride=0, row_offset=0,
                 array_rows=0):
        self.cfg = _SimConfig(transmits, rows_per_transmit, channels, samples, pitch, fs, fc, c_sound, snr_db,
                              1 if hadamard else 0, array_rows, row_stride, row_offset)
        self.shape = (transmits, channels, samples)
        self._h = _lib().cutb_sim_create(ctypes.byref(self.cfg))
        _check(self._h, "cutb_sim_create")

    def close(self):
        if getattr(self, "_h", None):
            _lib().cutb_sim_destroy(self._h)
            self._h = None

    __del__ = close

    def run(self, scatterers, channel_map, seed, raw=None, gain=None, stream=None):
        """scatterers: float32 [n][4] (numpy or CUDA tensor); channel_map: [C] ints.
        Returns (raw int16 CUDA tensor [C][T*S], gain float32 CUDA tensor [1])."""
        T, C, S = self.shape
        if not isinstance(scatterers, torch.Tensor):
            scatterers = torch.from_numpy(np.ascontiguousarray(scatterers, dtype=np.float32)).cuda()
        assert scatterers.is_cuda and scatterers.dtype == torch.float32 and scatterers.shape[1] == 4
        scatterers = scatterers.contiguous()
        cmap = np.ascontiguousarray(channel_map, dtype=np.int16)
        assert cmap.size == C
        raw = torch.empty((C, T * S), dtype=torch.int16, device="cuda") if raw is None else raw
        gain = torch.empty(1, dtype=torch.float32, device="cuda") if gain is None else gain
        _check(_lib().cutb_sim_run(self._h, scatterers.data_ptr(), scatterers.shape[0],
                                   cmap.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)), int(seed), raw.data_ptr(),
                                   gain.data_ptr(), _stream_handle(stream)), "cutb_sim_run")
        return raw, gain

    def signal(self, stream=None):
        """The encoded, noisy FP32 signal [T][C][S] of the last run."""
        out = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        _check(_lib().cutb_sim_copy_signal(self._h, out.data_ptr(), _stream_handle(stream)), "cutb_sim_copy_signal")
        return out
