"""ctypes wrapper of the upstream sources compiled for the CPU (oracle/_ref, built by
oracle/Makefile.ref). TEST INFRASTRUCTURE ONLY: used to generate the golden fixtures under
tests/golden/ and to pin the oracle; absent on machines without the upstream sources."""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(_HERE, "_ref", "libcuda_toolkit_ref.so")
_lib = None


def available():
    return os.path.exists(PATH)


def lib():
    global _lib
    if _lib is None:
        from cuda_ultrasound_toolkit_b200.params import CudaBeamformerParameters
        L = ctypes.CDLL(PATH)
        vp, u = ctypes.c_void_p, ctypes.c_uint
        L.ref_encoding_matrix.argtypes = [u, ctypes.c_int, vp]
        L.ref_encoding_matrix.restype = ctypes.c_int
        L.ref_register_buffer.argtypes = [u, vp, ctypes.c_size_t]
        L.beamform_i16_matlab.argtypes = [vp, CudaBeamformerParameters, vp]
        L.beamform_f32_matlab.argtypes = [vp, CudaBeamformerParameters, vp]
        L.init_cuda_configuration.argtypes = [ctypes.POINTER(u), ctypes.POINTER(u)]
        L.register_cuda_buffers.argtypes = [ctypes.POINTER(u), u, u]
        L.cuda_set_channel_mapping.argtypes = [ctypes.POINTER(ctypes.c_int16)]
        L.cuda_set_match_filter.argtypes = [ctypes.POINTER(ctypes.c_float), u]
        L.cuda_decode.argtypes = [ctypes.c_size_t, u]
        L.cuda_hilbert.argtypes = [u, u]
        L.ref_convert_demod.argtypes = [vp, ctypes.c_int, u, u, u, u, u, vp, ctypes.c_float, ctypes.c_float, vp,
                                        ctypes.c_int, vp]
        L.ref_convert_demod.restype = ctypes.c_int
        for f in ("init_cuda_configuration", "register_cuda_buffers", "cuda_set_channel_mapping",
                  "cuda_set_match_filter", "cuda_decode", "cuda_hilbert"):
            getattr(L, f).restype = ctypes.c_bool
        _lib = L
    return _lib


def encoding_matrix(n, ordering):
    out = np.empty((n, n), np.float32)
    if lib().ref_encoding_matrix(n, ordering, out.ctypes.data) != 0:
        raise ValueError(f"upstream rejects order {n}")
    return out


def beamform(raw, bp):
    """Upstream beamform_i16_matlab / beamform_f32_matlab: complex64 [Z][Y][X]."""
    out = np.zeros(bp.volume_shape, np.complex64)
    raw = np.ascontiguousarray(raw)
    fn = lib().beamform_i16_matlab if raw.dtype == np.int16 else lib().beamform_f32_matlab
    fn(raw.ctypes.data, bp, out.ctypes.data)
    return out


def decode_and_hilbert(raw, bp, taps=None):
    """Upstream GL front end: init_cuda_configuration, cuda_decode, cuda_hilbert on host buffers.
    Returns (decoded [T][C][S] float32 = .x of cuda_decode's output, analytic signal complex64)."""
    L = lib()
    S, C, T = bp.dims
    raw = np.ascontiguousarray(raw, np.int16)
    dec = np.zeros((T, C, S), np.complex64)
    iq = np.zeros((T, C, S), np.complex64)
    L.ref_register_buffer(1, raw.ctypes.data, raw.nbytes)
    L.ref_register_buffer(2, dec.ctypes.data, dec.nbytes)
    L.ref_register_buffer(3, iq.ctypes.data, iq.nbytes)
    ok = L.init_cuda_configuration((ctypes.c_uint * 2)(int(bp.rf_raw_dim[0]), int(bp.rf_raw_dim[1])),
                                   (ctypes.c_uint * 3)(S, C, T))
    ok = ok and L.register_cuda_buffers((ctypes.c_uint * 2)(2, 3), 2, 1)
    m = np.zeros(256, np.int16)
    m[:C] = np.ctypeslib.as_array(bp.channel_mapping)[:C]
    ok = ok and L.cuda_set_channel_mapping(m.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)))
    t = np.zeros(0, np.float32) if taps is None else np.ascontiguousarray(taps, np.float32)
    ok = ok and L.cuda_set_match_filter(t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(t))
    ok = ok and L.cuda_decode(0, 0) and L.cuda_hilbert(0, 1)
    L.deinit_cuda_configuration()
    if not ok:
        raise RuntimeError("upstream front end failed")
    return dec.real.copy(), iq


def convert_demod(raw, bp, demod_freq, sample_freq, taps=None):
    """RfProcessor::convert_demod of the upstream CPU build: complex64 [T][C][S] (S complex samples)."""
    S, C, T = bp.dims
    raw = np.ascontiguousarray(raw)
    from cuda_ultrasound_toolkit_b200.params import InputDataTypes
    dtype = int(InputDataTypes.TYPE_I16 if raw.dtype == np.int16 else InputDataTypes.TYPE_F32)
    cmap = np.zeros(256, np.int16)
    cmap[:C] = np.ctypeslib.as_array(bp.channel_mapping)[:C]
    t = np.zeros(0, np.float32) if taps is None else np.ascontiguousarray(taps, dtype=np.float32)
    out = np.zeros((T, C, S), np.complex64)
    rc = lib().ref_convert_demod(raw.ctypes.data, dtype, int(bp.rf_raw_dim[0]), int(bp.rf_raw_dim[1]), S, C, T,
                                 cmap.ctypes.data, float(demod_freq), float(sample_freq), t.ctypes.data if len(t) else None,
                                 len(t), out.ctypes.data)
    if rc != 0:
        raise RuntimeError("upstream convert_demod failed")
    return out
