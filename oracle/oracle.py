"""ctypes wrapper of the CPU oracle (liboracle.so). TEST INFRASTRUCTURE ONLY: imported by
tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py, never by the package."""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        vp, u, i = ctypes.c_void_p, ctypes.c_uint, ctypes.c_int
        L.orc_encoding_matrix.argtypes = [u, i, vp]
        L.orc_convert_decode_i16.argtypes = [vp, u, u, u, u, u, vp, i, vp, i]
        L.orc_convert_decode_f64.argtypes = [vp, i, u, u, u, u, u, vp, i, vp, i]
        L.orc_hilbert.argtypes = [vp, ctypes.c_size_t, u, vp, u, vp, i]
        L.orc_das.argtypes = [vp, vp, vp, ctypes.c_size_t, vp, i]
        L.orc_corr_images.argtypes = [vp, u, u, vp, u, u, vp]
        L.orc_motion_detection.argtypes = [vp, vp, vp, i]
        for f in (L.orc_encoding_matrix, L.orc_convert_decode_i16, L.orc_convert_decode_f64, L.orc_hilbert,
                  L.orc_das, L.orc_corr_images, L.orc_motion_detection):
            f.restype = i
        _lib = L
    return _lib


def _ok(rc, what):
    if rc != 0:
        raise ValueError(f"oracle rejected {what}")


def encoding_matrix(n, ordering=1):
    out = np.empty((n, n), dtype=np.int8)
    _ok(lib().orc_encoding_matrix(n, ordering, out.ctypes.data), "encoding order")
    return out


def _dims(bp):
    return int(bp.rf_raw_dim[0]), int(bp.rf_raw_dim[1]), int(bp.dec_data_dim[0]), int(bp.dec_data_dim[1]), \
        int(bp.dec_data_dim[2])


def decode_i16(raw, bp, threads=0):
    """Bit-exact FP32 result of the upstream convert + decode for int16 raw data: [T][C][S]."""
    R0, R1, S, C, T = _dims(bp)
    raw = np.ascontiguousarray(raw, dtype=np.int16)
    cmap = np.ctypeslib.as_array(bp.channel_mapping)[:C].astype(np.int16).copy()
    out = np.empty((T, C, S), dtype=np.float32)
    _ok(lib().orc_convert_decode_i16(raw.ctypes.data, R0, R1, S, C, T, cmap.ctypes.data, int(bp.decode),
                                     out.ctypes.data, threads), "decode dims")
    return out


def decode_f64(raw, bp, threads=0):
    R0, R1, S, C, T = _dims(bp)
    raw = np.ascontiguousarray(raw)
    dt = 1 if raw.dtype == np.int16 else 2
    cmap = np.ctypeslib.as_array(bp.channel_mapping)[:C].astype(np.int16).copy()
    out = np.empty((T, C, S), dtype=np.float64)
    _ok(lib().orc_convert_decode_f64(raw.ctypes.data, dt, R0, R1, S, C, T, cmap.ctypes.data, int(bp.decode),
                                     out.ctypes.data, threads), "decode dims")
    return out


def hilbert(rows, taps=None, threads=0):
    """FP64 match-filtered analytic signal of each row of a real [..., N] array."""
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    N = rows.shape[-1]
    flat = rows.reshape(-1, N)
    taps = np.zeros(0, np.float32) if taps is None else np.ascontiguousarray(taps, dtype=np.float32)
    out = np.empty(flat.shape, dtype=np.complex128)
    _ok(lib().orc_hilbert(flat.ctypes.data, flat.shape[0], N, taps.ctypes.data, len(taps), out.ctypes.data,
                          threads), "hilbert length")
    return out.reshape(rows.shape)


def das(iq, bp, voxels=None, threads=0):
    """FP64 delay-and-sum of complex [T][C][S] into [Z][Y][X] (or the listed linear voxels)."""
    iq = np.ascontiguousarray(iq, dtype=np.complex128)
    if voxels is None:
        n = int(bp.output_points[0]) * int(bp.output_points[1]) * int(bp.output_points[2])
        out = np.empty(n, dtype=np.complex128)
        _ok(lib().orc_das(iq.ctypes.data, ctypes.byref(bp), None, 0, out.ctypes.data, threads), "das parameters")
        z, y, x = (int(bp.output_points[2]), int(bp.output_points[1]), int(bp.output_points[0]))
        return out.reshape(z, y, x)
    vox = np.ascontiguousarray(voxels, dtype=np.int64)
    out = np.empty(len(vox), dtype=np.complex128)
    _ok(lib().orc_das(iq.ctypes.data, ctypes.byref(bp), vox.ctypes.data, len(vox), out.ctypes.data, threads),
        "das parameters")
    return out


def pipeline(raw, bp, voxels=None, threads=0):
    """decode (FP64) -> Hilbert (FP64) -> DAS (FP64)."""
    S = int(bp.dec_data_dim[0])
    dec = decode_f64(raw, bp, threads)
    taps = np.ctypeslib.as_array(bp.rf_filter)[: int(bp.filter_length)].astype(np.float32)
    iq = hilbert(dec, taps if len(taps) else None, threads)
    return das(iq, bp, voxels, threads), iq, dec


def convert_demod(raw, bp, taps=None):
    """FP64 restatement of the bandpass front end (TEST INFRASTRUCTURE ONLY).

    Every two raw samples of a transmit are an IQ pair (data_conversion_kernels.cuh:46-65). The
    transmit decode is applied exactly to the raw pairs first (as decode_i16 / decode_f64 with
    2 S samples per row), then z[s] = (x[2s] - i x[2s+1]) exp(-i 2 pi s fc / fs)
    (data_conversion_kernels.cuh:14-20, with fc the parameter block's centre frequency), then the
    time-domain filter of data_conversion_kernels.cuh:67-102: correlation with the reversed taps,
    normalised by the number of taps inside the row. Returns complex [T][C][S]."""
    S, C, T = bp.dims
    sub = bp.copy()
    sub.dec_data_dim[0] = 2 * S
    sub.sample_type = 0
    if np.asarray(raw).dtype == np.int16:
        dec = decode_i16(raw, sub).astype(np.float64)
    else:
        dec = decode_f64(raw, sub)
    z = dec[..., 0::2] - 1j * dec[..., 1::2]
    r = float(bp.center_frequency) / float(bp.sampling_frequency)
    s = np.arange(S)
    z = z * np.exp(-2j * np.pi * np.mod(s * r, 1.0))
    if taps is None or len(taps) == 0:
        return z
    h = np.asarray(taps, dtype=np.float64)
    L, half = len(h), len(h) // 2
    acc = np.zeros_like(z)
    cnt = np.zeros(S)
    for i in range(L):
        lo, hi = max(0, half - i), min(S, S + half - i)
        acc[..., lo:hi] += z[..., lo + i - half:hi + i - half] * h[L - 1 - i]
        cnt[lo:hi] += 1
    return acc / cnt


def corr_images(template, source):
    """Zero-mean normalised cross-correlation, valid positions: (hs - ht + 1, ws - wt + 1)."""
    t = np.ascontiguousarray(template, dtype=np.float32)
    s = np.ascontiguousarray(source, dtype=np.float32)
    (th, tw), (sh, sw) = t.shape, s.shape
    out = np.empty((sh - th + 1, sw - tw + 1), dtype=np.float32)
    _ok(lib().orc_corr_images(t.ctypes.data, tw, th, s.ctypes.data, sw, sh, out.ctypes.data), "image sizes")
    return out


def motion_detection(frames, params, threads=0):
    """Block-matching motion maps [frame][grid y][grid x][dx, dy, peak, no-shift peak]."""
    f = np.ascontiguousarray(frames, dtype=np.float32)
    gx, gy = int(params.motion_grid_dims[0]), int(params.motion_grid_dims[1])
    out = np.empty((int(params.frame_count), gy, gx, 4), dtype=np.float32)
    _ok(lib().orc_motion_detection(f.ctypes.data, ctypes.addressof(params), out.ctypes.data, threads),
        "motion parameters")
    return out
