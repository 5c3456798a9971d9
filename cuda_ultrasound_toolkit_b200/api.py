"""Python host mirror of the library's C ABI.

Three layers, all calling libcuda_toolkit_b200.so through ctypes (no CPU fallback: a
missing or unloadable library raises):

* ``beamform`` / ``beamform_i16`` / ``beamform_f32``: host arrays in, host volume out,
  through the upstream-compatible entry points (cuda_toolkit::beamform and the MATLAB
  wrappers; upstream cuda_toolkit/src/api/cuda_toolkit.cpp:109-199,
  cuda_toolkit_matlab.cpp:9-37).
* ``Plan``: the device-resident stages (cutb_decode / cutb_hilbert / cutb_das /
  cutb_beamform) on torch CUDA tensors and the current torch stream.
* ``RfSession``: the buffer-registry front end (init_cuda_configuration ... cuda_hilbert;
  upstream cuda_toolkit_ogl.cpp:105-273), with device tensors standing in for GL buffers.
* ``motion_detection`` / ``corr_images`` (host arrays, cuda_toolkit::motion_detection and
  ::corr_images, cuda_toolkit.cpp:201-329), their MATLAB forms ``motion_detect_f32`` /
  ``corr_images_f32`` and the device forms ``motion_detection_device`` / ``corr_images_device``.
"""
import ctypes
import os

import numpy as np

from .params import CorrImagesParameters, CudaBeamformerParameters, InputDataTypes, MAX_CHANNEL_COUNT, \
    NccMotionParameters

_LIB_NAME = "libcuda_toolkit_b200.so"
_lib = None


class CutbError(RuntimeError):
    """A library call returned false; ``code`` is cutb_last_error()."""

    def __init__(self, what, code, message):
        super().__init__(f"{what} failed (code {code}): {message}")
        self.code = code
        self.message = message


def library_path():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), _LIB_NAME)


def lib():
    """Loads the native library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `make -C {os.path.dirname(path)}`")
    L = ctypes.CDLL(path)
    P = ctypes.POINTER(CudaBeamformerParameters)
    vp, sz, u, b = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint, ctypes.c_bool
    sig = {
        "cutb_last_error": ([], ctypes.c_int),
        "cutb_last_error_message": ([], ctypes.c_char_p),
        "cutb_clear_error": ([], None),
        "cutb_version": ([], ctypes.c_int),
        "cutb_encoding_matrix": ([u, ctypes.c_int, ctypes.POINTER(ctypes.c_int8)], b),
        "cutb_plan_create": ([P, vp], vp),
        "cutb_plan_destroy": ([vp], None),
        "cutb_plan_raw_bytes": ([vp], sz),
        "cutb_plan_iq_bytes": ([vp], sz),
        "cutb_plan_volume_bytes": ([vp], sz),
        "cutb_plan_last_launch_count": ([vp], ctypes.c_int),
        "cutb_decode": ([vp, vp, sz, vp, u, vp], b),
        "cutb_hilbert": ([vp, vp, u, vp, vp], b),
        "cutb_das": ([vp, vp, vp, vp], b),
        "cutb_beamform": ([vp, vp, sz, vp, vp], b),
        "cutb_debug_fail_allocations_after": ([ctypes.c_int], None),
        "cutb_calibrate_fp32": ([ctypes.POINTER(ctypes.c_double), vp], b),
        "cutb_plan_check": ([vp, vp], b),
        "cutb_debug_das_skip_stage": ([vp, ctypes.c_int, ctypes.c_longlong], b),
        "cutb_plan_das_tile_shape": ([vp, ctypes.POINTER(u)], b),
        "cutb_batch_create": ([P, vp, u], vp),
        "cutb_batch_destroy": ([vp], None),
        "cutb_batch_run": ([vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_int, vp], b),
        "cutb_batch_check": ([vp, vp], b),
        "cutb_batch_launches_per_run": ([vp], ctypes.c_int),
        "cutb_batch_das_launches": ([vp], ctypes.c_int),
        "cutb_das_tiles": ([vp, vp, vp, ctypes.POINTER(ctypes.c_int), u, u, vp], b),
        "cutb_das_zslab": ([vp, vp, vp, u, u, vp], b),
        "init_cuda_configuration": ([ctypes.POINTER(u), ctypes.POINTER(u)], b),
        "register_cuda_buffers": ([ctypes.POINTER(u), u, u], b),
        "cuda_set_channel_mapping": ([ctypes.POINTER(ctypes.c_int16)], b),
        "cuda_set_match_filter": ([ctypes.POINTER(ctypes.c_float), u], b),
        "cuda_hilbert": ([u, u], b),
        "cuda_decode": ([sz, u], b),
        "deinit_cuda_configuration": ([], None),
        "cuda_register_device_buffer": ([u, vp, sz], b),
        "beamform_i16_matlab": ([vp, CudaBeamformerParameters, vp], None),
        "beamform_f32_matlab": ([vp, CudaBeamformerParameters, vp], None),
        "motion_detect_f32_matlab": ([vp, NccMotionParameters, vp], None),
        "corr_images_f32_matlab": ([vp, vp, CorrImagesParameters, vp], None),
        "cutb_motion_detection": ([vp, ctypes.POINTER(NccMotionParameters), vp, vp], b),
        "cutb_corr_images": ([vp, vp, ctypes.POINTER(u), ctypes.POINTER(u), vp, vp], b),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    # cuda_toolkit::beamform(std::span<const u8>, std::span<u8>, const CudaBeamformerParameters&):
    # on x86-64 SysV each span (pointer, size) travels in two integer registers.
    cxx = getattr(L, "_ZN12cuda_toolkit8beamformESt4spanIKhLm18446744073709551615EES0_IhLm18446744073709551615EERK24CudaBeamformerParameters")
    cxx.argtypes = [vp, sz, vp, sz, P]
    cxx.restype = b
    L.cxx_beamform = cxx
    # cuda_toolkit::motion_detection(span<const u8>, span<u8>, const NccMotionParameters&) and
    # cuda_toolkit::corr_images(span<const float>, span<const float>, span<float>, const uint*, const uint*)
    mot = getattr(L, "_ZN12cuda_toolkit16motion_detectionESt4spanIKhLm18446744073709551615EES0_IhLm18446744073709551615EERK19NccMotionParameters")
    mot.argtypes = [vp, sz, vp, sz, ctypes.POINTER(NccMotionParameters)]
    mot.restype = b
    L.cxx_motion_detection = mot
    cor = getattr(L, "_ZN12cuda_toolkit11corr_imagesESt4spanIKfLm18446744073709551615EES2_S0_IfLm18446744073709551615EEPKjS5_")
    cor.argtypes = [vp, sz, vp, sz, vp, sz, ctypes.POINTER(u), ctypes.POINTER(u)]
    cor.restype = b
    L.cxx_corr_images = cor
    _lib = L
    return L


def last_error():
    L = lib()
    return L.cutb_last_error(), L.cutb_last_error_message().decode(errors="replace")


def _check(ok, what):
    if not ok:
        code, msg = last_error()
        raise CutbError(what, code, msg)


def encoding_matrix(n, ordering=1):
    """Order-n transmit encoding matrix (+1/-1 int8, rows in output order)."""
    out = np.empty((n, n), dtype=np.int8)
    _check(lib().cutb_encoding_matrix(n, ordering, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))),
           "cutb_encoding_matrix")
    return out


def calibrate_fp32(stream=None):
    """Measured FP32 FMA throughput of the current device, TFLOP/s."""
    v = ctypes.c_double()
    _check(lib().cutb_calibrate_fp32(ctypes.byref(v), _stream_handle(stream)), "cutb_calibrate_fp32")
    return v.value


# ---- host-span entry points --------------------------------------------------------------------
def beamform(raw, bp: CudaBeamformerParameters, out=None):
    """cuda_toolkit::beamform on host arrays; returns the complex64 volume [Z][Y][X]."""
    raw = np.ascontiguousarray(raw)
    if out is None:
        out = np.empty(bp.volume_shape, dtype=np.complex64)
    _check(lib().cxx_beamform(raw.ctypes.data, raw.nbytes, out.ctypes.data, out.nbytes, ctypes.byref(bp)),
           "cuda_toolkit::beamform")
    return out


def beamform_i16(raw, bp, out=None):
    """beamform_i16_matlab (errors are only logged upstream; here they raise)."""
    raw = np.ascontiguousarray(raw, dtype=np.int16)
    if out is None:
        out = np.empty(bp.volume_shape, dtype=np.complex64)
    lib().cutb_clear_error()
    lib().beamform_i16_matlab(raw.ctypes.data, bp, out.ctypes.data)
    code, msg = last_error()
    if code:
        raise CutbError("beamform_i16_matlab", code, msg)
    return out


def beamform_f32(raw, bp, out=None):
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    if out is None:
        out = np.empty(bp.volume_shape, dtype=np.complex64)
    lib().cutb_clear_error()
    lib().beamform_f32_matlab(raw.ctypes.data, bp, out.ctypes.data)
    code, msg = last_error()
    if code:
        raise CutbError("beamform_f32_matlab", code, msg)
    return out


# ---- image correlation and motion detection ------------------------------------------------------
def _maps_shape(params):
    return (int(params.frame_count), int(params.motion_grid_dims[1]), int(params.motion_grid_dims[0]), 4)


def _corr_shape(template, source):
    (th, tw), (sh, sw) = template.shape, source.shape
    return (max(sh - th + 1, 0), max(sw - tw + 1, 0))


def motion_detection(frames, params: NccMotionParameters, out=None):
    """cuda_toolkit::motion_detection on host frames [F][H][W] (float32); returns the motion maps
    [F][grid y][grid x][dx, dy, peak, no-shift peak]."""
    frames = np.ascontiguousarray(frames, dtype=np.float32)
    if out is None:
        out = np.empty(_maps_shape(params), dtype=np.float32)
    _check(lib().cxx_motion_detection(frames.ctypes.data, frames.nbytes, out.ctypes.data, out.nbytes,
                                      ctypes.byref(params)), "cuda_toolkit::motion_detection")
    return out


def motion_detect_f32(frames, params: NccMotionParameters, out=None):
    """motion_detect_f32_matlab (errors are only logged upstream; here they raise)."""
    frames = np.ascontiguousarray(frames, dtype=np.float32)
    if out is None:
        out = np.empty(_maps_shape(params), dtype=np.float32)
    lib().cutb_clear_error()
    lib().motion_detect_f32_matlab(frames.ctypes.data, params, out.ctypes.data)
    code, msg = last_error()
    if code:
        raise CutbError("motion_detect_f32_matlab", code, msg)
    return out


def corr_images(template, source, out=None, dims=None):
    """cuda_toolkit::corr_images on host images [H][W]; returns the valid correlation map.
    ``dims`` = ((tw, th), (sw, sh)) overrides the sizes passed (spans keep the arrays' sizes)."""
    t = np.ascontiguousarray(template, dtype=np.float32)
    s = np.ascontiguousarray(source, dtype=np.float32)
    (tw, th), (sw, sh) = dims if dims is not None else ((t.shape[1], t.shape[0]), (s.shape[1], s.shape[0]))
    if out is None:
        out = np.empty((max(sh - th + 1, 0), max(sw - tw + 1, 0)), dtype=np.float32)
    td = (ctypes.c_uint * 2)(tw, th)
    sd = (ctypes.c_uint * 2)(sw, sh)
    _check(lib().cxx_corr_images(t.ctypes.data, t.size, s.ctypes.data, s.size, out.ctypes.data, out.size, td, sd),
           "cuda_toolkit::corr_images")
    return out


def corr_images_f32(template, source, out=None):
    """corr_images_f32_matlab (errors raise here)."""
    t = np.ascontiguousarray(template, dtype=np.float32)
    s = np.ascontiguousarray(source, dtype=np.float32)
    p = CorrImagesParameters()
    p.template_dims[0], p.template_dims[1] = t.shape[1], t.shape[0]
    p.source_dims[0], p.source_dims[1] = s.shape[1], s.shape[0]
    if out is None:
        out = np.empty(_corr_shape(t, s), dtype=np.float32)
    lib().cutb_clear_error()
    lib().corr_images_f32_matlab(t.ctypes.data, s.ctypes.data, p, out.ctypes.data)
    code, msg = last_error()
    if code:
        raise CutbError("corr_images_f32_matlab", code, msg)
    return out


def motion_detection_device(frames, params: NccMotionParameters, out=None, stream=None):
    """cutb_motion_detection on a CUDA float32 tensor [F][H][W]; asynchronous on `stream`."""
    import torch
    assert frames.is_cuda and frames.dtype == torch.float32 and frames.is_contiguous()
    if out is None:
        out = torch.empty(_maps_shape(params), dtype=torch.float32, device=frames.device)
    _check(lib().cutb_motion_detection(frames.data_ptr(), ctypes.byref(params), out.data_ptr(),
                                       _stream_handle(stream)), "cutb_motion_detection")
    return out


def corr_images_device(template, source, out=None, stream=None):
    """cutb_corr_images on CUDA float32 tensors [H][W]; asynchronous on `stream`."""
    import torch
    assert template.is_cuda and source.is_cuda and template.dtype == source.dtype == torch.float32
    template, source = template.contiguous(), source.contiguous()
    if out is None:
        out = torch.empty(_corr_shape(template, source), dtype=torch.float32, device=source.device)
    td = (ctypes.c_uint * 2)(template.shape[1], template.shape[0])
    sd = (ctypes.c_uint * 2)(source.shape[1], source.shape[0])
    _check(lib().cutb_corr_images(template.data_ptr(), source.data_ptr(), td, sd, out.data_ptr(),
                                  _stream_handle(stream)), "cutb_corr_images")
    return out


# ---- device-resident stages ----------------------------------------------------------------------
class _Options(ctypes.Structure):
    _fields_ = [("iq_bf16", ctypes.c_int), ("das_tile", ctypes.c_int), ("decode_tc", ctypes.c_int),
                ("das_schedule", ctypes.c_int), ("das_rows_per_stage", ctypes.c_int), ("reserved", ctypes.c_int * 11)]


def _stream_handle(stream):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Plan:
    """cutb_plan over torch CUDA tensors. Stage calls are asynchronous on `stream`
    (default: the current torch stream)."""

    def __init__(self, bp: CudaBeamformerParameters, iq_bf16=False, das_tile=0, decode_tc=False, das_schedule=0,
                 das_rows_per_stage=0):
        import torch  # noqa: F401  (device memory comes from torch)
        self.bp = bp.copy()
        opts = _Options(int(iq_bf16), int(das_tile), int(decode_tc), int(das_schedule), int(das_rows_per_stage))
        self._L = lib()
        self._h = self._L.cutb_plan_create(ctypes.byref(self.bp), ctypes.byref(opts))
        _check(self._h, "cutb_plan_create")
        self.iq_bf16 = bool(iq_bf16)
        self.raw_bytes = lib().cutb_plan_raw_bytes(self._h)
        self.iq_bytes = lib().cutb_plan_iq_bytes(self._h)
        self.volume_bytes = lib().cutb_plan_volume_bytes(self._h)

    def close(self):
        # _L is bound at construction: at interpreter exit the module globals may be gone.
        if getattr(self, "_h", None):
            self._L.cutb_plan_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def launches(self):
        return lib().cutb_plan_last_launch_count(self._h)

    # Allocation helpers -------------------------------------------------------------------------
    def empty_decoded(self, out_stride=1):
        """Decoded rows: S samples, or the 2 S reals of the IQ pairs of a bandpass plan."""
        import torch
        S, C, T = self.bp.dims
        if self.bp.sample_type == 1:  # SAMPLE_BANDPASS
            S *= 2
        return torch.empty((T, C, S * out_stride), dtype=torch.float32, device="cuda")

    def empty_iq(self):
        import torch
        S, C, T = self.bp.dims
        if self.iq_bf16:
            return torch.empty((T, C, S, 2), dtype=torch.bfloat16, device="cuda")
        return torch.empty((T, C, S), dtype=torch.complex64, device="cuda")

    def empty_volume(self):
        import torch
        return torch.empty(self.bp.volume_shape, dtype=torch.complex64, device="cuda")

    # Stages ------------------------------------------------------------------------------------
    def decode(self, raw, out=None, out_stride=1, stream=None):
        out = self.empty_decoded(out_stride) if out is None else out
        _check(lib().cutb_decode(self._h, raw.data_ptr(), raw.numel() * raw.element_size(), out.data_ptr(),
                                 out_stride, _stream_handle(stream)), "cutb_decode")
        return out

    def hilbert(self, decoded, in_stride=1, out=None, stream=None):
        out = self.empty_iq() if out is None else out
        _check(lib().cutb_hilbert(self._h, decoded.data_ptr(), in_stride, out.data_ptr(), _stream_handle(stream)),
               "cutb_hilbert")
        return out

    def das(self, iq, out=None, stream=None):
        out = self.empty_volume() if out is None else out
        _check(lib().cutb_das(self._h, iq.data_ptr(), out.data_ptr(), _stream_handle(stream)), "cutb_das")
        return out

    @property
    def tile_shape(self):
        """(x, y, z) voxels of a delay-and-sum tile."""
        shape = (ctypes.c_uint * 3)()
        _check(lib().cutb_plan_das_tile_shape(self._h, shape), "cutb_plan_das_tile_shape")
        return tuple(shape)

    def das_zslab(self, iq, z0, z1, out=None, stream=None):
        """Delay-and-sum of the z-planes z0 .. z1 - 1 into a [z1 - z0][Y][X] slab (cutb_das_zslab)."""
        import torch
        z, y, x = self.bp.volume_shape
        if out is None:
            out = torch.empty((z1 - z0, y, x), dtype=torch.complex64, device="cuda")
        _check(lib().cutb_das_zslab(self._h, iq.data_ptr(), out.data_ptr(), int(z0), int(z1), _stream_handle(stream)),
               "cutb_das_zslab")
        return out

    def das_tiles(self, iq, tiles, splits=1, out=None, stream=None):
        """Delay-and-sum of the listed tile ids only (others zero), stages split over `splits` CTAs."""
        out = self.empty_volume() if out is None else out
        t = np.ascontiguousarray(tiles, dtype=np.int32)
        _check(lib().cutb_das_tiles(self._h, iq.data_ptr(), out.data_ptr(), t.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    t.size, splits, _stream_handle(stream)), "cutb_das_tiles")
        return out

    def check(self, stream=None):
        """Synchronises the stream; raises if a device-side bounded wait gave up."""
        _check(lib().cutb_plan_check(self._h, _stream_handle(stream)), "cutb_plan_check")

    def debug_skip_stage(self, stage, wait_limit_cycles=0):
        """Test hook: the delay-and-sum never issues stage `stage` (-1: off), so its bounded wait
        runs out after `wait_limit_cycles` (0: the default limit)."""
        _check(lib().cutb_debug_das_skip_stage(self._h, int(stage), int(wait_limit_cycles)),
               "cutb_debug_das_skip_stage")

    def beamform(self, raw, out=None, stream=None):
        out = self.empty_volume() if out is None else out
        _check(lib().cutb_beamform(self._h, raw.data_ptr(), raw.numel() * raw.element_size(), out.data_ptr(),
                                   _stream_handle(stream)), "cutb_beamform")
        return out


class Batch:
    """cutb_batch: many frames of uneven size beamformed with one persistent delay-and-sum launch
    per kernel variant, optionally replayed from a captured CUDA graph."""

    def __init__(self, params, das_tiles=None):
        n = len(params)
        self._bps = (CudaBeamformerParameters * n)(*[bp.copy() for bp in params])
        opts = None
        if das_tiles is not None:
            opts = (_Options * n)(*[_Options(0, int(t), 0) for t in das_tiles])
        self._L = lib()
        self._h = self._L.cutb_batch_create(self._bps, opts, n)
        _check(self._h, "cutb_batch_create")
        self.n = n
        self.shapes = [bp.volume_shape for bp in params]

    def close(self):
        if getattr(self, "_h", None):
            self._L.cutb_batch_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def launches_per_run(self):
        return lib().cutb_batch_launches_per_run(self._h)

    @property
    def das_launches(self):
        return lib().cutb_batch_das_launches(self._h)

    def empty_volumes(self):
        import torch
        return [torch.empty(s, dtype=torch.complex64, device="cuda") for s in self.shapes]

    def run(self, raws, volumes=None, graph=False, stream=None):
        volumes = self.empty_volumes() if volumes is None else volumes
        assert len(raws) == self.n and len(volumes) == self.n
        rp = (ctypes.c_void_p * self.n)(*[r.data_ptr() for r in raws])
        vp_ = (ctypes.c_void_p * self.n)(*[v.data_ptr() for v in volumes])
        _check(lib().cutb_batch_run(self._h, rp, vp_, int(graph), _stream_handle(stream)), "cutb_batch_run")
        return volumes

    def check(self, stream=None):
        _check(lib().cutb_batch_check(self._h, _stream_handle(stream)), "cutb_batch_check")


# ---- buffer-registry front end ------------------------------------------------------------------
class RfSession:
    """init_cuda_configuration / register_cuda_buffers / cuda_decode / cuda_hilbert with torch
    tensors registered as the 'GL buffers' (ids are assigned here)."""

    def __init__(self, raw_dims, dec_dims):
        L = lib()
        self._ids = {}
        self._next = 1
        _check(L.init_cuda_configuration((ctypes.c_uint * 2)(*raw_dims), (ctypes.c_uint * 3)(*dec_dims)),
               "init_cuda_configuration")

    def register(self, tensor):
        bid = self._next
        self._next += 1
        _check(lib().cuda_register_device_buffer(bid, tensor.data_ptr(), tensor.numel() * tensor.element_size()),
               "cuda_register_device_buffer")
        self._ids[bid] = tensor
        return bid

    def register_buffers(self, rf_ids, raw_id):
        _check(lib().register_cuda_buffers((ctypes.c_uint * max(1, len(rf_ids)))(*rf_ids), len(rf_ids), raw_id),
               "register_cuda_buffers")

    def set_channel_mapping(self, mapping):
        m = np.zeros(MAX_CHANNEL_COUNT, dtype=np.int16)
        m[: len(mapping)] = mapping
        _check(lib().cuda_set_channel_mapping(m.ctypes.data_as(ctypes.POINTER(ctypes.c_int16))),
               "cuda_set_channel_mapping")

    def set_match_filter(self, taps):
        taps = np.ascontiguousarray(taps, dtype=np.float32)
        _check(lib().cuda_set_match_filter(taps.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(taps)),
               "cuda_set_match_filter")

    def decode(self, input_offset, out_idx):
        _check(lib().cuda_decode(input_offset, out_idx), "cuda_decode")

    def hilbert(self, in_idx, out_idx):
        _check(lib().cuda_hilbert(in_idx, out_idx), "cuda_hilbert")

    def close(self):
        lib().deinit_cuda_configuration()
        self._ids.clear()
