"""cutb_hilbert_static: the analytic signal for callers that cannot let the library allocate.

Applications that own the GPU memory budget (an acquisition loop that reserves all its buffers
before scanning, a plugin host that lends the library its own buffers) need a call that makes no
device allocation: cudaMalloc/cudaFree can stall on device-wide synchronisation mid-frame, and
they fail once the host has reserved the memory. cutb_hilbert_static keeps its FFT tables in a
fixed device array instead of a plan. This test calls it through the C ABI and checks it against
the plan-based entry point cutb_hilbert and against the FP64 oracle, on calls in a row that rewrite
the shared array with different sizes and filters, up to the longest row the array holds, while the
library's allocator is made to fail every request. The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200 import EncodingMatrix, Plan, lib, synth

pytestmark = pytest.mark.gpu

TOL_HILBERT = 2e-6  # the relative-L2 bar of the other Hilbert parity tests


def _static_entry():
    fn = lib().cutb_hilbert_static
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint, ctypes.c_size_t,
                   ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
    fn.restype = ctypes.c_bool
    return fn


def _plan(S, C, T, taps):
    w = synth.Workload("static", T, C, S, 8, 8, 8, 0, cubic=True, cf=0.0, encoding=EncodingMatrix.NONE)
    bp = synth.make_params(w)
    bp.filter_length = len(taps)
    for i, v in enumerate(taps):
        bp.rf_filter[i] = float(v)
    return Plan(bp)


def test_static_hilbert_matches_plan_entry_point(orc):
    import torch
    fn = _static_entry()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(11)
    # Calls in a row with different lengths, filters and input strides: the longest power-of-two
    # row the array holds (16384), a length that is not a power of two (6000, run padded to 16384)
    # and two shorter ones.
    cases = [(4096, 5, 3, synth.chirp_taps(64), 1), (1024, 4, 2, synth.chirp_taps(17), 2),
             (16384, 3, 1, synth.chirp_taps(64), 1), (6000, 3, 1, synth.chirp_taps(33), 2)]
    prepared = []
    for S, C, T, taps, stride in cases:
        rows = rng.normal(size=(T, C, S)).astype(np.float32)
        d_rows = torch.from_numpy(rows).cuda()
        want = _plan(S, C, T, taps).hilbert(d_rows).cpu().numpy()
        exact = orc.hilbert(rows.astype(np.float64), taps)
        if stride == 2:
            src = torch.zeros((T, C, S, 2), dtype=torch.float32, device="cuda")
            src[..., 0] = d_rows
        else:
            src = d_rows
        out = torch.full((T, C, S), 99 + 99j, dtype=torch.complex64, device="cuda")
        prepared.append((S, C, T, np.ascontiguousarray(taps, dtype=np.float32), stride, src, out, want, exact))
    torch.cuda.synchronize()
    # Every device allocation the library attempts from here on fails: the calls must not need one.
    lib().cutb_debug_fail_allocations_after(0)
    try:
        for S, C, T, t, stride, src, out, want, exact in prepared:
            assert fn(src.data_ptr(), stride, out.data_ptr(), S, T * C, t.ctypes.data, len(t),
                      ctypes.c_void_p(stream.cuda_stream)), lib().cutb_last_error_message()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            err = np.linalg.norm(got - want) / np.linalg.norm(want)
            assert err < TOL_HILBERT, (S, err)
            err = np.linalg.norm(got - exact) / np.linalg.norm(exact)
            assert err < TOL_HILBERT, (S, err)
    finally:
        lib().cutb_debug_fail_allocations_after(-1)


def test_static_hilbert_rejects_rows_beyond_capacity():
    import torch
    fn = _static_entry()
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    assert not fn(buf.data_ptr(), 1, buf.data_ptr(), 32768, 1, None, 0, None)
    assert lib().cutb_last_error() == 1
    # 10000 samples would need a transform of 32768 points: also beyond the fixed tables
    assert not fn(buf.data_ptr(), 1, buf.data_ptr(), 10000, 1, None, 0, None)
    assert lib().cutb_last_error() == 1


def test_static_hilbert_refuses_stream_capture():
    """Its tables are uploaded from host memory that the call frees, so a captured call is refused."""
    import torch
    fn = _static_entry()
    src = torch.zeros(4 * 256, dtype=torch.float32, device="cuda")
    dst = torch.zeros(4 * 256, dtype=torch.complex64, device="cuda")
    graph = torch.cuda.CUDAGraph()
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph, stream=stream):
        ok = fn(src.data_ptr(), 1, dst.data_ptr(), 256, 4, None, 0, ctypes.c_void_p(stream.cuda_stream))
        code = lib().cutb_last_error()
    assert not ok and code == 2  # CUTB_ERR_UNSUPPORTED
    # outside a capture the same call runs
    assert fn(src.data_ptr(), 1, dst.data_ptr(), 256, 4, None, 0, None)
    torch.cuda.synchronize()
