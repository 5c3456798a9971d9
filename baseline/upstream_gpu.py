#!/usr/bin/env python
"""Times upstream's own CUDA build (baseline/_ref/libcuda_toolkit_upstream.so, built by
baseline/Makefile from the upstream sources for sm_100a) through its public entry point
cuda_toolkit::beamform(span<const u8>, span<u8>, const CudaBeamformerParameters&) on host
buffers, the only API upstream has (cuda_toolkit/src/api/cuda_toolkit.cpp:109-199).

Measurement infrastructure, run by bench.py in a child process so that upstream's stdout
chatter, its process-wide singletons and its own CUDA runtime stay out of the benchmark's
process. Usage:

  python baseline/upstream_gpu.py <dir>    # reads <dir>/raw.npy, <dir>/params.bin; writes
                                           # <dir>/volume.npy and prints one JSON line

Before the first call the input is checked on the host against the one out-of-bounds read the
upstream kernel can make: its cubic interpolation reads sample i + 2 of the row at the clamp
index i = S - 2, i.e. sample S, which is past the end of the analytic-signal buffer for the last
row (beamformer_utils.cuh:99-125 with the clamp at templated_beamformer.cuh:184-188). The largest
delay of the volume, over its corners and the aperture's corners, is computed in FP64, and the
run is refused unless every index stays below S - 3.
"""
import ctypes
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "_ref", "libcuda_toolkit_upstream.so")
SYMBOL = ("_ZN12cuda_toolkit8beamformESt4spanIKhLm18446744073709551615EES0_"
          "IhLm18446744073709551615EERK24CudaBeamformerParameters")


def max_sample_index(bp):
    """Upper bound (FP64) on upstream's HERCULES plane-wave sample index over the volume: the
    largest transmit + receive path, at the volume's and the aperture's corners (the path is
    convex in the voxel and in the element position, so its maximum is at a corner)."""
    spm = bp.sampling_frequency / bp.speed_of_sound
    px, py = bp.xdc_element_pitch[0], bp.xdc_element_pitch[1]
    ex = (-bp.xdc_transform[12] + px / 2, bp.xdc_transform[12] - px / 2)
    ey = (-bp.xdc_transform[13] + py / 2, bp.xdc_transform[13] - py / 2)
    vx = (bp.output_min_coordinate[0], bp.output_max_coordinate[0])
    # upstream reuses the x step for y (beamformer.cu:39-49)
    ny = int(bp.output_points[1])
    res_x = (vx[1] - vx[0]) / max(int(bp.output_points[0]) - 1, 1)
    vy = (bp.output_min_coordinate[1], bp.output_min_coordinate[1] + res_x * max(ny - 1, 0))
    vz = (bp.output_min_coordinate[2], bp.output_max_coordinate[2])
    worst = 0.0
    for x in vx:
        for y in vy:
            for z in vz:
                for e in ex:
                    for f in ey:
                        worst = max(worst, abs(z) + math.sqrt((e - x) ** 2 + (f - y) ** 2 + z * z))
    return worst * spm + int(bp.time_offset * bp.sampling_frequency)


def main():
    sys.path.insert(0, ROOT)
    from cuda_ultrasound_toolkit_b200.params import CudaBeamformerParameters
    d = sys.argv[1]
    reps = int(sys.argv[2]) if len(sys.argv) > 2 else 3
    raw = np.load(os.path.join(d, "raw.npy"))
    with open(os.path.join(d, "params.bin"), "rb") as f:
        bp = CudaBeamformerParameters.from_buffer_copy(f.read())
    S = int(bp.dec_data_dim[0])
    top = max_sample_index(bp)
    if not (bp.das_shader_id == 2 and math.isinf(bp.foci[2]) and top < S - 3):
        print(json.dumps({"refused": f"largest sample index {top:.1f} not below S - 3 = {S - 3}, or not a "
                                     "HERCULES plane wave"}))
        return
    L = ctypes.CDLL(LIB)
    fn = getattr(L, SYMBOL)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                   ctypes.POINTER(CudaBeamformerParameters)]
    fn.restype = ctypes.c_bool
    z, y, x = int(bp.output_points[2]), int(bp.output_points[1]), int(bp.output_points[0])
    vol = np.zeros((z, y, x), np.complex64)
    raw = np.ascontiguousarray(raw)

    def call():
        return fn(raw.ctypes.data, raw.nbytes, vol.ctypes.data, vol.nbytes, ctypes.byref(bp))

    # upstream prints progress on stdout: keep it off this process's JSON line
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        ok = call()  # first call: allocations, cuFFT/cuBLAS plans
        times = []
        for _ in range(reps):
            t = time.perf_counter()
            ok = call() and ok
            times.append(time.perf_counter() - t)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    np.save(os.path.join(d, "volume.npy"), vol)
    ms = 1e3 * float(np.median(times))
    print(json.dumps({"ok": bool(ok), "ms": ms, "volumes_per_s": 1e3 / ms, "reps": reps,
                      "max_sample_index": top, "api": "upstream cuda_toolkit::beamform (host spans)"}))


if __name__ == "__main__":
    main()
