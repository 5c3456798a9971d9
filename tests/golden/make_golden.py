#!/usr/bin/env python
"""Generates the golden fixtures in this directory by running the upstream toolkit's own code.

The upstream sources are compiled, unmodified, for the CPU by oracle/Makefile.ref (CUDA runtime,
cuBLAS, cuFFT and GL interop are emulated on the host by oracle/ref_shim/). This script feeds
that build seeded synthetic inputs through upstream's entry points and stores inputs + outputs:

  encoding_matrices.npz  every supported encoding order (HADAMARD and WALSH), from
                         HadamardDecoder::generate_hadamard (hadamard_decoder.cpp:110-222)
  frontend.npz           cuda_decode + cuda_hilbert outputs (cuda_toolkit_ogl.cpp:192-273)
  volumes.npz            beamform_i16_matlab volumes (cuda_toolkit_matlab.cpp:9-22) for HERCULES,
                         FORCES, TPW and UFORCES parameter sets
  bandpass.npz           RfProcessor::convert_demod (rf_processor.cpp:225-246) on bandpass IQ pairs

Run from the repository root (needs the upstream sources and a C++ compiler, no GPU):
  make -C oracle -f Makefile.ref REF=/path/to/upstream && python tests/golden/make_golden.py
"""
import ctypes
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cuda_ultrasound_toolkit_b200 import synth  # noqa: E402
from cuda_ultrasound_toolkit_b200.params import ApoType, EncodingMatrix, SequenceId  # noqa: E402
from oracle import ref  # noqa: E402

ORDERS = [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 12, 24, 48, 96, 192, 384, 768, 20, 40, 80, 160, 320, 640]

# Front-end cases: (name, T, C, S, raw padding, extra raw channels, filter taps, seed)
FRONTEND = [
    ("t16_c6_s128", 16, 6, 128, 0, 0, 0, 1),
    ("t8_c4_s256_pad_filter", 8, 4, 256, 13, 3, 32, 2),
    ("t12_c4_s64_base12", 12, 4, 64, 0, 0, 16, 3),
    ("t20_c3_s64_base20", 20, 3, 64, 5, 1, 0, 4),
    # sample counts that are not powers of two (upstream's cuFFT plans any length)
    ("t4_c3_s100_filter", 4, 3, 100, 0, 0, 16, 5),
    ("t8_c2_s2500_pad_filter", 8, 2, 2500, 3, 1, 64, 6),
    ("t12_c2_s3072", 12, 2, 3072, 0, 0, 0, 7),
    ("t4_c2_s6000_filter", 4, 2, 6000, 0, 0, 64, 8),
]

# Delay-and-sum cases on one small frame (T=8, C=8, S=512, volume 12 x 6 x 20). Upstream always
# interpolates cubically and never applies the coherence factor in HERCULES, so these cases use
# interpolate=True and, for HERCULES, coherency_weighting=0.
VOLUMES = [
    ("hercules_plane", dict()),
    ("hercules_focus", dict(focus_z=9e-3)),
    ("hercules_time_offset", dict(time_offset=1.5e-7)),
    ("hercules_fn_rx", dict(fn_rx=1.0)),
    ("hercules_rx_to_sin", dict(apo=ApoType.RX_TO_SIN)),
    ("hercules_readi_hadamard", dict(readi=2, readi_id=1)),
    ("hercules_readi_walsh", dict(readi=4, readi_id=2, decode=EncodingMatrix.WALSH)),
    ("forces_rx_hann", dict(seq=SequenceId.FORCES, cf=0.5)),
    ("forces_fn", dict(seq=SequenceId.FORCES, fn_rx=1.0, fn_tx=1.5, cf=1.0)),
    ("forces_tx_to_sin", dict(seq=SequenceId.FORCES, apo=ApoType.TX_TO_SIN)),
    ("forces_both_to_sin", dict(seq=SequenceId.FORCES, apo=ApoType.BOTH_TO_SIN, cf=0.3)),
    ("forces_readi", dict(seq=SequenceId.FORCES, readi=2, readi_id=1)),
    # Tilted plane waves (angles in foci[t][2]): a YZ plane (transmit rows, receive columns) and
    # an XZ plane (same orientation).
    ("tpw_yz", dict(seq=SequenceId.RCA_TPW, angles=np.linspace(-0.15, 0.15, 8), fn_rx=1.0, cf=0.5)),
    ("tpw_xz", dict(seq=SequenceId.RCA_TPW, angles=np.linspace(-0.1, 0.2, 8), same_orientation=True, cf=1.0)),
    # UFORCES (focused, same orientation, sparse transmit elements). X * Y is a multiple of the
    # upstream kernel's 128-thread block: its `> X * Y` guard writes one voxel past a slice otherwise.
    ("uforces", dict(seq=SequenceId.UFORCES, same_orientation=True, focus_z=25e-3, elems=[0, 1, 3, 4, 6, 7, 9, 10],
                     fn_rx=1.0, cf=0.5, X=16, Y=8)),
    ("uforces_dense", dict(seq=SequenceId.UFORCES, same_orientation=True, focus_z=30e-3, elems=list(range(8)), cf=1.0,
                           X=16, Y=8)),
]


def volume_params(cmap, seq=SequenceId.HERCULES, cf=0.0, fn_rx=0.0, fn_tx=0.0, apo=ApoType.RX_HANN, readi=0,
                  readi_id=0, decode=EncodingMatrix.HADAMARD, focus_z=math.inf, time_offset=0.0, angles=None,
                  same_orientation=False, elems=None, X=12, Y=6):
    w = synth.Workload("golden", 8, 8, 512, X, Y, 20, 0, cubic=True, cf=cf, encoding=decode,
                       box_xy=1.5e-3, z_range=(4e-3, 16e-3))
    bp = synth.make_params(w, channel_map=cmap)
    if same_orientation:
        bp.tx_orientation = bp.rx_orientation
    if angles is not None:
        for t, a in enumerate(angles):
            bp.foci[3 * t + 2] = float(a)
    if elems is not None:
        for t, e in enumerate(elems):
            bp.sparse_elements[t] = int(e)
    bp.das_shader_id = int(seq)
    bp.fn_rx, bp.fn_tx = fn_rx, fn_tx
    bp.apo_type = int(apo)
    bp.to_power = 2
    bp.readi_group_count, bp.readi_group_id = readi, readi_id
    if angles is None:
        bp.foci[2] = focus_z
    bp.time_offset = time_offset
    return bp


def main():
    if not ref.available():
        sys.exit("oracle/_ref/libcuda_toolkit_ref.so is missing: run make -C oracle -f Makefile.ref first")

    mats = {}
    for n in ORDERS:
        for ordering in (EncodingMatrix.HADAMARD, EncodingMatrix.WALSH):
            mats[f"n{n}_o{int(ordering)}"] = ref.encoding_matrix(n, int(ordering)).astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "encoding_matrices.npz"), **mats)

    fe = {}
    for name, T, C, S, pad, extra, ntaps, seed in FRONTEND:
        rng = np.random.default_rng(seed)
        R1 = C + extra
        raw = rng.integers(-32768, 32768, size=(R1, T * S + pad), dtype=np.int16)
        cmap = rng.permutation(R1)[:C].astype(np.int16)
        w = synth.Workload(name, T, C, S, 4, 4, 4, 0, cubic=True, cf=0.0)
        bp = synth.make_params(w, channel_map=cmap, raw_padding=pad)
        bp.rf_raw_dim[1] = R1
        taps = synth.chirp_taps(ntaps) if ntaps else None
        dec, iq = ref.decode_and_hilbert(raw, bp, taps)
        fe[f"{name}.raw"] = raw
        fe[f"{name}.params"] = np.frombuffer(bytes(bp), np.uint8)
        fe[f"{name}.taps"] = np.zeros(0, np.float32) if taps is None else taps
        fe[f"{name}.decoded"] = dec
        fe[f"{name}.iq"] = iq
    np.savez_compressed(os.path.join(HERE, "frontend.npz"), **fe)

    w = synth.Workload("golden", 8, 8, 512, 12, 6, 20, 6, cubic=True, cf=0.0, box_xy=1.5e-3,
                       z_range=(4e-3, 16e-3))
    raw, cmap, _, _ = synth.synth_frame(w, 77)
    vols = {"raw": raw}
    for name, kw in VOLUMES:
        bp = volume_params(cmap, **kw)
        vols[f"{name}.params"] = np.frombuffer(bytes(bp), np.uint8)
        vols[f"{name}.volume"] = ref.beamform(raw, bp)
    np.savez_compressed(os.path.join(HERE, "volumes.npz"), **vols)

    # Bandpass IQ pairs through upstream's RfProcessor::convert_demod (no upstream entry point
    # calls it): int16 and f32 input, with and without the time-domain filter.
    bpd = {}
    for name, dtype, ntaps, seed in (("i16_nofilter", np.int16, 0, 11), ("i16_filter", np.int16, 16, 12),
                                     ("f32_filter", np.float32, 9, 13)):
        rng = np.random.default_rng(seed)
        T, C, S, pad, extra = 8, 6, 256, 6, 2
        w = synth.Workload(name, T, C, S, 8, 8, 8, 0, cubic=True, cf=0.0, encoding=EncodingMatrix.NONE)
        cmap = rng.permutation(C + extra)[:C].astype(np.int16)
        bp = synth.make_params(w, channel_map=cmap, raw_padding=pad + T * S)
        bp.rf_raw_dim[1] = C + extra
        bp.sample_type = 1
        if dtype == np.int16:
            raw = rng.integers(-32768, 32768, size=(C + extra, 2 * T * S + pad), dtype=np.int16)
        else:
            bp.data_type = 2
            raw = rng.normal(0, 1000, size=(C + extra, 2 * T * S + pad)).astype(np.float32)
        taps = synth.chirp_taps(ntaps) if ntaps else np.zeros(0, np.float32)
        bp.filter_length = ntaps  # the parameter block carries the filter the plan applies
        for i, v in enumerate(taps):
            bp.rf_filter[i] = float(v)
        bpd[f"{name}.raw"] = raw
        bpd[f"{name}.params"] = np.frombuffer(bytes(bp), np.uint8)
        bpd[f"{name}.taps"] = taps
        bpd[f"{name}.iq"] = ref.convert_demod(raw, bp, bp.center_frequency, bp.sampling_frequency,
                                              taps if ntaps else None)
    np.savez_compressed(os.path.join(HERE, "bandpass.npz"), **bpd)
    for f in ("encoding_matrices.npz", "frontend.npz", "volumes.npz", "bandpass.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
