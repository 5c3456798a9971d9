#!/usr/bin/env python
"""Generates tests/golden/ncc.npz by running upstream's own motion-detection pipeline on a GPU.

oracle/Makefile.ref (target `ncc`) compiles upstream's ImageProcessor (image_processor.cpp, on
NPP's nppiCrossCorrValid_NormLevel_32f_C1R) and block-match kernels (block_match_kernels.cu,
CUB top-32 selection and quadratic peak fit) unmodified into oracle/_ref/libncc_ref.so, with
oracle/ncc_ref/harness.cu restating the host side of cuda_toolkit::motion_detection and
cuda_toolkit::corr_images (api/cuda_toolkit.cpp:201-329). This script feeds it seeded synthetic
B-mode-like frames (8-bit speckle envelopes, translated by known sub-pixel shifts) and stores
inputs, parameters and upstream's outputs.

Build here (needs the upstream sources and nvcc, no GPU), run where a GPU is:
  make -C oracle -f Makefile.ref REF=/path/to/upstream ncc
  python tests/golden/make_ncc_golden.py --out tests/golden/ncc.npz
"""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cuda_ultrasound_toolkit_b200.params import NccMotionParameters  # noqa: E402
from cuda_ultrasound_toolkit_b200.synth import speckle_frames  # noqa: E402


# (name, image (width, height), per-frame shifts, seed, parameters)
MOTION = [
    ("subpixel_ref0", (96, 80), [(0, 0), (1.6, -0.8), (3.3, -1.5), (-2.4, 2.2)], 11,
     dict(patch_size=16, motion_grid_spacing=16, motion_grid_dims=(6, 5), search_margins=(6, 6),
          abs_cor_threshold=0.3, rel_cor_threshold=0.0, min_patch_variance=0.0, use_subpixel=True,
          reference_frame=0, neighbour_compare=False)),
    ("neighbour_integer", (88, 72), [(0, 0), (1, 0), (2, 1), (3, 1), (4, 2)], 12,
     dict(patch_size=15, motion_grid_spacing=12, motion_grid_dims=(7, 6), search_margins=(4, 3),
          abs_cor_threshold=0.2, rel_cor_threshold=0.02, min_patch_variance=0.05, use_subpixel=False,
          reference_frame=2, neighbour_compare=True)),
    # 49 x 49 correlation map: upstream's peak search sees only its first 2048 values.
    ("wide_search", (112, 112), [(0, 0), (9.5, 7.2), (-12.3, 4.1)], 13,
     dict(patch_size=16, motion_grid_spacing=40, motion_grid_dims=(3, 3), search_margins=(24, 24),
          abs_cor_threshold=0.1, rel_cor_threshold=0.0, min_patch_variance=0.0, use_subpixel=True,
          reference_frame=0, neighbour_compare=False)),
    # 3 x 3 correlation map (fewer than 32 candidates) and strict thresholds.
    ("tiny_search_strict", (64, 64), [(0, 0), (0.4, 0.3), (-0.6, 0.2)], 14,
     dict(patch_size=9, motion_grid_spacing=8, motion_grid_dims=(8, 8), search_margins=(1, 1),
          abs_cor_threshold=0.9, rel_cor_threshold=0.05, min_patch_variance=0.5, use_subpixel=True,
          reference_frame=1, neighbour_compare=False)),
    # Independent frames: weak, often rejected peaks.
    ("uncorrelated", (64, 48), None, 15,
     dict(patch_size=12, motion_grid_spacing=10, motion_grid_dims=(6, 4), search_margins=(5, 5),
          abs_cor_threshold=0.5, rel_cor_threshold=0.1, min_patch_variance=0.1, use_subpixel=True,
          reference_frame=2, neighbour_compare=True)),
]

# (name, template (w, h), source (w, h), seed, kind)
CORR = [
    ("crop_noise", (16, 12), (64, 48), 21, "crop"),
    ("same_size", (20, 14), (20, 14), 22, "crop"),
    ("flat_block", (8, 8), (48, 40), 23, "flat_block"),
    ("flat_template", (6, 5), (40, 32), 24, "flat_template"),
    ("one_pixel", (1, 1), (12, 9), 25, "crop"),
    ("row_template", (17, 1), (64, 8), 26, "crop"),
    ("large", (31, 29), (200, 150), 27, "crop"),
]


def corr_inputs(seed, td, sd, kind):
    rng = np.random.default_rng(seed)
    src = speckle_frames(seed, sd[0], sd[1], [(0, 0)])[0]
    if kind == "flat_block":
        src = src.copy()
        src[12:32, 10:30] = 128
    x0 = int(rng.integers(0, sd[0] - td[0] + 1))
    y0 = int(rng.integers(0, sd[1] - td[1] + 1))
    tpl = src[y0:y0 + td[1], x0:x0 + td[0]].astype(np.int32) + rng.integers(-6, 7, (td[1], td[0]))
    if kind == "flat_template":
        tpl = np.full((td[1], td[0]), 77)
    return np.clip(tpl, 0, 255).astype(np.uint8), src


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ncc.npz"))
    ap.add_argument("--lib", default=os.path.join(ROOT, "oracle", "_ref", "libncc_ref.so"))
    args = ap.parse_args()
    lib = ctypes.CDLL(args.lib)
    f32p = ctypes.POINTER(ctypes.c_float)
    u32p = ctypes.POINTER(ctypes.c_uint)
    lib.ref_motion_detection.argtypes = [f32p, ctypes.POINTER(NccMotionParameters), f32p]
    lib.ref_corr_images.argtypes = [f32p, f32p, u32p, u32p, f32p]
    out = {}
    for name, (w, h), shifts, seed, kw in MOTION:
        if shifts is None:
            frames = np.stack([speckle_frames(seed + 100 * k, w, h, [(0, 0)])[0] for k in range(3)])
        else:
            frames = speckle_frames(seed, w, h, shifts)
        p = NccMotionParameters.make(frame_count=frames.shape[0], image_dims=(w, h), **kw)
        img = np.ascontiguousarray(frames.astype(np.float32))
        gx, gy = kw["motion_grid_dims"]
        maps = np.zeros((frames.shape[0], gy, gx, 4), np.float32)
        rc = lib.ref_motion_detection(img.ctypes.data_as(f32p), ctypes.byref(p), maps.ctypes.data_as(f32p))
        assert rc == 0, name
        out[f"motion/{name}/frames"] = frames
        out[f"motion/{name}/maps"] = maps
        for k, v in p.as_dict().items():
            out[f"motion/{name}/p/{k}"] = np.asarray(v)
        print(name, "valid vectors:", int((maps[..., 2] > 0).sum()), "of", maps[..., 0].size)
    for name, td, sd, seed, kind in CORR:
        tpl, src = corr_inputs(seed, td, sd, kind)
        t = np.ascontiguousarray(tpl.astype(np.float32))
        s = np.ascontiguousarray(src.astype(np.float32))
        corr = np.zeros((sd[1] - td[1] + 1, sd[0] - td[0] + 1), np.float32)
        tdims = (ctypes.c_uint * 2)(*td)
        sdims = (ctypes.c_uint * 2)(*sd)
        rc = lib.ref_corr_images(t.ctypes.data_as(f32p), s.ctypes.data_as(f32p), tdims, sdims,
                                 corr.ctypes.data_as(f32p))
        assert rc == 0, name
        out[f"corr/{name}/template"] = tpl
        out[f"corr/{name}/source"] = src
        out[f"corr/{name}/corr"] = corr
        print(name, "corr range", float(np.nanmin(corr)), float(np.nanmax(corr)), "nan", int(np.isnan(corr).sum()))
    np.savez_compressed(args.out, **out)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
