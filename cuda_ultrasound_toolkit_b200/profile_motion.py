"""Runs the motion-detection kernel (and the image-correlation kernels) on the benchmark case,
for profilers.

    python -m cuda_ultrasound_toolkit_b200.profile_motion [--repeat 3] [--corr]

Launch order: `repeat` x (clear of the maps, block_match_kernel); with --corr, then one
corr_images of a 64 x 48 template over a 512 x 512 frame (template statistics, row moments,
tiles). With ncu, select the block-match launches with `-k regex:block_match`.
"""
import argparse

import torch

from . import api, synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--corr", action="store_true")
    args = ap.parse_args()
    frames, p = synth.motion_workload()
    d = torch.from_numpy(frames).cuda()
    maps = torch.empty((p.frame_count, p.motion_grid_dims[1], p.motion_grid_dims[0], 4), device="cuda")
    for _ in range(args.repeat):
        api.motion_detection_device(d, p, out=maps)
    if args.corr:
        api.corr_images_device(d[0, 100:148, 200:264].contiguous(), d[1])
    torch.cuda.synchronize()
    print(f"ok: {args.repeat} block-match launches, {int((maps[..., 2] > 0).sum())} accepted vectors")


if __name__ == "__main__":
    main()
