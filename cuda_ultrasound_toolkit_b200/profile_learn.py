"""Runs the restoration network's kernels on one volume for profiling: three forward passes
(warm-up) followed by one forward pass and one training step.

  python -m cuda_ultrasound_toolkit_b200.profile_learn [--size 128] [--batch 1]
"""
import argparse

import numpy as np
import torch

from . import learn


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--batch", type=int, default=1)
    a = ap.parse_args()
    shape = (a.size, a.size, a.size)
    rng = np.random.default_rng(0)
    vol = (rng.normal(size=(a.batch,) + shape) + 1j * rng.normal(size=(a.batch,) + shape)).astype(np.complex64)
    v = torch.from_numpy(vol).cuda()
    t = v * 0.5
    net = learn.UNet(shape, max_batch=a.batch, seed=1)
    for _ in range(3):
        net.forward(v)
    torch.cuda.synchronize()
    net.forward(v)
    net.train_step(v, t, 1e-4)
    net.check()
    print("ok")


if __name__ == "__main__":
    main()
