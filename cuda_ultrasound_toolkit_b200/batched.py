"""The batched form: a seeded stream of frames of mixed size, beamformed together by cutb_batch
(every frame's front end, then one persistent delay-and-sum launch per kernel variant, replayed
from a captured CUDA graph), with delay-and-sum tile shapes chosen by the autotuner (tune.py).

Frame mix (seeded): transmits in {32, 64, 128} with a matching order Hadamard code, receive
channels in {64, 128}, samples in {1024, 2048, 4096, 8192}, output volumes in {64^3,
128 x 128 x 128, 128 x 128 x 256}, 20-300 point scatterers per frame. Every frame is HERCULES
plane-wave, cubic interpolation with coherence factor. The lateral box is 70 % of the smaller
aperture half-width (at most 9 mm); the depth range starts at 8 mm and ends where the longest
round trip still fits the frame's samples (at most 40 mm). Frames are simulated on the GPU.
"""
import math

import numpy as np
import torch

from . import synth
from .simulate import Simulator

TRANSMITS = (32, 64, 128)
CHANNELS = (64, 128)
SAMPLES = (1024, 2048, 4096, 8192)
VOLUMES = ((64, 64, 64), (128, 128, 128), (256, 128, 128))  # Z, Y, X


def frame_specs(seed, n=64):
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n):
        Z, Y, X = VOLUMES[rng.integers(len(VOLUMES))]
        specs.append(dict(T=int(rng.choice(TRANSMITS)), C=int(rng.choice(CHANNELS)), S=int(rng.choice(SAMPLES)),
                          X=X, Y=Y, Z=Z, scatterers=int(rng.integers(20, 301)), seed=seed * 1000 + k))
    return specs


def depth_limit(spec, margin=40):
    """Largest depth whose round trip from the box corner still fits the samples (metres)."""
    spm = synth.FS / synth.C_SOUND
    reach = (spec["S"] - margin) / spm
    hx, hy = spec["C"] * synth.PITCH / 2, spec["T"] * synth.PITCH / 2
    # z + sqrt(hx^2 + hy^2 + z^2) = reach  ->  z = (reach^2 - hx^2 - hy^2) / (2 reach)
    return min(40e-3, (reach * reach - hx * hx - hy * hy) / (2 * reach))


def workload(spec):
    box = min(9e-3, 0.7 * min(spec["T"], spec["C"]) * synth.PITCH / 2)
    return synth.Workload("batched", spec["T"], spec["C"], spec["S"], spec["X"], spec["Y"], spec["Z"],
                          spec["scatterers"], cubic=True, cf=1.0, box_xy=box, z_range=(8e-3, depth_limit(spec)))


def make_frames(specs):
    """[(raw int16 CUDA tensor, params)] simulated on the GPU."""
    sims = {}
    frames = []
    for spec in specs:
        w = workload(spec)
        key = (w.T, w.C, w.S)
        if key not in sims:
            sims[key] = Simulator(w.T, w.C, w.S)
        rng = np.random.default_rng(spec["seed"])
        scat = synth.phantom(rng, w.scatterers, 0, box_xy=w.box_xy, z_range=w.z_range)
        cmap = np.arange(w.C, dtype=np.int16)
        raw, _ = sims[key].run(scat, cmap, spec["seed"])
        frames.append((raw, synth.make_params(w, channel_map=cmap)))
    torch.cuda.synchronize()
    return frames


def work(params):
    """Voxel-transmit-channel evaluations of a list of frames."""
    return sum(math.prod(bp.volume_shape) * bp.dims[1] * bp.dims[2] for bp in params)
