"""Loader of tests/golden/ncc.npz: outputs of upstream's own motion-detection pipeline (NPP
correlation, CUB candidate sort, quadratic peak fit) on seeded 8-bit speckle frames, produced on a
GPU by tests/golden/make_ncc_golden.py."""
import os

import numpy as np

from cuda_ultrasound_toolkit_b200.params import NccMotionParameters

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ncc.npz")
FLT_MAX = np.float32(3.4028235e38)


def load():
    return np.load(PATH)


def cases(g, kind):
    return sorted({k.split("/")[1] for k in g.files if k.startswith(kind + "/")})


def motion_case(g, name):
    """(frames float32 [F][H][W], params, upstream maps [F][gy][gx][4])."""
    kw = {}
    for k in g.files:
        if k.startswith(f"motion/{name}/p/"):
            v = g[k]
            kw[k.split("/")[-1]] = tuple(v.tolist()) if v.ndim else v.item()
    frames = g[f"motion/{name}/frames"].astype(np.float32)
    return frames, NccMotionParameters.make(**kw), g[f"motion/{name}/maps"]


def corr_case(g, name):
    """(template float32, source float32, upstream correlation map)."""
    return (g[f"corr/{name}/template"].astype(np.float32), g[f"corr/{name}/source"].astype(np.float32),
            g[f"corr/{name}/corr"])
