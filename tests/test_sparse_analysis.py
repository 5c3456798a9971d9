"""Host-side pieces of the learned path's error analysis (sparse.py `analyze`), on CPU tensors:
the phantom split into point targets and speckle, and the least-squares filter along y."""
import numpy as np
import torch

from cuda_ultrasound_toolkit_b200 import sparse as SP


def test_phantom_parts_split_the_training_phantom():
    for seed in (0, 7, 1_000_003):
        whole = SP.phantom(seed)
        assert np.array_equal(SP.phantom_part(seed, "mixed"), whole)
        pts, spk = SP.phantom_part(seed, "points"), SP.phantom_part(seed, "speckle")
        assert np.array_equal(np.concatenate([pts, spk]), whole)
        assert len(spk) == SP.N_SPECKLE and 50 <= len(pts) <= 400
        assert np.all(pts[:, 3] >= 0.5)


def test_y_filter_recovers_a_shift_and_scale_along_y():
    Z, Y, X = SP.GRID
    g = torch.Generator().manual_seed(3)
    xs = torch.complex(torch.randn((2, Z, Y, X), generator=g), torch.randn((2, Z, Y, X), generator=g))
    # ys[z, y] = c * xs[z, y + 2] (zero past the last row): a filter of half-width 2 represents it
    c = complex(0.5, -1.25)
    ys = torch.zeros_like(xs)
    ys[:, :, :Y - 2] = c * xs[:, :, 2:]
    taps = SP.fit_y_filter(xs, ys, half=2, depths=(0,), ridge=1e-9)
    assert torch.allclose(taps[5], torch.tensor([0, 0, 0, 0, c], dtype=torch.complex64), atol=1e-4)
    out = SP.apply_y_filter(xs, taps, half=2, depths=(0,))
    assert float(torch.linalg.vector_norm(out - ys) / torch.linalg.vector_norm(ys)) < 1e-4
    # regressors of an out-of-volume depth are zero columns
    cols = SP.y_filter_columns(xs[:1], 0, 1, (-1, 0))
    assert cols.shape == (X * Y, 6) and torch.count_nonzero(cols[:, :3]) == 0
