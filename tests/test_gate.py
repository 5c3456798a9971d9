"""The learned path's gate estimator (sparse.Gate) on host tensors: tile sums, the sampling
design and the NRMSE estimate, without a GPU. A volume with a few bright tiles stands in for a
phantom; errors proportional to the signal, additive errors and a mixture are checked against
the exact NRMSE, and the mean of the estimate over draws against the truth."""
import numpy as np
import pytest
import torch

from cuda_ultrasound_toolkit_b200.sparse import Gate

GRID = (64, 64, 64)  # Z, Y, X
TILE = (8, 8, 16)    # x, y, z


def volume(seed):
    g = torch.Generator().manual_seed(seed)
    Z, Y, X = GRID
    v = torch.complex(torch.randn(Z, Y, X, generator=g), torch.randn(Z, Y, X, generator=g)) * 0.05
    for _ in range(12):  # bright point-like blobs: most of the energy in a few tiles
        z, y, x = (int(torch.randint(2, n - 2, (1,), generator=g)) for n in GRID)
        v[z - 2:z + 2, y - 2:y + 2, x - 2:x + 2] += 5.0
    return v


def exact(vhat, v):
    return float(torch.linalg.vector_norm(vhat - v) / torch.linalg.vector_norm(v))


def test_tile_sums_follow_tile_ids():
    gate = Gate(TILE, GRID)
    v = torch.arange(np.prod(GRID), dtype=torch.float64).reshape(GRID)
    sums = gate.tile_sums(v)
    tx, ty, tz = TILE
    nx, ny = GRID[2] // tx, GRID[1] // ty
    for tid in (0, 1, nx, nx * ny, gate.ntiles - 1):
        x, y, z = tid % nx, (tid // nx) % ny, tid // (nx * ny)
        assert sums[tid] == v[z * tz:(z + 1) * tz, y * ty:(y + 1) * ty, x * tx:(x + 1) * tx].sum()


def test_choice_is_distinct_and_weighted():
    gate = Gate(TILE, GRID, fraction=8)
    v = volume(1)
    tiles, w = gate.choose(v, seed=3)
    assert len(np.unique(tiles)) == len(tiles) <= gate.n
    assert (w >= 1.0 - 1e-12).all()
    # the weights of a full design add up to the number of tiles
    assert abs(w.sum() - gate.ntiles) / gate.ntiles < 0.5


@pytest.mark.parametrize("kind", ["proportional", "additive", "mixed"])
@pytest.mark.parametrize("target", [0.01, 0.02, 0.05])
def test_estimate_tracks_exact_nrmse(kind, target):
    gate = Gate(TILE, GRID, fraction=8)
    errs = []
    for seed in range(6):
        v = volume(seed)
        g = torch.Generator().manual_seed(100 + seed)
        n = torch.complex(torch.randn(GRID, generator=g), torch.randn(GRID, generator=g))
        if kind == "proportional":
            e = v * n
        elif kind == "additive":
            e = n
        else:
            e = v * n + n * v.abs().mean()
        e = e * (target * torch.linalg.vector_norm(v) / torch.linalg.vector_norm(e))
        vhat = v + e
        tiles, w = gate.choose(vhat, seed)
        full_tiles = torch.zeros_like(v)
        mask = torch.zeros(gate.ntiles, dtype=torch.bool)
        mask[torch.from_numpy(tiles.astype(np.int64))] = True
        m = mask.reshape(gate.nz, 1, gate.ny, 1, gate.nx, 1).expand(-1, TILE[2], -1, TILE[1], -1, TILE[0])
        full_tiles[m.reshape(GRID)] = v[m.reshape(GRID)]
        est = gate.estimate(vhat, full_tiles, tiles, w)
        errs.append(abs(est - exact(vhat, v)))
    assert max(errs) < 0.25 * target + 0.001, errs
