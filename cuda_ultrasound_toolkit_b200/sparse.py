"""The learned sparse-transmit path: beamform a 4x sparser transmit acquisition, restore it with
the U-Net (csrc/unet.cu, trained by the library's own tcgen05 kernels), and gate every volume
with an online NRMSE estimate against the plain full-transmit delay-and-sum, falling back to
the full-transmit volume when the estimate exceeds the bar.

Acquisitions (row-column array of 128 transmit rows and 128 receive columns, 4096 samples,
fs 20 MHz, pitch 0.3 mm):
  full    128 transmit events, one row each, order-128 Hadamard encoding
  sparse   32 transmit events on every 4th row (rows 2, 6, ..., 126), order-32 Hadamard
           encoding -- a 4x sparser transmit aperture of the same extent
Both are beamformed by the plain pipeline (decode + Hilbert + delay-and-sum, cubic
interpolation, no coherence factor) onto the same 128^3 grid over x, y in [-9, 9] mm and
z in [10, 40] mm, and divided by the simulator's gain, so volumes are in scatterer units.

Phantoms: 50-400 point scatterers with U(0.5, 1) amplitudes plus 20 000 speckle scatterers
with N(0, 0.05) amplitudes, uniform in the box; phantom k is seeded by k.

NRMSE = ||V_hat - V|| / ||V|| over the complex volume, V the plain full-transmit volume.
Gate: the full-transmit front end runs, and the full-transmit delay-and-sum is evaluated on 1/64
of the delay-and-sum tiles (cutb_das_tiles, stages split over CTAs). The tiles are drawn with
probability proportional to half the restored volume's energy in the tile plus half a uniform
share (systematic PPS sampling; tiles whose share would exceed one draw are always taken), and
the squared NRMSE is estimated as the ratio of the Horvitz-Thompson estimates of sum |V_hat - V|^2
and sum |V|^2 over those tiles. Uniformly drawn tiles mostly missed the few bright tiles that
hold most of the energy, and their estimate was off by ~0.04 at NRMSE ~0.4. Above 2 % the volume
falls back to the full-transmit delay-and-sum of the already decoded analytic signal, whose cost
is charged to the learned path.

  python -m cuda_ultrasound_toolkit_b200.sparse train --phantoms 2048 --epochs 4 --out weights.npz
  python -m cuda_ultrasound_toolkit_b200.sparse evaluate --weights weights.npz --phantoms 256
  python -m cuda_ultrasound_toolkit_b200.sparse analyze --phantoms 16 --ab-phantoms 1024

`analyze` measures where the restored volume's error comes from: the NRMSE on point-only and
speckle-only phantoms, the best any linear per-depth filter along y (a global y-deconvolution) can
do on held-out phantoms, and, with --ab-phantoms, the U-Net trained on the sparse volume against the
same U-Net trained on that filter's output.
"""
import argparse
import json
import math
import os
import time

import numpy as np
import torch

from . import learn, synth
from .api import Plan
from .simulate import Simulator

C, S = 128, 4096
ROWS = 128                        # transmit rows of the array
FULL_T, SPARSE_T = 128, 32
SPARSE_STRIDE, SPARSE_OFFSET = 4, 2
GRID = (128, 128, 128)            # Z, Y, X
BOX_XY, Z_RANGE = 9e-3, (10e-3, 40e-3)
N_SPECKLE = 20000
NRMSE_BAR = 0.02
GATE_FRACTION = 64                # the gate evaluates 1 in GATE_FRACTION tiles
GATE_SPLITS = 16                  # stage slices per gate tile
TRAIN_SEED0, EVAL_SEED0 = 0, 1_000_000
CHANNEL_MAP = np.arange(C, dtype=np.int16)
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "unet_sparse4.npz")


def acquisition_params(T, stride=1, offset=0, grid=GRID):
    """Pipeline parameters for T transmit events on rows offset, offset + stride, ... of the array."""
    Z, Y, X = grid
    w = synth.Workload("full" if stride == 1 else "sparse", T, C, S, X, Y, Z, 0, cubic=True, cf=0.0,
                       box_xy=BOX_XY, z_range=Z_RANGE)
    bp = synth.make_params(w, channel_map=CHANNEL_MAP)
    # Transmit j sits on row r = offset + j * stride at y = -ROWS p / 2 + p / 2 + r p; the
    # beamformer places it at -xdc_transform[13] + pitch_y / 2 + j * pitch_y.
    p = synth.PITCH
    bp.xdc_element_pitch[1] = stride * p
    bp.xdc_transform[13] = ROWS * p / 2 - offset * p + (stride - 1) * p / 2
    return bp


def phantom(seed):
    rng = np.random.default_rng(seed)
    return synth.phantom(rng, int(rng.integers(50, 401)), N_SPECKLE, box_xy=BOX_XY, z_range=Z_RANGE)


class Acquisition:
    """Simulator + pipeline for one transmit scheme; volumes in scatterer units."""

    def __init__(self, T, stride=1, offset=0):
        self.sim = Simulator(T, C, S, row_stride=stride, row_offset=offset, array_rows=ROWS)
        self.plan = Plan(acquisition_params(T, stride, offset))
        self.raw = torch.empty((C, T * S), dtype=torch.int16, device="cuda")
        self.gain = torch.empty(1, dtype=torch.float32, device="cuda")

    def acquire(self, scat, seed):
        self.sim.run(scat, CHANNEL_MAP, seed, raw=self.raw, gain=self.gain)
        return self.raw

    def volume(self, out=None):
        out = self.plan.beamform(self.raw, out=out)
        out /= self.gain
        return out


def full_acquisition():
    return Acquisition(FULL_T)


def sparse_acquisition():
    return Acquisition(SPARSE_T, SPARSE_STRIDE, SPARSE_OFFSET)


def nrmse(est, ref):
    return float(torch.linalg.vector_norm(est - ref) / torch.linalg.vector_norm(ref))


def phantom_part(seed, part):
    """phantom(seed) restricted to its point targets ("points"), its speckle ("speckle"), or whole."""
    rng = np.random.default_rng(seed)
    npts = int(rng.integers(50, 401))
    scat = synth.phantom(rng, npts, N_SPECKLE, box_xy=BOX_XY, z_range=Z_RANGE)
    return scat[:npts] if part == "points" else scat[npts:] if part == "speckle" else scat


def make_pairs(n, seed0, log=print, part="mixed"):
    """(sparse volumes, full volumes) for phantoms seed0 .. seed0 + n - 1, complex64 on the GPU."""
    Z, Y, X = GRID
    xs = torch.empty((n, Z, Y, X), dtype=torch.complex64, device="cuda")
    ys = torch.empty_like(xs)
    full, sparse = full_acquisition(), sparse_acquisition()
    t0 = time.time()
    for k in range(n):
        scat = torch.from_numpy(phantom_part(seed0 + k, part)).cuda()
        full.acquire(scat, 2 * (seed0 + k))
        full.volume(out=ys[k])
        sparse.acquire(scat, 2 * (seed0 + k) + 1)
        sparse.volume(out=xs[k])
        if (k + 1) % 256 == 0:
            torch.cuda.synchronize()
            log(f"pairs {k + 1}/{n} {time.time() - t0:.1f}s")
    full.plan.check()
    sparse.plan.check()
    return xs, ys


def held_out_nrmse(net, xs, ys):
    """Median and mean NRMSE of the restored volumes net(xs[k]) against ys[k], and of xs itself."""
    out = torch.empty_like(xs[:1])
    vals = []
    for k in range(xs.shape[0]):
        net.forward(xs[k:k + 1], out=out)
        vals.append(nrmse(out[0], ys[k]))
    return float(np.median(vals)), float(np.mean(vals))


def train(args, log=print):
    torch.manual_seed(0)
    xs, ys = make_pairs(args.phantoms, TRAIN_SEED0, log)
    net = learn.UNet(GRID, max_batch=args.batch, seed=args.seed)
    steps = args.epochs * (args.phantoms // args.batch)
    gen = torch.Generator(device="cpu").manual_seed(args.seed)
    curve = []
    if args.curve:
        # learning curve: held-out NRMSE after every epoch, on phantoms the training never sees
        hx, hy = make_pairs(args.curve, EVAL_SEED0 + 500_000, log)
        base = float(np.median([nrmse(hx[k], hy[k]) for k in range(args.curve)]))
        log(f"held-out sparse-only NRMSE median {base:.4f}")
    t0, step, hist = time.time(), 0, []
    for ep in range(args.epochs):
        perm = torch.randperm(args.phantoms, generator=gen)
        for b in range(args.phantoms // args.batch):
            idx = perm[b * args.batch:(b + 1) * args.batch].cuda()
            lr = args.lr * 0.5 * (1 + math.cos(math.pi * step / steps))
            net.train_step(xs.index_select(0, idx), ys.index_select(0, idx), lr)
            step += 1
            if step % 200 == 0 or step == steps:
                loss = net.last_loss()
                hist.append((step, loss))
                log(f"epoch {ep} step {step}/{steps} loss {loss:.5f} {time.time() - t0:.1f}s")
        if args.curve:
            med, mean = held_out_nrmse(net, hx, hy)
            curve.append((ep + 1, (ep + 1) * args.phantoms, med, mean))
            log(f"epoch {ep + 1}: held-out NRMSE median {med:.4f} mean {mean:.4f}")
    torch.cuda.synchronize()
    train_s = time.time() - t0
    params = net.get_params()
    np.savez_compressed(args.out, params=params, grid=np.array(GRID), phantoms=args.phantoms, epochs=args.epochs,
                        batch=args.batch, lr=args.lr, loss=np.array(hist), train_seconds=train_s,
                        curve=np.array(curve, dtype=np.float64).reshape(-1, 4))
    if args.curve:
        log(json.dumps({"phantoms": args.phantoms, "epochs": args.epochs, "held_out": args.curve,
                        "sparse_only_nrmse_median": base,
                        "curve": [dict(epoch=e, phantom_passes=n, nrmse_median=m, nrmse_mean=a)
                                  for e, n, m, a in curve]}))
        del hx, hy
    log(f"saved {args.out} ({net.param_count} parameters, {train_s:.1f}s of training)")
    del xs, ys
    return net


def load(path=WEIGHTS, max_batch=1):
    d = np.load(path)
    net = learn.UNet(tuple(int(v) for v in d["grid"]), max_batch=max_batch, seed=0)
    net.set_params(d["params"])
    return net


class LearnedPath:
    """Sparse beamforming + restoration + gate + fallback, with per-stage CUDA-event timing."""

    def __init__(self, net):
        self.net = net
        self.sparse = sparse_acquisition()
        self.full = full_acquisition()
        Z, Y, X = GRID
        self.vs = torch.empty((1, Z, Y, X), dtype=torch.complex64, device="cuda")
        self.vo = torch.empty_like(self.vs)
        self.vf = torch.empty((Z, Y, X), dtype=torch.complex64, device="cuda")
        self.vg = torch.empty_like(self.vf)
        self.dec = self.full.plan.empty_decoded()
        self.iq = self.full.plan.empty_iq()
        self.gate = Gate(self.full.plan.tile_shape, GRID)

    def run(self, scat, seed):
        """Acquires both schemes (untimed), then times the learned path's stages and the plain
        path on the device. Returns stage times (ms) and NRMSEs."""
        self.sparse.acquire(scat, 2 * seed + 1)
        self.full.acquire(scat, 2 * seed)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        plan = self.full.plan
        ev[0].record()
        self.sparse.volume(out=self.vs[0])
        ev[1].record()
        self.net.forward(self.vs, out=self.vo)
        ev[2].record()
        plan.decode(self.full.raw, out=self.dec)
        plan.hilbert(self.dec, out=self.iq)
        ev[3].record()
        tiles, weights = self.gate.choose(self.vo[0], seed)
        plan.das_tiles(self.iq, tiles, splits=GATE_SPLITS, out=self.vg)
        self.vg /= self.full.gain
        est = self.gate.estimate(self.vo[0], self.vg, tiles, weights)
        ev[4].record()
        plan.das(self.iq, out=self.vf)   # plain path's delay-and-sum, also the fallback
        self.vf /= self.full.gain
        ev[5].record()
        torch.cuda.synchronize()
        t = [ev[i].elapsed_time(ev[i + 1]) for i in range(5)]
        return dict(sparse_ms=t[0], unet_ms=t[1], front_ms=t[2], gate_ms=t[3], das_ms=t[4], gate_nrmse=float(est),
                    nrmse_net=nrmse(self.vo[0], self.vf), nrmse_plain=nrmse(self.vs[0], self.vf))


class Gate:
    """Spot check of a restored volume against the full-transmit delay-and-sum on 1 in
    GATE_FRACTION tiles. choose() picks the tiles from the restored volume (one device-to-host
    copy of its 2048 tile energies), estimate() returns the NRMSE estimate from the restored
    volume and the full-transmit delay-and-sum of the chosen tiles."""

    def __init__(self, tile_shape, grid, fraction=GATE_FRACTION, uniform_share=0.5):
        self.tx, self.ty, self.tz = tile_shape
        Z, Y, X = grid
        self.nx, self.ny, self.nz = -(-X // self.tx), -(-Y // self.ty), -(-Z // self.tz)
        assert (self.nx * self.tx, self.ny * self.ty, self.nz * self.tz) == (X, Y, Z), "whole tiles only"
        self.ntiles = self.nx * self.ny * self.nz
        self.n = max(1, self.ntiles // fraction)
        self.uniform_share = uniform_share

    def tile_sums(self, v):
        """Sum over each tile of v (Z, Y, X) -> tile id order (z-major, then y, then x)."""
        t = v.reshape(self.nz, self.tz, self.ny, self.ty, self.nx, self.tx)
        return t.sum(dim=(1, 3, 5)).reshape(-1)

    def choose(self, restored, seed):
        """(tile ids int32, Horvitz-Thompson weights 1 / inclusion probability) for this volume."""
        energy = self.tile_sums(restored.real.square() + restored.imag.square()).double().cpu().numpy()
        N, n = self.ntiles, self.n
        tot = energy.sum()
        p = (1 - self.uniform_share) * (energy / tot if tot > 0 else np.full(N, 1.0 / N)) + self.uniform_share / N
        certain = np.zeros(N, dtype=bool)
        while True:  # tiles that would be drawn with probability >= 1 are taken outright
            rest = np.flatnonzero(~certain)
            m = n - int(certain.sum())
            q = p[rest] / p[rest].sum()
            big = rest[q * m >= 1.0]
            if len(big) == 0 or m <= 0:
                break
            certain[big] = True
        rest = np.flatnonzero(~certain)
        m = n - int(certain.sum())
        tiles, weights = list(np.flatnonzero(certain)), [1.0] * int(certain.sum())
        if m > 0:
            q = p[rest] / p[rest].sum()
            start = np.random.default_rng(seed).random()
            picks = np.searchsorted(np.cumsum(q), (start + np.arange(m)) / m, side="right")
            picks = np.minimum(picks, len(rest) - 1)
            tiles += list(rest[picks])
            weights += list(1.0 / (m * q[picks]))
        # a tile drawn twice (only possible through rounding at the edge q m -> 1) is listed once,
        # with its weights added: the delay-and-sum adds the partial sums of a listed tile
        ids, inv = np.unique(np.asarray(tiles, dtype=np.int64), return_inverse=True)
        w = np.zeros(len(ids))
        np.add.at(w, inv, np.asarray(weights, dtype=np.float64))
        return ids.astype(np.int32), w

    def estimate(self, restored, full_tiles, tiles, weights):
        """NRMSE estimate: sqrt(HT(sum |restored - full|^2) / HT(sum |full|^2)) over the tiles."""
        d = restored - full_tiles
        err = self.tile_sums(d.real.square() + d.imag.square())
        en = self.tile_sums(full_tiles.real.square() + full_tiles.imag.square())
        idx = torch.from_numpy(tiles.astype(np.int64)).to(restored.device)
        w = torch.from_numpy(weights).to(restored.device)
        num = (err.index_select(0, idx).double() * w).sum()
        den = (en.index_select(0, idx).double() * w).sum()
        return float(torch.sqrt(num / den))


def summarize(rows, bar=NRMSE_BAR):
    """Volumes/s of the plain path (front end + delay-and-sum of the full acquisition) and of
    the learned path (sparse volume + network + full front end + gate, plus the full
    delay-and-sum for every volume the gate rejects)."""
    n = len(rows)
    plain = sum(r["front_ms"] + r["das_ms"] for r in rows)
    passed = [r["gate_nrmse"] <= bar for r in rows]
    learned = sum(r["sparse_ms"] + r["unet_ms"] + r["front_ms"] + r["gate_ms"] + (0.0 if ok else r["das_ms"])
                  for r, ok in zip(rows, passed))
    true_ok = [r["nrmse_net"] <= bar for r in rows]
    oracle_gated = sum(r["sparse_ms"] + r["unet_ms"] + (0.0 if ok else r["front_ms"] + r["das_ms"])
                       for r, ok in zip(rows, true_ok))
    delivered = [r["nrmse_net"] if ok else 0.0 for r, ok in zip(rows, passed)]
    mean = lambda k: float(np.mean([r[k] for r in rows]))  # noqa: E731
    return dict(
        volumes=n, plain_volumes_per_s=1e3 * n / plain, learned_volumes_per_s=1e3 * n / learned,
        learned_oracle_gated_volumes_per_s=1e3 * n / oracle_gated, speedup=plain / learned,
        gate_pass_fraction=sum(passed) / n, true_pass_fraction=sum(true_ok) / n,
        nrmse_net_median=float(np.median([r["nrmse_net"] for r in rows])), nrmse_net_mean=mean("nrmse_net"),
        nrmse_plain_sparse_median=float(np.median([r["nrmse_plain"] for r in rows])),
        nrmse_delivered_max=float(max(delivered)) if delivered else 0.0,
        gate_error_median=float(np.median([abs(r["gate_nrmse"] - r["nrmse_net"]) for r in rows])),
        ms=dict(sparse=mean("sparse_ms"), unet=mean("unet_ms"), front=mean("front_ms"), gate=mean("gate_ms"),
                das=mean("das_ms")))


def evaluate(net, n, seed0=EVAL_SEED0, warmup=2, log=print):
    path = LearnedPath(net)
    for k in range(warmup):
        path.run(torch.from_numpy(phantom(seed0 + k)).cuda(), seed0 + k)
    rows = []
    for k in range(n):
        rows.append(path.run(torch.from_numpy(phantom(seed0 + k)).cuda(), seed0 + k))
    path.full.plan.check()
    path.sparse.plan.check()
    net.check()
    return summarize(rows), rows


# ---- Where the error comes from -------------------------------------------------------------
def y_filter_columns(v, k, half, depths):
    """Regressors of output depth k: v[:, k + a, y + o, x] for a in depths, o = -half .. half (zero
    outside the volume), one row per (volume, x, y)."""
    Z, Y, X = GRID
    cols = []
    for a in depths:
        if not 0 <= k + a < Z:
            cols.append(torch.zeros((v.shape[0] * X * Y, 2 * half + 1), dtype=v.dtype, device=v.device))
            continue
        p = torch.nn.functional.pad(torch.view_as_real(v[:, k + a]).permute(0, 3, 2, 1), (half, half))
        u = p.unfold(3, 2 * half + 1, 1)  # [n][2][X][Y][taps]
        cols.append(torch.complex(u[:, 0], u[:, 1]).reshape(-1, 2 * half + 1))
    return torch.cat(cols, 1)


def fit_y_filter(xs, ys, half, depths, ridge=1e-3):
    """Complex taps per output depth minimising sum |ys - filter(xs)|^2 (ridge relative to the
    Gram matrix's mean diagonal): the best linear mixing along y (and nearby depths) there is."""
    taps = []
    for k in range(GRID[0]):
        A = y_filter_columns(xs, k, half, depths)
        t = ys[:, k].permute(0, 2, 1).reshape(-1)
        G = A.conj().T @ A
        G += ridge * torch.trace(G).real / G.shape[0] * torch.eye(G.shape[0], device=G.device)
        taps.append(torch.linalg.solve(G, A.conj().T @ t))
    return taps


def apply_y_filter(v, taps, half, depths, chunk=32):
    Z, Y, X = GRID
    out = torch.empty_like(v)
    for c in range(0, v.shape[0], chunk):
        vc = v[c:c + chunk]
        for k in range(Z):
            out[c:c + chunk, k] = (y_filter_columns(vc, k, half, depths) @ taps[k]).reshape(-1, X, Y).permute(0, 2, 1)
    return out


def median_nrmse(xs, ys):
    return float(np.median([nrmse(xs[k], ys[k]) for k in range(xs.shape[0])]))


def train_on(xs, ys, hx, hy, epochs, batch=2, lr=1e-3, seed=1, log=print, tag=""):
    """Trains a fresh U-Net on the pairs (xs, ys) with the schedule of `train`; returns the held-out
    median NRMSE on (hx, hy) after each epoch."""
    net = learn.UNet(GRID, max_batch=batch, seed=seed)
    n = xs.shape[0]
    steps, step, curve = epochs * (n // batch), 0, []
    gen = torch.Generator(device="cpu").manual_seed(seed)
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen)
        for b in range(n // batch):
            idx = perm[b * batch:(b + 1) * batch].cuda()
            net.train_step(xs.index_select(0, idx), ys.index_select(0, idx),
                           lr * 0.5 * (1 + math.cos(math.pi * step / steps)))
            step += 1
        curve.append(held_out_nrmse(net, hx, hy)[0])
        log(f"{tag}epoch {ep + 1}: held-out NRMSE median {curve[-1]:.4f}")
    net.check()
    net.close()
    return curve


def analyze(args, log=print):
    """Prints (and returns) the measurements behind the learned path's error floor."""
    res = {}
    net = load(args.weights)
    n = args.phantoms
    parts = {}
    for part in ("mixed", "points", "speckle"):
        xs, ys = make_pairs(n, EVAL_SEED0, log=lambda *a: None, part=part)
        out, vals = torch.empty_like(xs[:1]), []
        for k in range(n):
            net.forward(xs[k:k + 1], out=out)
            vals.append(nrmse(out[0], ys[k]))
        res[part] = dict(sparse=median_nrmse(xs, ys), unet=float(np.median(vals)))
        log(f"{part:8s} phantoms: sparse volume NRMSE {res[part]['sparse']:.4f}, restored {res[part]['unet']:.4f}")
        parts[part] = ys
        del xs
    share = [float(torch.linalg.vector_norm(parts["speckle"][k]) ** 2 /
                   (torch.linalg.vector_norm(parts["points"][k]) ** 2 + torch.linalg.vector_norm(parts["speckle"][k]) ** 2))
             for k in range(n)]
    res["speckle_energy_share"] = float(np.median(share))
    log(f"speckle share of the full volume's energy: median {res['speckle_energy_share']:.3f}")
    del parts
    fx, fy = make_pairs(n, EVAL_SEED0, log=lambda *a: None)
    hx, hy = make_pairs(n, EVAL_SEED0 + 5000, log=lambda *a: None)
    res["y_filter"] = []
    for half, depths in ((0, (0,)), (16, (0,)), (48, (0,)), (96, (0,)), (48, (-1, 0, 1)), (48, (-3, -2, -1, 0, 1, 2, 3))):
        taps = fit_y_filter(fx, fy, half, depths)
        e = median_nrmse(apply_y_filter(hx, taps, half, depths), hy)
        res["y_filter"].append(dict(half_width=half, depths=list(depths), held_out_nrmse=e))
        log(f"linear filter along y, {2 * half + 1} taps x {len(depths)} depths: held-out NRMSE {e:.4f} "
            f"(sparse volume {median_nrmse(hx, hy):.4f})")
    del fx, fy, hx, hy
    if args.ab_phantoms:
        half, depths = 48, (-1, 0, 1)
        xs, ys = make_pairs(args.ab_phantoms, TRAIN_SEED0, log)
        hx, hy = make_pairs(64, EVAL_SEED0 + 500_000, log=lambda *a: None)
        taps = fit_y_filter(xs[:64], ys[:64], half, depths)
        res["ab_plain"] = train_on(xs, ys, hx, hy, args.ab_epochs, log=log, tag="U-Net on the sparse volume: ")
        xs = apply_y_filter(xs, taps, half, depths)
        res["ab_y_filtered"] = train_on(xs, ys, apply_y_filter(hx, taps, half, depths), hy, args.ab_epochs, log=log,
                                        tag="U-Net on the y-filtered volume: ")
    return res


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--phantoms", type=int, default=2048)
    t.add_argument("--epochs", type=int, default=4)
    t.add_argument("--batch", type=int, default=2)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--eval", type=int, default=0, help="evaluate on this many held-out phantoms afterwards")
    t.add_argument("--curve", type=int, default=0,
                   help="held-out phantoms whose NRMSE is logged after every epoch (learning curve)")
    e = sub.add_parser("evaluate")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--phantoms", type=int, default=256)
    e.add_argument("--json", default=None)
    n = sub.add_parser("analyze")
    n.add_argument("--weights", default=WEIGHTS)
    n.add_argument("--phantoms", type=int, default=16)
    n.add_argument("--ab-phantoms", type=int, default=0, help="also train the A/B pair on this many phantoms")
    n.add_argument("--ab-epochs", type=int, default=4)
    n.add_argument("--json", default=None)
    a = ap.parse_args()
    if a.cmd == "analyze":
        res = analyze(a)
        if a.json:
            with open(a.json, "w") as f:
                json.dump(res, f)
        return
    if a.cmd == "train":
        net = train(a)
        if a.eval:
            s, _ = evaluate(net, a.eval)
            print(json.dumps(s))
    else:
        net = load(a.weights)
        s, rows = evaluate(net, a.phantoms)
        print(json.dumps(s))
        if a.json:
            with open(a.json, "w") as f:
                json.dump(dict(summary=s, rows=rows), f)


if __name__ == "__main__":
    main()
