"""Autotuner for the delay-and-sum tile shape and engine.

For a parameter block it times the delay-and-sum of every candidate (`candidates`) on the device
with CUDA events and keeps the fastest: the 4 x 8 x 32 and 8 x 8 x 16 tiles for HERCULES and for
tilted plane waves in a y-z plane, and, for TPW and UFORCES, the staged engine against the
one-thread-per-voxel kernel (which wins on grids too coarse for the staged windows). Results
are keyed by everything that changes the kernel's work per tile -- dimensions, grid steps,
interpolation, coherence factor, apodization, storage -- and kept in memory and, when a cache
path is given, in a JSON file that later runs reload.
"""
import json
import os

import torch

from .api import Plan

CANDIDATES = (1, 2)  # HERCULES: 4 x 8 x 32, 8 x 8 x 16


def candidates(bp):
    """das_tile values worth timing for this parameter block (cutb_options.das_tile)."""
    from .params import SequenceId
    seq = int(bp.das_shader_id)
    if seq == SequenceId.HERCULES:
        return CANDIDATES
    if seq == SequenceId.RCA_TPW and bp.tx_orientation != bp.rx_orientation:  # plane waves over y
        return (1, 2, 3)
    if seq in (SequenceId.RCA_TPW, SequenceId.UFORCES):
        return (2, 3)  # the staged engine (y-invariant layout), one thread per voxel
    return (0,)


def key(bp, iq_bf16=False):
    S, C, T = bp.dims
    z, y, x = bp.volume_shape
    rx = (bp.output_max_coordinate[0] - bp.output_min_coordinate[0]) / max(x - 1, 1)
    rz = (bp.output_max_coordinate[2] - bp.output_min_coordinate[2]) / max(z - 1, 1)
    return (f"seq{bp.das_shader_id}_T{T}_C{C}_S{S}_X{x}_Y{y}_Z{z}_rx{rx:.4e}_rz{rz:.4e}_cubic{int(bool(bp.interpolate))}"
            f"_cf{bp.coherency_weighting:.3f}_fn{bp.fn_rx:.3f}_apo{bp.apo_type}_bf16{int(iq_bf16)}")


class DasTuner:
    def __init__(self, cache_path=None, reps=3):
        self.cache_path = cache_path
        self.reps = reps
        self.table = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.table = json.load(f)

    def measure(self, bp, tile, iq=None, reps=None):
        """Median device time (ms) of one delay-and-sum with the given tile."""
        plan = Plan(bp, das_tile=tile)
        if iq is None:
            iq = torch.zeros(plan.empty_iq().shape, dtype=torch.complex64, device="cuda")
        vol = plan.empty_volume()
        plan.das(iq, out=vol)
        times = []
        for _ in range(reps or self.reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            plan.das(iq, out=vol)
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        plan.check()
        plan.close()
        return sorted(times)[len(times) // 2]

    def choose(self, bp, iq=None):
        """The fastest tile id for this parameter block (measured once per key)."""
        k = key(bp)
        if k not in self.table:
            ms = {str(t): self.measure(bp, t, iq) for t in candidates(bp)}
            best = min(ms, key=ms.get)
            self.table[k] = {"tile": int(best), "ms": ms}
            self.save()
        return self.table[k]["tile"]

    def save(self):
        if self.cache_path:
            tmp = self.cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.table, f, indent=1, sort_keys=True)
            os.replace(tmp, self.cache_path)
