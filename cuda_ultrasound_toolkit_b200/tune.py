"""Autotuner for the knobs of a plan (cutb_options).

For a parameter block it times candidates on the device with CUDA events and keeps the fastest:
  * the delay-and-sum engine and tile (`candidates`): the 4 x 8 x 32 and 8 x 8 x 16 tiles for
    HERCULES and for tilted plane waves in a y-z plane; for TPW and UFORCES, the staged engine
    against the one-thread-per-voxel kernel (which wins on grids too coarse for the staged windows);
  * the delay-and-sum schedule (`schedules`): one CTA per tile, stream-K over the last waves, and,
    for FORCES, TPW and UFORCES, the split of a small volume's tiles over several CTAs;
  * the receive channels per TMA stage (`ROWS`), tried at the best tile and schedule;
  * the decode engine: the int16 fast Walsh-Hadamard transform or the int8 tensor-core
    contraction, where the plan supports the latter.
The FFT of the Hilbert stage has no knob: its radix sequence is fixed by the row length (radix-16
passes, then one of 2, 4 or 8). Results are keyed by everything that changes the kernels' work --
dimensions, grid steps, interpolation, coherence factor, apodization, storage -- and kept in memory
and, when a cache path is given, in a JSON file that later runs reload.
"""
import json
import os

import torch

from .api import CutbError, Plan

CANDIDATES = (1, 2)  # HERCULES: 4 x 8 x 32, 8 x 8 x 16
ROWS = (8, 4)        # receive channels per stage of the staged engine (8: the buffers' capacity)


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


def schedules(bp, tile):
    """das_schedule values for a tile: 0 (HERCULES: one CTA per tile; the other sequences also split
    small volumes over CTAs), 1 (one CTA per tile) where that differs from 0, and 2 (stream-K). The
    one-thread-per-voxel kernel (tile 3) has no schedule."""
    from .params import SequenceId
    if tile == 3:
        return (0,)
    return (0, 2) if int(bp.das_shader_id) == SequenceId.HERCULES else (0, 1, 2)


def config_name(tile, schedule, rows):
    return f"tile{tile}/schedule{schedule}/rows{rows}"


def key(bp, iq_bf16=False):
    S, C, T = bp.dims
    z, y, x = bp.volume_shape
    rx = (bp.output_max_coordinate[0] - bp.output_min_coordinate[0]) / max(x - 1, 1)
    rz = (bp.output_max_coordinate[2] - bp.output_min_coordinate[2]) / max(z - 1, 1)
    return (f"seq{bp.das_shader_id}_T{T}_C{C}_S{S}_X{x}_Y{y}_Z{z}_rx{rx:.4e}_rz{rz:.4e}_cubic{int(bool(bp.interpolate))}"
            f"_cf{bp.coherency_weighting:.3f}_fn{bp.fn_rx:.3f}_apo{bp.apo_type}_bf16{int(iq_bf16)}")


def _median_ms(fn, reps):
    fn()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return sorted(times)[len(times) // 2]


class DasTuner:
    def __init__(self, cache_path=None, reps=3):
        self.cache_path = cache_path
        self.reps = reps
        self.table = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.table = json.load(f)

    def measure(self, bp, tile, iq=None, reps=None, schedule=0, rows=0):
        """Median device time (ms) of one delay-and-sum with the given tile, schedule and rows per
        stage."""
        plan = Plan(bp, das_tile=tile, das_schedule=schedule, das_rows_per_stage=rows)
        if iq is None:
            iq = torch.zeros(plan.empty_iq().shape, dtype=torch.complex64, device="cuda")
        vol = plan.empty_volume()
        ms = _median_ms(lambda: plan.das(iq, out=vol), reps or self.reps)
        plan.check()
        plan.close()
        return ms

    def measure_decode(self, bp, tc, raw=None, reps=None):
        """Median device time (ms) of one decode with the FWHT (tc False) or the tensor-core engine;
        None when the plan does not support the tensor-core engine."""
        try:
            plan = Plan(bp, decode_tc=tc)
        except CutbError:
            return None
        if raw is None:
            from .params import InputDataTypes
            dt = torch.int16 if int(bp.data_type) == InputDataTypes.TYPE_I16 else torch.float32
            n = int(bp.rf_raw_dim[0]) * int(bp.rf_raw_dim[1])
            raw = torch.zeros(n, dtype=dt, device="cuda")
        dec = plan.empty_decoded()
        ms = _median_ms(lambda: plan.decode(raw, out=dec), reps or self.reps)
        plan.check()
        plan.close()
        return ms

    def _search(self, bp, iq):
        ms = {}
        for t in candidates(bp):
            for s in schedules(bp, t):
                ms[config_name(t, s, 0)] = (t, s, 0, self.measure(bp, t, iq, schedule=s))
        t, s, _, _ = min(ms.values(), key=lambda v: v[3])
        if t != 3:  # rows per stage, at the best tile and schedule
            for r in ROWS[1:]:
                ms[config_name(t, s, r)] = (t, s, r, self.measure(bp, t, iq, schedule=s, rows=r))
        t, s, r, _ = min(ms.values(), key=lambda v: v[3])
        dec = {str(tc): self.measure_decode(bp, tc) for tc in (False, True)}
        dec = {k: v for k, v in dec.items() if v is not None}
        return {"tile": t, "schedule": s, "rows": r, "ms": {k: v[3] for k, v in ms.items()},
                "decode_tc": min(dec, key=dec.get) == "True", "decode_ms": dec}

    def entry(self, bp, iq=None):
        """The measured table entry for this parameter block (searched once per key)."""
        k = key(bp)
        if k not in self.table or "schedule" not in self.table[k]:
            self.table[k] = self._search(bp, iq)
            self.save()
        return self.table[k]

    def choose(self, bp, iq=None):
        """The fastest tile id for this parameter block."""
        return self.entry(bp, iq)["tile"]

    def choose_config(self, bp, iq=None):
        """Plan keyword arguments of the fastest measured configuration: Plan(bp, **config)."""
        e = self.entry(bp, iq)
        return dict(das_tile=e["tile"], das_schedule=e["schedule"], das_rows_per_stage=e["rows"],
                    decode_tc=e["decode_tc"])

    def save(self):
        if self.cache_path:
            tmp = self.cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.table, f, indent=1, sort_keys=True)
            os.replace(tmp, self.cache_path)
