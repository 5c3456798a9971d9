#!/usr/bin/env python
"""Benchmark of the RF -> volume pipeline (one JSON line on rank 0).

Workload ("full"): 128 transmits x 128 receive channels x 4096 samples of Hadamard-encoded
int16 RF (128 MiB raw), 64-tap chirp match filter, HERCULES plane-wave delay-and-sum into a
128 x 128 x 256 complex64 volume with cubic interpolation and coherence-factor weighting.
One step = convert + reorder + decode -> Hilbert -> delay-and-sum of one frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (launched by torchrun) every rank beamforms its own frames (frames are
independent: no collective on the data path) and the job-wide volumes/s is reported
(weak scaling). --impl reference times the CPU path (the FP64 oracle) on a bounded
sample of the same workload on rank 0.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "volumes/s (plain full-transmit RF->volume pipeline)"
UNIT = "volumes/s"
WORKLOAD = "full"


def parallelism(world):
    return f"frame-parallel x{world}" if world > 1 else "single GPU"


def workload_config(extra=None):
    from cuda_ultrasound_toolkit_b200 import synth
    w = synth.CONFIGS[WORKLOAD]
    cfg = {"workload": "rca128_hercules_cubic_cf", "transmits": w.T, "channels": w.C, "samples": w.S,
           "volume": [w.X, w.Y, w.Z], "input": "int16 Hadamard-encoded", "match_filter_taps": w.filter_taps,
           "interpolation": "cubic", "coherence_factor": w.cf,
           "l2": "inputs > L2 (128 MiB raw, 512 MiB analytic signal; two raw frames alternate)"}
    if extra:
        cfg.update(extra)
    return cfg


# ---- frame-parallel sharding ------------------------------------------------------------------------
def frame_seeds(rank, world, per_rank=2, base=7000):
    """Seeds of the frames rank `rank` beamforms: disjoint across ranks, fixed per rank (weak scaling)."""
    return [base + per_rank * rank + k for k in range(per_rank)]


def max_over_ranks(values, world, device=None):
    """Element-wise max of per-rank timings (the job is as slow as its slowest rank)."""
    if world <= 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


# ---- clocks sampled during the timed region ------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "of measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "of fallback"


def shared_roofline(vct, cubic, das_ms, sm_mhz, sms=148):
    """Shared-memory roofline of the delay-and-sum: algorithmic coefficient bytes (32 B cubic / 16 B
    linear per voxel-transmit-channel) over the SMs' shared data path (128 B per clock per SM) at
    the median SM clock sampled during the timed region."""
    if not sm_mhz:
        return None
    nbytes = vct * (32 if cubic else 16)
    achieved = nbytes / (das_ms * 1e-3) / 1e12
    peak = sms * 128 * sm_mhz * 1e6 / 1e12
    return {"bytes_per_launch": nbytes, "achieved_tbs": achieved, "peak_tbs": peak, "frac": achieved / peak,
            "unit": "TB/s", "peak_source": f"{sms} SMs x 128 B/clk x {sm_mhz:.0f} MHz (sampled SM clock)"}


def profile_traffic(name):
    """DRAM bytes per launch recorded by ncu for a kernel (profiles/<name>.json), if committed."""
    path = os.path.join(ROOT, "profiles", f"{name}.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    return None


# ---- CPU reference arm -------------------------------------------------------------------------------
N_VOXEL_SUBSETS = 64   # the delay-and-sum of a CPU step covers one seeded 1/64 of the voxels
PARITY_VOXELS = 16384  # seeded voxel sample the GPU volume is compared on, against the FP64 oracle


def voxel_subset(bp, k, n=N_VOXEL_SUBSETS, seed=0):
    """Subset k of n disjoint, seeded voxel subsets that together cover the volume."""
    z, y, x = bp.volume_shape
    perm = np.random.default_rng(seed).permutation(x * y * z)
    return np.sort(np.array_split(perm, n)[k % n])


def cpu_sample(raw, bp, threads, subset=0, n_subsets=N_VOXEL_SUBSETS, channels=None, keep_iq=False, elapsed=None):
    """Times the FP64 oracle on one bounded sample of a frame and extrapolates seconds per volume:
    convert + decode and the Hilbert analytic signal of `channels` receive channels (default: all,
    i.e. the front end in full), and the delay-and-sum of voxel subset `subset` of `n_subsets`
    (scaled by n_subsets). Returns (seconds per volume, description, analytic signal or None); the
    sample's own duration is appended to the list `elapsed` when one is given."""
    from oracle import oracle as O
    S, C, T = bp.dims
    z, y, x = bp.volume_shape
    sub_c = C if channels is None else max(1, min(C, int(channels)))
    sub = bp.copy()
    sub.dec_data_dim[1] = sub_c
    t0 = time.perf_counter()
    dec = O.decode_f64(raw, sub, threads)
    t1 = time.perf_counter()
    taps = np.ctypeslib.as_array(bp.rf_filter)[: int(bp.filter_length)].astype(np.float32)
    iq = O.hilbert(dec, taps if len(taps) else None, threads)
    t2 = time.perf_counter()
    del dec
    if sub_c < C:  # the delay-and-sum needs every row: tile the sampled channels over the aperture
        iq = iq[:, np.arange(C) % sub_c]
    vox = voxel_subset(bp, subset, n_subsets)
    t3 = time.perf_counter()
    O.das(iq, bp, vox, threads)
    t4 = time.perf_counter()
    per_volume = (t2 - t0) * C / sub_c + (t4 - t3) * (x * y * z) / len(vox)
    if elapsed is not None:
        elapsed.append((t2 - t0) + (t4 - t3))
    front = "in full" if sub_c == C else f"on {sub_c} of {C} receive channels, scaled"
    sample = (f"FP64 oracle: convert + decode + Hilbert of {T} x {C} rows x {S} samples {front}; "
              f"delay-and-sum of the seeded voxel subset {subset % n_subsets} of {n_subsets} ({len(vox)} of "
              f"{x * y * z} voxels, all {T * C} rows), extrapolated linearly to one volume")
    return per_volume, sample, (iq if keep_iq else None)


def run_reference(args, rank):
    if rank != 0:
        return
    from cuda_ultrasound_toolkit_b200 import synth
    raw, bp = synth.frame(WORKLOAD)
    threads = os.cpu_count() or 1
    for k in range(args.warmup):  # untimed: a light pass over the same code
        cpu_sample(raw, bp, threads, subset=k, n_subsets=4096, channels=8)
    # A step is one bounded sample (the front end in full, 1/64 of the voxels): ms_per_step is its
    # measured duration, and value extrapolates the samples to whole volumes per second.
    times, ran = [], []
    sample = ""
    for k in range(args.steps):
        sec, sample, _ = cpu_sample(raw, bp, threads, subset=k, elapsed=ran)
        times.append(sec)
    value = len(times) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(ran) / len(ran),
            "step": "one bounded sample of the frame (front end in full, delay-and-sum of 1/64 of the voxels); "
                    f"{1e3 * sum(times) / len(times):.0f} ms per volume extrapolated",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded phantom, 200 point scatterers, 40 dB SNR)",
            "config": workload_config({"parallelism": parallelism(int(os.environ.get("WORLD_SIZE", "1")))}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample + "; step k times subset k"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def upstream_gpu_section(raw, bp, ours_vol, reps=3, fp64=None):
    """Upstream's own CUDA build (baseline/_ref, built by baseline/Makefile for sm_100a) timed
    through its cuda_toolkit::beamform on host buffers, in a child process, on the benchmark
    frame with the settings upstream honours: cubic interpolation and no coherence factor
    (upstream's HERCULES kernel computes the factor but never applies it). `ours_vol` is this
    library's volume of the same frame and settings; fp64 = (voxels, FP64 oracle volume there)."""
    import subprocess
    import tempfile
    lib = os.path.join(ROOT, "baseline", "_ref", "libcuda_toolkit_upstream.so")
    if not os.path.exists(lib):
        return {"unavailable": "baseline/_ref/libcuda_toolkit_upstream.so not built (make -C baseline REF=...)"}
    with tempfile.TemporaryDirectory() as d:
        np.save(os.path.join(d, "raw.npy"), raw)
        with open(os.path.join(d, "params.bin"), "wb") as f:
            f.write(bytes(bp))
        r = subprocess.run([sys.executable, os.path.join(ROOT, "baseline", "upstream_gpu.py"), d, str(reps)],
                           capture_output=True, text=True, timeout=600)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode != 0 or not lines:
            return {"failed": f"rc {r.returncode}: {(r.stderr or r.stdout)[-300:]}"}
        out = json.loads(lines[-1])
        if os.path.exists(os.path.join(d, "volume.npy")):
            ref = np.load(os.path.join(d, "volume.npy"))
            out["rel_l2_ours_vs_upstream"] = float(np.linalg.norm(ours_vol - ref) / np.linalg.norm(ref))
            if fp64 is not None:
                vox, exact = fp64
                rel = lambda v: float(np.linalg.norm(v.reshape(-1)[vox] - exact) / np.linalg.norm(exact))  # noqa: E731
                out["rel_l2_vs_fp64"] = {"upstream": rel(ref), "ours": rel(ours_vol), "voxels": len(vox)}
    out["settings"] = "interpolate=true (cubic), coherency_weighting=0; same frame"
    return out


# ---- GPU arm ------------------------------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from cuda_ultrasound_toolkit_b200 import Plan, beamform, synth
    from cuda_ultrasound_toolkit_b200.api import calibrate_fp32

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    # Frames of one acquisition: same probe set-up (channel map), different echoes.
    seeds = frame_seeds(rank, world)
    frames = [synth.frame(WORKLOAD, seed=seeds[0])]
    cmap = np.ctypeslib.as_array(frames[0][1].channel_mapping)[: frames[0][1].dims[1]].copy()
    frames += [synth.frame(WORKLOAD, seed=sd, channel_map=cmap) for sd in seeds[1:]]
    bp = frames[0][1]
    for _, b in frames[1:]:  # same geometry; only the data and channel map differ per frame
        assert b.dims == bp.dims
    plans = [Plan(b) for _, b in frames]
    d_raw = [torch.from_numpy(r).to(dev) for r, _ in frames]
    vol = plans[0].empty_volume()
    stream = torch.cuda.current_stream()

    def step(k):
        plans[k % 2].beamform(d_raw[k % 2], out=vol, stream=stream)

    def barrier():
        if world > 1:
            dist.barrier()

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        step(k)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clock = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = plans[0].launches * args.steps

    # Per-stage timing on the same stream (dominant kernel = delay-and-sum).
    p = plans[0]
    dec = p.empty_decoded()
    iq = p.empty_iq()
    stage_ms = {}
    for name, fn in (("decode", lambda: p.decode(d_raw[0], out=dec, stream=stream)),
                     ("hilbert", lambda: p.hilbert(dec, out=iq, stream=stream)),
                     ("das", lambda: p.das(iq, out=vol, stream=stream))):
        fn()
        reps = 3 if name == "das" else 20
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        stage_ms[name] = a.elapsed_time(b) / reps

    # End to end through the host-span entry point (cuda_toolkit::beamform): pinned host
    # input, H2D copy, pipeline, D2H of the volume, every step.
    host_raw = [torch.from_numpy(r).pin_memory() for r, _ in frames]
    host_vol = torch.empty(bp.volume_shape, dtype=torch.complex64).pin_memory()
    raw_np = [h.numpy() for h in host_raw]
    vol_np = host_vol.numpy()
    for k in range(2):
        beamform(raw_np[k % 2], frames[k % 2][1], out=vol_np)
    e2e_steps = max(3, args.steps // 2)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        beamform(raw_np[k % 2], frames[k % 2][1], out=vol_np)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    barrier()

    # One frame split over the ranks by z-slabs (broadcast of the raw frame, every rank's slab,
    # all-gather of the slabs): the latency of a single frame on N GPUs. Every rank takes part.
    sharded_ms = None
    if world > 1:
        from cuda_ultrasound_toolkit_b200.sharded import ShardedFrame
        sf = ShardedFrame(bp, rank, world)
        d_frame = d_raw[0].clone()
        sf.beamform(d_frame)
        torch.cuda.synchronize()
        barrier()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(3):
            sf.beamform(d_frame)
        s1.record(stream)
        torch.cuda.synchronize()
        barrier()
        sf.plan.check()
        sharded_ms = s0.elapsed_time(s1) / 3
        del sf, d_frame

    # Max over ranks.
    ms, e2e_s = max_over_ranks([ms, e2e_s], world, dev)
    if sharded_ms is not None:
        sharded_ms = max_over_ranks([sharded_ms], world, dev)[0]
    if rank != 0:
        return

    S, C, T = bp.dims
    z, y, x = bp.volume_shape
    vct = x * y * z * T * C
    flops_per_vct = 49 if bp.interpolate else 23  # cubic + CF / linear, no CF
    if bp.interpolate and bp.coherency_weighting <= 0:
        flops_per_vct = 45
    fp32_peak = calibrate_fp32()
    das_tflops = vct * flops_per_vct / (stage_ms["das"] * 1e-3) / 1e12
    peaks, peak_src = measured_peaks()
    hbm = peaks["hbm_gbs"]
    dec_bytes = T * C * S * (2 + 4)
    hil_bytes = T * C * S * (4 + 8)
    value = args.steps * world / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (int16 input, int32 exact decode)",
        "data": "synthetic (seeded phantom, 200 point scatterers, 40 dB SNR)",
        "config": workload_config({"parallelism": parallelism(world)}),
        "e2e": {"value": e2e_steps * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(raw_np[0].nbytes),
                "d2h_bytes_per_step": int(vol_np.nbytes), "api": "cuda_toolkit::beamform (host spans)"},
        "roofline": {"bound": "fp32", "kernel": "das", "achieved": das_tflops, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": das_tflops / fp32_peak, "traffic": profile_traffic("das_full"),
                     "algorithmic": f"{flops_per_vct} FLOP per voxel-transmit-channel x {vct} per launch",
                     "peak_source": "measured FP32 FMA probe (cutb_calibrate_fp32) on this GPU",
                     # the data path the kernel saturates first: every voxel-transmit-channel reads
                     # its interval's four complex cubic coefficients (32 B) from shared memory, and
                     # an SM moves 128 B of shared data per clock
                     "shared_memory": shared_roofline(vct, bp.interpolate, stage_ms["das"], clock.get("sm_mhz"))},
        "stages": {
            "decode": {"ms": stage_ms["decode"], "achieved_gbs": dec_bytes / (stage_ms["decode"] * 1e-3) / 1e9,
                       "peak_gbs": hbm, "frac": dec_bytes / (stage_ms["decode"] * 1e-3) / 1e9 / hbm,
                       "peak_note": peak_src, "traffic": profile_traffic("decode_full")},
            "hilbert": {"ms": stage_ms["hilbert"], "achieved_gbs": hil_bytes / (stage_ms["hilbert"] * 1e-3) / 1e9,
                        "peak_gbs": hbm, "frac": hil_bytes / (stage_ms["hilbert"] * 1e-3) / 1e9 / hbm,
                        "peak_note": peak_src, "traffic": profile_traffic("hilbert_full")},
            "das": {"ms": stage_ms["das"], "tflops": das_tflops},
        },
        "gpu_launches": launches,
        "clocks": clock,
    }
    if sharded_ms is not None:
        line["single_frame_zslabs"] = {
            "ms_per_frame": sharded_ms, "volumes_per_s": 1e3 / sharded_ms, "ranks": world,
            "what": "one frame split by voxel z-slabs: NCCL broadcast of the raw frame, decode + Hilbert on "
                    "every rank, each rank's slab (cutb_das_zslab), all-gather of the slabs; max over ranks"}
    if args.learned > 0 and world == 1:
        line["learned"] = learned_path(args.learned)
    if args.precision and world == 1:
        try:
            line["precision"] = precision_form()
        except Exception as exc:  # must not hide the plain pipeline's number
            line["precision"] = {"failed": str(exc)}
    if args.batched > 0 and world == 1:
        try:
            line["batched"] = batched_stream(args.batched)
        except Exception as exc:  # must not hide the plain pipeline's number
            line["batched"] = {"failed": str(exc)}
    if args.motion and world == 1:
        try:
            line["motion"] = motion_section()
        except Exception as exc:  # must not hide the plain pipeline's number
            line["motion"] = {"failed": str(exc)}
    if args.sequences and world == 1:
        try:
            line["sequences"] = sequences_section()
        except Exception as exc:  # must not hide the plain pipeline's number
            line["sequences"] = {"failed": str(exc)}
    if args.transfer and world == 1:
        try:
            line["transfer"] = transfer_section()
        except Exception as exc:  # must not hide the plain pipeline's number
            line["transfer"] = {"failed": str(exc)}
    threads = os.cpu_count() or 1
    iq_ref = None
    try:
        per_vol, sample, iq_ref = cpu_sample(frames[0][0], bp, threads, subset=0, keep_iq=True)
        line["cpu_baseline"] = {"value": 1.0 / per_vol, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": sample}
    except Exception as exc:  # the baseline must not hide the GPU number
        line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"failed: {exc}"}
    try:
        line["parity"] = full_frame_parity(plans[0], d_raw[0], frames[0][0], bp, iq_ref, threads)
    except Exception as exc:  # must not hide the plain pipeline's number
        line["parity"] = {"failed": str(exc)}
    if args.upstream and world == 1:
        try:
            ref_bp = bp.copy()
            ref_bp.coherency_weighting = 0.0
            fp64 = None
            if iq_ref is not None:  # FP64 volume of upstream's settings on the parity voxels
                from oracle import oracle as O
                z, y, x = bp.volume_shape
                vox = np.sort(np.random.default_rng(21).choice(x * y * z, PARITY_VOXELS, replace=False))
                fp64 = (vox, O.das(iq_ref, ref_bp, vox, threads))
            ours = beamform(frames[0][0], ref_bp)
            e2e_ref = []
            for _ in range(3):
                t = time.perf_counter()
                beamform(frames[0][0], ref_bp, out=ours)
                e2e_ref.append(time.perf_counter() - t)
            up = upstream_gpu_section(frames[0][0], ref_bp, ours, fp64=fp64)
            up["ours_same_settings"] = {"ms": 1e3 * float(np.median(e2e_ref)),
                                        "volumes_per_s": 1.0 / float(np.median(e2e_ref)),
                                        "api": "cuda_toolkit::beamform (host spans)"}
            if up.get("ms"):
                up["speedup_ours_vs_upstream"] = up["ms"] / up["ours_same_settings"]["ms"]
            line["upstream_gpu"] = up
        except Exception as exc:  # must not hide the plain pipeline's number
            line["upstream_gpu"] = {"failed": str(exc)}
    del iq_ref
    print(json.dumps(line), flush=True)


def full_frame_parity(plan, d_raw, raw, bp, iq_ref, threads):
    """The benchmark frame's GPU result against the FP64 oracle, outside the timed region: the
    decode bit for bit, the volume on PARITY_VOXELS seeded voxels (relative L2). iq_ref is the
    oracle's analytic signal of the frame, when the CPU baseline has computed it."""
    import torch
    from oracle import oracle as O
    dec = plan.decode(d_raw).cpu().numpy()
    exact = bool(np.array_equal(dec, O.decode_i16(raw, bp, threads)))
    del dec
    vol = plan.beamform(d_raw)
    plan.check()
    z, y, x = bp.volume_shape
    vox = np.sort(np.random.default_rng(21).choice(x * y * z, PARITY_VOXELS, replace=False))
    if iq_ref is None:
        _, _, iq_ref = cpu_sample(raw, bp, threads, keep_iq=True)
    ref = O.das(iq_ref, bp, vox, threads)
    got = vol.reshape(-1)[torch.from_numpy(vox).to(vol.device)].cpu().numpy()
    return {"decode_bit_exact": exact, "rel_l2_vs_fp64": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            "voxels": PARITY_VOXELS, "bar": 1e-5,
            "oracle": "FP64 decode -> Hilbert -> delay-and-sum of the same frame (oracle/oracle.cpp)"}


def learned_path(volumes):
    """The learned sparse-transmit path against the plain full-transmit path on held-out phantoms
    (128 x 128 rows/columns, 4096 samples, 128^3 volume, cubic, no coherence factor): 32 transmits
    on every 4th row -> delay-and-sum -> U-Net, gated by a full-transmit spot check (1/64 of the
    tiles) with fallback to the full delay-and-sum above 2 % NRMSE; both paths timed on the device
    from the int16 raw frames in HBM."""
    from cuda_ultrasound_toolkit_b200 import sparse
    if not os.path.exists(sparse.WEIGHTS):
        return {"unavailable": f"no trained weights at {os.path.relpath(sparse.WEIGHTS, ROOT)}"}
    try:
        meta = np.load(sparse.WEIGHTS)
        net = sparse.load(sparse.WEIGHTS)
        summary, _ = sparse.evaluate(net, volumes)
        summary.update({"nrmse_bar": sparse.NRMSE_BAR, "eval_seeds": f"{sparse.EVAL_SEED0}..",
                        "network_parameters": net.param_count, "trained_phantoms": int(meta["phantoms"]),
                        "trained_epochs": int(meta["epochs"]),
                        "workload": "rca128 full 128-tx vs sparse 32-tx (every 4th row), 128^3, cubic, no CF"})
        net.close()
        return summary
    except Exception as exc:  # the learned path must not hide the plain pipeline's number
        return {"failed": str(exc)}


def batched_stream(n_frames, seed=4):
    """Config 4: a seeded stream of frames of mixed size (transmits 32/64/128, channels 64/128,
    samples 1024-8192, volumes 64^3 / 128^2 x 128 / 128^2 x 256), simulated on the GPU. Times the
    frame-by-frame path (per-frame plans: decode, Hilbert, delay-and-sum launches) against one
    cutb_batch run replayed from its CUDA graph (front ends + one persistent delay-and-sum per
    kernel variant), tile shapes from the autotuner, inputs resident in HBM."""
    import torch
    from cuda_ultrasound_toolkit_b200 import Batch, Plan, batched
    from cuda_ultrasound_toolkit_b200.tune import DasTuner
    specs = batched.frame_specs(seed, n_frames)
    frames = batched.make_frames(specs)
    params = [bp for _, bp in frames]
    raws = [r for r, _ in frames]
    t0 = time.perf_counter()
    tuner = DasTuner(reps=2)
    tiles = [tuner.choose(bp) for bp in params]
    tuning_s = time.perf_counter() - t0
    plans = [Plan(bp, das_tile=t) for bp, t in zip(params, tiles)]
    n_dec = max(p.empty_decoded().numel() for p in plans)
    dec = torch.empty(n_dec, dtype=torch.float32, device="cuda")
    iq = torch.empty(n_dec, dtype=torch.complex64, device="cuda")
    batch = Batch(params, das_tiles=tiles)
    vols = batch.empty_volumes()

    def loop():
        for p, r, v in zip(plans, raws, vols):
            S, C, T = p.bp.dims
            d = dec[:T * C * S].view(T, C, S)
            q = iq[:T * C * S].view(T, C, S)
            p.decode(r, out=d)
            p.hilbert(d, out=q)
            p.das(q, out=v)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    loop_ms = timed(loop, 2)
    for p in plans:
        p.check()
    batch_ms = timed(lambda: batch.run(raws, vols, graph=True), 3)
    batch.check()
    work = batched.work(params)
    return {"frames": n_frames, "seed": seed, "voxel_transmit_channel": work,
            "frame_loop": {"ms": loop_ms, "volumes_per_s": 1e3 * n_frames / loop_ms,
                           "launches": 3 * n_frames},
            "batched_graph": {"ms": batch_ms, "volumes_per_s": 1e3 * n_frames / batch_ms,
                              "launches": batch.launches_per_run, "das_launches": batch.das_launches,
                              "vct_per_s": work / (batch_ms * 1e-3)},
            "speedup": loop_ms / batch_ms, "tile_choice": {str(t): tiles.count(t) for t in set(tiles)},
            "tuning_seconds": tuning_s}


def precision_form(seed=3000):
    """Config 3: 256 transmits x 256 channels x 8192 samples (1 GiB of int16, simulated on the
    GPU), 128 x 128 x 256 volume, linear, no coherence factor. Decode on int8 tensor cores (hi/lo
    byte split) checked bit-exact against the FWHT decode; analytic signal stored as FP32 and as
    BF16, each compared with the FP64 oracle on 64 sampled rows; volumes from both storages."""
    import torch
    from cuda_ultrasound_toolkit_b200 import Plan, synth
    from cuda_ultrasound_toolkit_b200.simulate import Simulator
    from oracle import oracle as O
    w = synth.CONFIGS["precision"]
    rng = np.random.default_rng(seed)
    cmap = rng.permutation(w.C).astype(np.int16)
    scat = synth.phantom(rng, w.scatterers, 0, box_xy=w.box_xy, z_range=w.z_range)
    raw, _ = Simulator(w.T, w.C, w.S).run(scat, cmap, seed)
    bp = synth.make_params(w, channel_map=cmap)
    p_tc, p_fw, p_bf = Plan(bp, decode_tc=True), Plan(bp), Plan(bp, decode_tc=True, iq_bf16=True)

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    dec_tc, dec_fw = p_tc.empty_decoded(), p_fw.empty_decoded()
    tc_ms = timed(lambda: p_tc.decode(raw, out=dec_tc))
    fw_ms = timed(lambda: p_fw.decode(raw, out=dec_fw))
    exact = bool(torch.equal(dec_tc, dec_fw))
    del dec_fw
    iq32, iq16 = p_tc.empty_iq(), p_bf.empty_iq()
    hil32_ms = timed(lambda: p_tc.hilbert(dec_tc, out=iq32))
    hil16_ms = timed(lambda: p_bf.hilbert(dec_tc, out=iq16))
    rows = np.sort(rng.choice(w.T * w.C, 64, replace=False))
    d = dec_tc.view(w.T * w.C, w.S)[torch.from_numpy(rows).cuda()].double().cpu().numpy()
    ref = O.hilbert(d.reshape(1, 64, w.S)).reshape(64, w.S)
    g32 = iq32.view(w.T * w.C, w.S)[torch.from_numpy(rows).cuda()].cpu().numpy()
    g16 = iq16.view(w.T * w.C, w.S, 2)[torch.from_numpy(rows).cuda()].float().cpu().numpy()
    g16 = g16[..., 0] + 1j * g16[..., 1]
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    vol32, vol16 = p_tc.empty_volume(), p_bf.empty_volume()
    das32_ms = timed(lambda: p_tc.das(iq32, out=vol32), 2)
    das16_ms = timed(lambda: p_bf.das(iq16, out=vol16), 2)
    p_tc.check()
    p_bf.check()
    vol_rel = float(torch.linalg.vector_norm(vol16 - vol32) / torch.linalg.vector_norm(vol32))
    # both volumes on a seeded voxel sample against the FP64 oracle's pipeline of the same frame
    z, y, x = bp.volume_shape
    vox = np.sort(rng.choice(x * y * z, 4096, replace=False))
    ref_vox, _, _ = O.pipeline(raw.cpu().numpy(), bp, voxels=vox, threads=os.cpu_count() or 1)
    pick = torch.from_numpy(vox).cuda()
    v32 = vol32.reshape(-1)[pick].cpu().numpy()
    v16 = vol16.reshape(-1)[pick].cpu().numpy()
    dec_bytes = w.T * w.C * w.S * 6
    return {"workload": "rca256 precision: 256 tx x 256 ch x 8192 samples -> 128x128x256, linear, no CF",
            "decode_tc": {"ms": tc_ms, "bit_exact_vs_fwht": exact, "achieved_gbs": dec_bytes / tc_ms / 1e6},
            "decode_fwht": {"ms": fw_ms, "achieved_gbs": dec_bytes / fw_ms / 1e6},
            "analytic_signal": {"fp32": {"rel_l2_vs_fp64": rel(g32, ref), "hilbert_ms": hil32_ms},
                                "bf16": {"rel_l2_vs_fp64": rel(g16, ref), "hilbert_ms": hil16_ms},
                                "sample": "64 random rows of 65536, FP64 oracle Hilbert of the same decoded rows"},
            "volume": {"das_ms_fp32_iq": das32_ms, "das_ms_bf16_iq": das16_ms,
                       "bf16_vs_fp32_iq_rel_l2": vol_rel,
                       "fp32_iq_rel_l2_vs_fp64": rel(v32, ref_vox), "bf16_iq_rel_l2_vs_fp64": rel(v16, ref_vox),
                       "fp64_sample": "4096 seeded voxels, FP64 oracle decode -> Hilbert -> delay-and-sum",
                       "volumes_per_s_fp32_iq": 1e3 / (tc_ms + hil32_ms + das32_ms),
                       "volumes_per_s_bf16_iq": 1e3 / (tc_ms + hil16_ms + das16_ms)}}


def motion_section(reps=10, warmup=3):
    """NCC block-matching motion detection: 16 B-mode-like frames of 512 x 512 (8-bit speckle,
    translated up to 10 px), 32-pixel patches every 16 px (32 x 32 grid), +-16 px search (33 x 33
    maps), every frame against frame 0. Ours: one fused launch over resident frames (device) and
    cuda_toolkit::motion_detection with host frames (e2e); upstream's own GPU pipeline (its sources
    built with NPP, oracle/_ref/libncc_ref.so) on the same host frames when it was built; the FP64
    oracle on one frame pair as the CPU baseline. Inputs (16 MiB) fit in L2; the kernel is
    compute-bound (FP32 correlation numerator)."""
    import ctypes
    import time
    import torch
    from cuda_ultrasound_toolkit_b200 import api
    from cuda_ultrasound_toolkit_b200.params import NccMotionParameters
    from oracle import oracle as O
    from cuda_ultrasound_toolkit_b200.synth import motion_workload
    W = H = 512
    F, P, sp, G, M = 16, 32, 16, 32, 16
    frames, p = motion_workload(F, W, P, sp, G, M)
    vectors = (F - 1) * G * G
    # algorithmic FLOPs of the correlation numerators (2 per template pixel per map position),
    # window by window with the border clipping
    flops = 0
    for i in range(G):
        for j in range(G):
            t0, l0 = i * sp - P // 2, j * sp - P // 2
            th = min(t0 + P - 1, H - 1) - max(t0, 0) + 1
            tw = min(l0 + P - 1, W - 1) - max(l0, 0) + 1
            sh = min(t0 + P - 1 + M, H - 1) - max(t0 - M, 0) + 1
            sw = min(l0 + P - 1 + M, W - 1) - max(l0 - M, 0) + 1
            flops += 2 * tw * th * (sw - tw + 1) * (sh - th + 1)
    flops *= F - 1
    d_frames = torch.from_numpy(frames).cuda()
    d_maps = torch.empty((F, G, G, 4), dtype=torch.float32, device="cuda")
    for _ in range(warmup):
        api.motion_detection_device(d_frames, p, out=d_maps)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        api.motion_detection_device(d_frames, p, out=d_maps)
    b.record()
    torch.cuda.synchronize()
    dev_ms = a.elapsed_time(b) / reps
    ours = d_maps.cpu().numpy()
    host_maps = np.empty_like(ours)
    api.motion_detection(frames, p, out=host_maps)
    t = time.perf_counter()
    for _ in range(reps):
        api.motion_detection(frames, p, out=host_maps)
    e2e_ms = (time.perf_counter() - t) / reps * 1e3
    fp32 = api.calibrate_fp32()
    out = {"workload": f"{F} frames {W}x{H}, patch {P}, grid {G}x{G} every {sp} px, margins {M} "
                       f"({2 * M + 1}x{2 * M + 1} maps), reference frame 0",
           "vectors": vectors, "device_ms": dev_ms, "vectors_per_s": vectors / dev_ms * 1e3,
           "e2e": {"ms": e2e_ms, "vectors_per_s": vectors / e2e_ms * 1e3, "h2d_bytes": frames.nbytes,
                   "d2h_bytes": ours.nbytes, "api": "cuda_toolkit::motion_detection (host spans)"},
           "roofline": {"bound": "fp32", "achieved_tflops": flops / dev_ms / 1e9, "peak_tflops": fp32,
                        "frac": flops / dev_ms / 1e9 / fp32, "flops_per_launch": flops,
                        "peak_source": "measured FP32 FMA probe (cutb_calibrate_fp32) on this GPU"},
           "gpu_launches_per_call": 2, "host_equals_device": bool(np.array_equal(ours, host_maps))}
    ref_lib = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "_ref", "libncc_ref.so")
    if os.path.exists(ref_lib):
        # upstream's own pipeline (NPP + CUB kernels, three launches per grid point); it prints
        # progress on stdout, which is silenced around the call
        L = ctypes.CDLL(ref_lib)
        fp = ctypes.POINTER(ctypes.c_float)
        L.ref_motion_detection.argtypes = [fp, ctypes.POINTER(NccMotionParameters), fp]
        ref_maps = np.zeros_like(ours)
        sys.stdout.flush()
        saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        try:
            os.dup2(devnull, 1)
            L.ref_motion_detection(frames.ctypes.data_as(fp), ctypes.byref(p), ref_maps.ctypes.data_as(fp))
            t = time.perf_counter()
            rc = L.ref_motion_detection(frames.ctypes.data_as(fp), ctypes.byref(p), ref_maps.ctypes.data_as(fp))
            ref_ms = (time.perf_counter() - t) * 1e3
        finally:
            os.dup2(saved, 1)
            os.close(saved)
            os.close(devnull)
        d = np.abs(ours - ref_maps)
        out["upstream_gpu"] = {"ms": ref_ms, "vectors_per_s": vectors / ref_ms * 1e3, "rc": int(rc),
                               "kind": "upstream image_processor.cpp + block_match_kernels.cu on NPP, host frames",
                               "max_abs_diff_peak": float(d[..., 2:].max()),
                               "max_abs_diff_offset": float(d[..., :2].max()),
                               "same_accept_reject": bool(((ours[..., 2] > 0) == (ref_maps[..., 2] > 0)).all())}
    t = time.perf_counter()
    sub = NccMotionParameters.make(**{**p.as_dict(), "frame_count": 2})
    O.motion_detection(frames[:2], sub, threads=os.cpu_count() or 1)
    cpu_s = time.perf_counter() - t
    out["cpu_baseline"] = {"vectors_per_s": G * G / cpu_s, "cores": os.cpu_count() or 1, "kind": "port",
                           "sample": f"FP64 oracle, frames 0-1 ({G * G} vectors)"}
    return out


def _event_ms(fn, reps, warmup):
    """Mean device time of fn() over reps calls (CUDA events on the current stream)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


_FP32 = []


def calibrate_fp32_cached():
    """The measured FP32 FMA rate (TFLOP/s), probed once per process."""
    if not _FP32:
        from cuda_ultrasound_toolkit_b200.api import calibrate_fp32
        _FP32.append(calibrate_fp32())
    return _FP32[0]


def sequences_section(reps=5, warmup=3, seed=11):
    """The other live sequences and the bandpass input, each on the GPU with the FP64 oracle timed
    beside it on a bounded sample.

    TPW (RCA_TPW, tilted plane waves in the x-z plane, IQ phase rotation) and UFORCES (sparse
    transmit elements, focus at 30 mm): 64 transmits x 128 channels x 2048 samples of analytic
    signal resident in HBM -> 256 x 1 x 512 (x, y, z), cubic + coherence factor; one thread per
    voxel, y-invariant. Bandpass: 128 transmits x 128 channels of 4096 complex samples sent as
    8192 interleaved int16 IQ values, Hadamard-encoded, 64-tap filter; exact decode of the raw
    pairs, then demodulation + filter, both HBM-bound."""
    import torch
    from cuda_ultrasound_toolkit_b200 import Plan, synth
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    out = {}
    T, C, S, X, Z = 64, 128, 2048, 256, 512
    # "tpw" / "uforces": the volume spans the whole aperture (x step 0.15 mm: the staged windows of a
    # 32-voxel-wide tile overflow, so the default engine is one thread per voxel); "_fine": a 9.6 mm
    # wide volume (x step 0.038 mm), on the staged engine
    for name in ("tpw", "uforces", "tpw_fine", "uforces_fine"):
        bp = synth.sequence_params(name, T, C, S, X, Z)
        half = -bp.output_min_coordinate[0]
        used = T if name.startswith("tpw") else T - 1  # UFORCES: transmit row 0 (the flash) is not summed
        plan = Plan(bp)
        iq = torch.complex(torch.randn(T, C, S, device="cuda"), torch.randn(T, C, S, device="cuda"))
        vol = plan.empty_volume()
        ms = _event_ms(lambda: plan.das(iq, out=vol), reps, warmup)
        plan.check()
        direct = Plan(bp, das_tile=3)  # the one-thread-per-voxel kernel, for comparison
        vol_d = direct.empty_volume()
        direct_ms = _event_ms(lambda: direct.das(iq, out=vol_d), reps, warmup)
        direct.check()
        vtc = X * Z * used * C
        n_vox = 256
        vox = rng.choice(X * Z, n_vox, replace=False)
        iq_h = iq.cpu().numpy().astype(np.complex128)
        t0 = time.perf_counter()
        ref = O.das(iq_h, bp, vox, threads)
        cpu_s = time.perf_counter() - t0
        got = vol.cpu().numpy().reshape(-1)[vox]
        engine = "one thread per voxel (das_direct.cu)" if plan.tile_shape == (1, 1, 1) else "staged windows (das.cu)"
        out[name] = {"workload": f"{T} tx x {C} ch x {S} samples -> {X} x 1 x {Z} over x in +-{half * 1e3:.1f} mm, "
                                 "cubic + CF",
                     "device_ms": ms, "vtc_per_s": vtc / ms * 1e3, "engine": engine,
                     "one_thread_per_voxel_ms": direct_ms,
                     "fp32_frac": vtc * 49 / (ms * 1e-3) / 1e12 / calibrate_fp32_cached(),
                     "rel_l2_vs_fp64_sample": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
                     "cpu_baseline": {"vtc_per_s": n_vox * used * C / cpu_s, "cores": threads, "kind": "port",
                                      "sample": f"FP64 oracle, {n_vox} random voxels"}}
        del iq, iq_h
    T, C, S, ntaps = 128, 128, 4096, 64
    w = synth.Workload("bandpass", T, C, S, 64, 64, 64, 0, cubic=True, cf=0.0)
    bp = synth.make_params(w)
    bp.rf_raw_dim[0] = 2 * T * S
    bp.sample_type = 1
    taps = synth.chirp_taps(ntaps)
    bp.filter_length = ntaps
    for i, v in enumerate(taps):
        bp.rf_filter[i] = float(v)
    plan = Plan(bp)
    raw = torch.randint(-32768, 32768, (C, 2 * T * S), dtype=torch.int16, device="cuda")
    dec, iqb = plan.empty_decoded(), plan.empty_iq()
    dec_ms = _event_ms(lambda: plan.decode(raw, out=dec), reps, warmup)
    dem_ms = _event_ms(lambda: plan.hilbert(dec, out=iqb), reps, warmup)
    plan.check()
    hbm, peak_src = measured_peaks()
    hbm = hbm["hbm_gbs"]
    dec_bytes, dem_bytes = T * C * 2 * S * (2 + 4), T * C * S * (2 * 4 + 8)
    sub_c = 8
    sub = bp.copy()
    sub.rf_raw_dim[1] = sub_c
    sub.dec_data_dim[1] = sub_c
    for c in range(sub_c):
        sub.channel_mapping[c] = c
    raw_h = raw[:sub_c].cpu().numpy()
    t0 = time.perf_counter()
    O.convert_demod(raw_h, sub, taps)
    cpu_s = time.perf_counter() - t0
    out["bandpass"] = {
        "workload": f"{T} tx x {C} ch x {S} complex samples (int16 IQ pairs), Hadamard, {ntaps}-tap filter",
        "decode": {"ms": dec_ms, "achieved_gbs": dec_bytes / dec_ms / 1e6, "frac": dec_bytes / dec_ms / 1e6 / hbm,
                   "bytes": dec_bytes},
        "demod_filter": {"ms": dem_ms, "achieved_gbs": dem_bytes / dem_ms / 1e6,
                         "frac": dem_bytes / dem_ms / 1e6 / hbm, "bytes": dem_bytes},
        "peak_gbs": hbm, "peak_note": peak_src,
        "cpu_baseline": {"ms_per_frame": cpu_s * 1e3 * C / sub_c, "cores": 1, "kind": "port",
                         "sample": f"FP64 oracle on {sub_c} of {C} channels, scaled"}}
    return out


def transfer_section(reps=5):
    """The out-of-process path on the full workload: beamform_i16 from libcuda_transfer.so to a
    cutb_transfer_server process (shared-memory input and output, command socket), against the
    same request through cuda_toolkit::beamform in this process. Wall-clock per volume, both
    with host buffers."""
    import time
    import uuid
    from cuda_ultrasound_toolkit_b200 import api, synth, transfer
    raw, bp = synth.frame("full")
    name = "cutbb" + uuid.uuid4().hex[:8]
    os.environ["CUDA_TRANSFER_NAME"] = name
    transfer.set_timeout_ms(600000)
    proc = transfer.spawn_server(name, data_bytes=256 << 20, timeout_ms=600000)
    try:
        out = np.empty(bp.volume_shape, np.complex64)
        transfer.beamform_i16(raw, bp, out=out)
        t = time.perf_counter()
        for _ in range(reps):
            transfer.beamform_i16(raw, bp, out=out)
        ipc_ms = (time.perf_counter() - t) / reps * 1e3
    finally:
        transfer.deinit()
        proc.terminate()
        proc.wait(30)
        os.environ.pop("CUDA_TRANSFER_NAME", None)
    ref = api.beamform(raw, bp)
    t = time.perf_counter()
    for _ in range(reps):
        api.beamform(raw, bp, out=ref)
    direct_ms = (time.perf_counter() - t) / reps * 1e3
    return {"workload": "full frame via the command socket + shared memory to a server process",
            "ipc_ms": ipc_ms, "ipc_volumes_per_s": 1e3 / ipc_ms, "direct_ms": direct_ms,
            "direct_volumes_per_s": 1e3 / direct_ms, "identical": bool(np.array_equal(out, ref)),
            "bytes_in": int(raw.nbytes), "bytes_out": int(out.nbytes)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--learned", type=int, default=16,
                    help="held-out volumes for the learned sparse-transmit path (0: skip)")
    ap.add_argument("--batched", type=int, default=64, help="frames of the batched mixed-size stream (0: skip)")
    ap.add_argument("--precision", type=int, default=1, help="run the 256 x 256 x 8192 precision form (0: skip)")
    ap.add_argument("--motion", type=int, default=1, help="run the NCC motion-detection section (0: skip)")
    ap.add_argument("--transfer", type=int, default=1, help="run the out-of-process transfer section (0: skip)")
    ap.add_argument("--sequences", type=int, default=1,
                    help="run the TPW / UFORCES / bandpass section (0: skip)")
    ap.add_argument("--upstream", type=int, default=1,
                    help="time upstream's own CUDA build on the same frame, when built in baseline/_ref (0: skip)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
