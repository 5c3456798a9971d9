"""Batched beamforming (cutb_batch: persistent delay-and-sum over many frames, CUDA graph replay)
and the tile autotuner.

The batch runs the same per-tile code as the single-frame path, so every frame's volume must be
bit-identical to cutb_beamform of that frame alone, with or without the graph.
"""
import numpy as np
import pytest
import torch

from cuda_ultrasound_toolkit_b200 import Batch, Plan, batched
from cuda_ultrasound_toolkit_b200.tune import DasTuner, candidates, schedules

pytestmark = pytest.mark.gpu

SPECS = [
    dict(T=8, C=8, S=512, X=20, Y=9, Z=40, scatterers=10, seed=1),
    dict(T=16, C=16, S=1024, X=16, Y=16, Z=24, scatterers=30, seed=2),
    dict(T=8, C=16, S=512, X=33, Y=3, Z=70, scatterers=12, seed=3),     # partial tiles in every direction
    dict(T=16, C=8, S=1024, X=12, Y=12, Z=12, scatterers=5, seed=4),
    dict(T=8, C=8, S=512, X=20, Y=9, Z=40, scatterers=17, seed=5),       # same parameters as frame 0
    dict(T=32, C=16, S=2048, X=24, Y=16, Z=64, scatterers=40, seed=6),
]


@pytest.fixture(scope="module")
def frames():
    return batched.make_frames(SPECS)


def reference(frames, tiles=None):
    out = []
    for k, (raw, bp) in enumerate(frames):
        plan = Plan(bp, das_tile=0 if tiles is None else tiles[k])
        out.append(plan.beamform(raw))
        plan.check()
    return out


def test_batch_equals_single_frames(frames):
    b = Batch([bp for _, bp in frames])
    vols = b.run([r for r, _ in frames])
    b.check()
    for v, ref in zip(vols, reference(frames)):
        assert torch.equal(v, ref)
    assert b.launches_per_run == 2 * len(frames) + b.das_launches
    assert 1 <= b.das_launches <= 2


def test_batch_graph_replay(frames):
    b = Batch([bp for _, bp in frames])
    raws = [r for r, _ in frames]
    vols = b.empty_volumes()
    ref = [v.clone() for v in b.run(raws, vols)]
    for _ in range(3):
        for v in vols:
            v.zero_()
        b.run(raws, vols, graph=True)
        b.check()
        for v, r in zip(vols, ref):
            assert torch.equal(v, r)
    # new output buffers: the graph is captured again for the new pointers
    vols2 = b.run(raws, graph=True)
    b.check()
    for v, r in zip(vols2, ref):
        assert torch.equal(v, r)


def test_batch_mixed_tiles(frames):
    tiles = [1, 2, 2, 1, 2, 1]
    b = Batch([bp for _, bp in frames], das_tiles=tiles)
    assert b.das_launches == 2
    vols = b.run([r for r, _ in frames], graph=True)
    b.check()
    for v, ref in zip(vols, reference(frames, tiles)):
        assert torch.equal(v, ref)


def test_batch_direct_and_persistent_frames():
    """A frame with a full wave of tiles (64 x 64 x 128: 512 tiles >= 148 SMs x 3 CTAs) runs its own
    grid launch on a side stream, the small frames one persistent launch on the other; every
    volume still equals the single-frame path, with and without the graph."""
    specs = [dict(T=8, C=8, S=1024, X=64, Y=64, Z=128, scatterers=20, seed=11), SPECS[0], SPECS[3]]
    fr = batched.make_frames(specs)
    b = Batch([bp for _, bp in fr])
    assert b.das_launches == 2
    assert b.launches_per_run == 2 * len(fr) + 2
    raws = [r for r, _ in fr]
    ref = reference(fr)
    for graph in (False, True, True):
        vols = b.run(raws, graph=graph)
        b.check()
        for v, r in zip(vols, ref):
            assert torch.equal(v, r)


def test_tuner_choice_is_fastest_on_remeasure(tmp_path):
    spec = dict(T=32, C=64, S=2048, X=64, Y=64, Z=64, scatterers=50, seed=9)
    bp = batched.make_frames([spec])[0][1]
    tuner = DasTuner(str(tmp_path / "tiles.json"), reps=3)
    cfg = tuner.choose_config(bp)
    entry = tuner.entry(bp)
    # every tile x schedule was timed, and rows per stage at the best of them
    assert {f"tile{t}/schedule{s}/rows0" for t in candidates(bp) for s in schedules(bp, t)} <= set(entry["ms"])
    assert any(k.endswith("rows4") for k in entry["ms"])
    times = {(t, s): tuner.measure(bp, t, schedule=s, reps=5) for t in candidates(bp) for s in schedules(bp, t)}
    chosen = tuner.measure(bp, cfg["das_tile"], schedule=cfg["das_schedule"], rows=cfg["das_rows_per_stage"], reps=5)
    assert chosen <= 1.1 * min(times.values()), (cfg, chosen, times)
    # 32 transmits and 2048 samples: both decode engines run; the faster one is kept
    assert set(entry["decode_ms"]) == {"False", "True"}
    dec = {tc: tuner.measure_decode(bp, tc, reps=5) for tc in (False, True)}
    assert dec[cfg["decode_tc"]] <= 1.15 * min(dec.values()), (cfg, dec)
    assert tuner.choose(bp) == cfg["das_tile"]
    # persisted and reloaded without measuring again
    again = DasTuner(str(tmp_path / "tiles.json"))
    assert again.choose_config(bp) == cfg
    Plan(bp, **cfg).close()


@pytest.mark.parametrize("half", [19.2e-3, 2.4e-3])  # a coarse grid over the aperture, a fine one
def test_tuner_picks_the_engine_for_tpw(tmp_path, half):
    """For tilted plane waves the tuner times the staged engine against one thread per voxel."""
    import numpy as np
    from cuda_ultrasound_toolkit_b200 import SequenceId, synth
    w = synth.Workload("tpw", 32, 64, 1024, 128, 1, 128, 0, cubic=True, cf=1.0, z_range=(5e-3, 20e-3))
    bp = synth.make_params(w)
    bp.das_shader_id = int(SequenceId.RCA_TPW)
    bp.tx_orientation = bp.rx_orientation
    bp.output_min_coordinate[0], bp.output_max_coordinate[0] = -half, half
    bp.fn_rx = 1.0
    for t, a in enumerate(np.linspace(-0.2, 0.2, 32)):
        bp.foci[3 * t + 2] = float(a)
    tuner = DasTuner(str(tmp_path / "tiles.json"), reps=3)
    cfg = tuner.choose_config(bp)
    assert cfg["das_tile"] in candidates(bp) == (2, 3)
    times = {(t, s): tuner.measure(bp, t, schedule=s, reps=5) for t in candidates(bp) for s in schedules(bp, t)}
    chosen = tuner.measure(bp, cfg["das_tile"], schedule=cfg["das_schedule"], rows=cfg["das_rows_per_stage"], reps=5)
    assert chosen <= 1.15 * min(times.values()), (cfg, chosen, times)
