"""GPU RF simulator against its CPU float64 restatement (oracle/sim_ref.py) on small frames.

The GPU accumulates echoes in FP32 with a recurrence for the pulse, so the noisy encoded
signal is compared by relative L2 error and the int16 frame may differ by one LSB where the
FP32 value lands next to a rounding boundary.
"""
import numpy as np
import pytest
import torch

from cuda_ultrasound_toolkit_b200 import synth
from cuda_ultrasound_toolkit_b200.simulate import Simulator

pytestmark = pytest.mark.gpu

TOL_SIGNAL = 2e-5


CASES = [
    # T, G (rows per transmit), stride, offset, C, S, scatterers, speckle, snr_db, hadamard
    (16, 1, 0, 0, 8, 1024, 12, 0, 40.0, True),
    (8, 4, 0, 0, 16, 2048, 20, 200, 40.0, True),
    (8, 1, 4, 2, 16, 2048, 20, 200, 40.0, True),
    (32, 1, 0, 0, 12, 512, 5, 50, 1000.0, False),
]


@pytest.mark.parametrize("T,G,stride,offset,C,S,npts,nspk,snr,had", CASES)
def test_simulator_matches_cpu(T, G, stride, offset, C, S, npts, nspk, snr, had):
    from oracle import sim_ref
    rng = np.random.default_rng(T * 100 + C)
    scat = synth.phantom(rng, npts, nspk, box_xy=2e-3, z_range=(3e-3, 8e-3))
    cmap = rng.permutation(C).astype(np.int16)
    sim = Simulator(T, C, S, rows_per_transmit=G, snr_db=snr, hadamard=had, row_stride=stride, row_offset=offset)
    raw, gain = sim.run(scat, cmap, seed=1234 + T)
    sig = sim.signal().cpu().numpy()
    raw = raw.cpu().numpy()
    ref_raw, ref_sig, ref_gain = sim_ref.simulate(scat, cmap, 1234 + T, T, G, C, S, synth.PITCH, synth.FS, synth.FC,
                                                  synth.C_SOUND, snr_db=snr, encoding=1 if had else 0, stride=stride,
                                                  offset=offset)
    err = np.linalg.norm(sig - ref_sig) / np.linalg.norm(ref_sig)
    assert err < TOL_SIGNAL, err
    assert abs(float(gain.item()) - ref_gain) < 1e-5 * ref_gain
    d = np.abs(raw.astype(np.int32) - ref_raw.astype(np.int32))
    assert d.max() <= 1
    assert np.count_nonzero(d) <= 1e-2 * d.size


def test_simulator_matches_numpy_generator():
    """Without noise or channel permutation, one transmit per row: the same echoes as the
    numpy generator that the pipeline benchmarks use."""
    w = synth.Workload("t", 8, 8, 1024, 4, 4, 4, 10, cubic=True, cf=0.0, box_xy=2e-3, z_range=(3e-3, 8e-3))
    rng = np.random.default_rng(5)
    pos, amp = synth.scatterer_field(w, rng)
    scat = np.concatenate([pos, amp[:, None]], axis=1).astype(np.float32)
    sim = Simulator(8, 8, 1024, snr_db=1000.0, hadamard=False)
    sim.run(scat, np.arange(8), seed=0)
    got = sim.signal().cpu().numpy()
    ref = synth.echoes(w, scat[:, :3].astype(np.float64), scat[:, 3].astype(np.float64))
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < TOL_SIGNAL


def test_simulator_rejects_bad_channel_map():
    from cuda_ultrasound_toolkit_b200 import CutbError
    sim = Simulator(4, 4, 256)
    with pytest.raises(CutbError):
        sim.run(np.zeros((1, 4), np.float32), np.array([0, 1, 2, 4]), seed=0)
