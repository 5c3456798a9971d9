"""Closed-form known answers that pin the CPU oracle (no GPU)."""
import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200 import synth
from cuda_ultrasound_toolkit_b200.params import CudaBeamformerParameters, EncodingMatrix


SUPPORTED = [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 12, 24, 48, 96, 192, 384, 768, 20, 40, 80, 160, 320, 640]


@pytest.mark.parametrize("n", SUPPORTED)
def test_hadamard_orthogonal(orc, n):
    for ordering in (1, 2):
        h = orc.encoding_matrix(n, ordering).astype(np.int64)
        assert (h @ h.T == n * np.eye(n, dtype=np.int64)).all()


def test_walsh_is_sequency_sorted(orc):
    for n in (8, 64, 256):
        w = orc.encoding_matrix(n, 2)
        flips = (w[:, 1:] != w[:, :-1]).sum(axis=1)
        assert (flips == np.arange(n)).all()


def test_unsupported_orders(orc):
    for n in (0, 3, 36, 60, 1025):
        with pytest.raises(ValueError):
            orc.encoding_matrix(n, 1)


def _bp(S, C, T, R0=None, R1=None, decode=EncodingMatrix.HADAMARD, cmap=None):
    bp = CudaBeamformerParameters()
    bp.rf_raw_dim[0] = R0 if R0 is not None else S * T
    bp.rf_raw_dim[1] = R1 if R1 is not None else C
    bp.dec_data_dim[0], bp.dec_data_dim[1], bp.dec_data_dim[2] = S, C, T
    bp.decode = int(decode)
    for c in range(C):
        bp.channel_mapping[c] = int(cmap[c]) if cmap is not None else c
    return bp


@pytest.mark.parametrize("T,ordering", [(8, 1), (16, 2), (12, 1), (20, 2), (64, 1)])
def test_decode_inverts_encoding(orc, T, ordering):
    """decode(H^T x) == x exactly (H H^T = T I)."""
    rng = np.random.default_rng(T)
    S, C = 32, 3
    x = rng.integers(-200, 200, size=(T, C, S)).astype(np.int64)
    h = orc.encoding_matrix(T, ordering).astype(np.int64)
    enc = np.einsum("kt,kcs->tcs", h, x)          # H^T x
    cmap = np.array([2, 0, 1])
    raw = np.zeros((C, T, S), dtype=np.int16)
    raw[cmap] = enc.transpose(1, 0, 2)
    out = orc.decode_i16(raw.reshape(C, T * S), _bp(S, C, T, decode=ordering, cmap=cmap))
    assert (out == x.astype(np.float32)).all()


def test_decode_bit_exact_formula_and_padding(orc):
    """Non-power-of-two order: out = fl32(fl32(1/T) * sum); rows longer than T*S (padding)."""
    rng = np.random.default_rng(7)
    S, C, T, pad = 16, 4, 12, 5
    R0, R1 = T * S + pad, 6
    raw = rng.integers(-32768, 32767, size=(R1, R0), dtype=np.int16)
    cmap = np.array([5, 1, 3, 0])
    out = orc.decode_i16(raw, _bp(S, C, T, R0, R1, cmap=cmap))
    h = orc.encoding_matrix(T, 1).astype(np.int64)
    x = raw[cmap, : T * S].reshape(C, T, S).astype(np.int64)
    acc = np.einsum("ut,cts->ucs", h, x)
    ref = np.float32(1.0 / np.float32(T)) * acc.astype(np.float32)
    assert (out == ref).all()


def test_convert_only(orc):
    rng = np.random.default_rng(3)
    S, C, T = 8, 3, 5
    raw = rng.integers(-1000, 1000, size=(C, T * S), dtype=np.int16)
    cmap = np.array([1, 2, 0])
    out = orc.decode_i16(raw, _bp(S, C, T, decode=EncodingMatrix.NONE, cmap=cmap))
    assert (out == raw[cmap].reshape(C, T, S).transpose(1, 0, 2)).all()


@pytest.mark.parametrize("N", [16, 64, 256])
def test_hilbert_known_answers(orc, N):
    n = np.arange(N)
    for k in (1, 3, N // 4):
        iq = orc.hilbert(np.cos(2 * np.pi * k * n / N)[None])[0]
        np.testing.assert_allclose(iq, 0.75 * np.exp(2j * np.pi * k * n / N), atol=1e-12)
    np.testing.assert_allclose(orc.hilbert(np.ones((1, N)))[0], 0.75, atol=1e-12)        # DC: 0.75
    np.testing.assert_allclose(orc.hilbert(((-1.0) ** n)[None])[0], 1.5 * (-1.0) ** n, atol=1e-12)  # Nyquist kept


def test_hilbert_filter_is_circular_convolution(orc):
    rng = np.random.default_rng(1)
    N, L = 64, 9
    x = rng.normal(size=N)
    h = rng.normal(size=L).astype(np.float32)
    conv = np.array([sum(float(h[j]) * x[(i - j) % N] for j in range(L)) for i in range(N)])
    np.testing.assert_allclose(orc.hilbert(x[None], h)[0], orc.hilbert(conv[None])[0], atol=1e-10)


def test_das_focuses_point_scatterer(orc):
    w = synth.CONFIGS["small"]
    raw, cmap, pos, amp = synth.synth_frame(w, 11)
    bp = synth.make_params(w, channel_map=cmap)
    dec = orc.decode_f64(raw, bp)
    iq = orc.hilbert(dec)
    res = 18e-3 / (w.X - 1)
    for p in pos[:3]:
        xi, yi = (int(round((p[k] + 9e-3) / res)) for k in (0, 1))
        zi = int(round((p[2] - 10e-3) / (30e-3 / (w.Z - 1))))
        zs = np.arange(max(0, zi - 6), min(w.Z, zi + 7))
        v = orc.das(iq, bp, (zs * w.Y + yi) * w.X + xi)
        assert abs(int(zs[np.argmax(np.abs(v))]) - zi) <= 1


def test_das_is_linear(orc):
    w = synth.CONFIGS["small"]
    bp = synth.make_params(w)
    rng = np.random.default_rng(5)
    shape = (w.T, w.C, w.S)
    a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    b = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    vox = rng.integers(0, w.X * w.Y * w.Z, 16)
    np.testing.assert_allclose(orc.das(a + 2 * b, bp, vox), orc.das(a, bp, vox) + 2 * orc.das(b, bp, vox),
                               rtol=1e-10, atol=1e-9)


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors published with Random123 (Salmon et al., SC 2011)."""
    from oracle import sim_ref
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in cases:
        got = sim_ref.philox4x32_10(*[np.array([c], dtype=np.uint64) for c in ctr], *key)
        assert tuple(int(g[0]) for g in got) == want


def test_sim_ref_matches_numpy_generator():
    """The simulator restatement without noise/encoding equals synth.echoes (one row per transmit)."""
    from oracle import sim_ref
    from cuda_ultrasound_toolkit_b200 import synth
    w = synth.Workload("t", 8, 6, 512, 4, 4, 4, 7, cubic=True, cf=0.0, box_xy=2e-3, z_range=(3e-3, 6e-3))
    pos, amp = synth.scatterer_field(w, np.random.default_rng(3))
    scat = np.concatenate([pos, amp[:, None]], axis=1)
    got = sim_ref.echoes(scat, 8, 1, 6, 512, synth.PITCH, synth.FS, synth.FC, synth.C_SOUND)
    ref = synth.echoes(w, pos, amp)
    assert np.max(np.abs(got - ref)) < 1e-5 * np.max(np.abs(ref))
    # grouped rows: the sum over the group's rows
    g4 = sim_ref.echoes(scat, 2, 4, 6, 512, synth.PITCH, synth.FS, synth.FC, synth.C_SOUND)
    assert np.allclose(g4[0], got[0:4].sum(0)) and np.allclose(g4[1], got[4:8].sum(0))


def test_sim_noise_is_standard_normal():
    from oracle import sim_ref
    z = sim_ref.gaussian_noise(200000, 77)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01
