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
