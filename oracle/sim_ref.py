"""CPU restatement of the GPU RF simulator (TEST INFRASTRUCTURE ONLY).

Restates cuda_ultrasound_toolkit_b200/csrc/simulate.cu in numpy float64: echoes of point
scatterers under the delay model of the upstream HERCULES kernel
(cuda_toolkit/src/beamformer/kernels/templated_beamformer.cuh:102-216, plane-wave transmit
along z), Sylvester-Hadamard encoding of the transmit events, Philox4x32-10 noise (Salmon et
al., SC 2011) with Box-Muller, scaling to 0.8 * 32767 / max|signal|, rounding to int16 and
the channel-map scatter. Only tests import it.
"""
import numpy as np

M32 = np.uint64(0xFFFFFFFF)
HALF_WIDTH = 16


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32 with 10 rounds on uint64 arrays holding 32-bit words; returns 4 words."""
    c0, c1, c2, c3 = (np.asarray(v, dtype=np.uint64) & M32 for v in (c0, c1, c2, c3))
    k0 = np.uint64(int(k0) & 0xFFFFFFFF)
    k1 = np.uint64(int(k1) & 0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & M32
        hi1, lo1 = p1 >> np.uint64(32), p1 & M32
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        k0 = (k0 + np.uint64(0x9E3779B9)) & M32
        k1 = (k1 + np.uint64(0xBB67AE85)) & M32
    return c0, c1, c2, c3


def gaussian_noise(count, seed):
    """The simulator's unit Gaussian for every sample index 0..count-1."""
    i = np.arange(count, dtype=np.uint64)
    x0, x1, _, _ = philox4x32_10(i & M32, i >> np.uint64(32), 0, 0, seed & 0xFFFFFFFF, seed >> 32)
    u1 = (x0.astype(np.float64) + 0.5) * 2.0 ** -32
    u2 = x1.astype(np.float64) * 2.0 ** -32
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def echoes(scat, T, G, C, S, pitch, fs, fc, c_sound, stride=0, offset=0, rows=0):
    """Unencoded echoes [T][C][S] (float64); event t fires rows t * stride + offset + k, k < G,
    of a `rows`-row array (defaults: stride G, rows T * stride)."""
    stride = stride or G
    R = rows or T * stride
    xc = -C * pitch / 2 + pitch / 2 + np.arange(C) * pitch
    yr = -R * pitch / 2 + pitch / 2 + np.arange(R) * pitch
    sigma = (2.0 / fc) / 2.3548 * fs
    offs = np.arange(-HALF_WIDTH, HALF_WIDTH + 1)
    out = np.zeros((T, C, S))
    fired = np.array([t * stride + offset + k for t in range(T) for k in range(G)])
    tidx = np.repeat(np.arange(T), G)
    yr = yr[fired]
    for x, y, z, a in scat.astype(np.float64):
        if a == 0:
            continue
        pos = (z + np.sqrt((xc[None, :] - x) ** 2 + (yr[:, None] - y) ** 2 + z * z)) / c_sound * fs  # [R][C]
        base = np.floor(pos).astype(np.int64)
        n = base[:, :, None] + offs
        u = n - pos[:, :, None]
        val = a * np.exp(-0.5 * (u / sigma) ** 2) * np.cos(2 * np.pi * fc / fs * u)
        ok = (n >= 0) & (n < S)
        r_i, c_i, _ = np.nonzero(ok)
        np.add.at(out, (tidx[r_i], c_i, n[ok]), val[ok])
    return out


def fwht(x):
    """Sylvester-Hadamard transform along axis 0 (length a power of two)."""
    x = x.copy()
    h = 1
    while h < x.shape[0]:
        for i in range(0, x.shape[0], 2 * h):
            a = x[i:i + h].copy()
            b = x[i + h:i + 2 * h].copy()
            x[i:i + h] = a + b
            x[i + h:i + 2 * h] = a - b
        h *= 2
    return x


def simulate(scat, channel_map, seed, T, G, C, S, pitch, fs, fc, c_sound, snr_db=40.0, encoding=1, stride=0,
             offset=0, rows=0):
    """(raw int16 [C][T*S], noisy encoded float64 signal [T][C][S], gain)."""
    e = echoes(scat, T, G, C, S, pitch, fs, fc, c_sound, stride, offset, rows)
    enc = fwht(e) if encoding == 1 else e
    if snr_db < 1000:
        rms = np.sqrt(np.mean(enc * enc))
        enc = enc + rms * 10 ** (-snr_db / 20) * gaussian_noise(enc.size, seed).reshape(enc.shape)
    mx = np.max(np.abs(enc))
    gain = 0.8 * 32767 / mx if mx > 0 else 0.0
    q = np.rint(enc * gain).astype(np.int16)
    raw = np.empty((C, T, S), dtype=np.int16)
    raw[np.asarray(channel_map, dtype=np.int64)] = q.transpose(1, 0, 2)
    return raw.reshape(C, T * S), enc, gain
