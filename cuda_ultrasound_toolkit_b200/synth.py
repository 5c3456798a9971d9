"""Seeded synthetic RF data for the benchmark and parity configurations.

The upstream toolkit is validated against recorded Verasonics data that is not public;
these generators stand in for it with the shapes, sizes and value ranges of the
workloads (row-column array, Hadamard-encoded transmits, int16 raw samples).

Model (the delay model of the upstream HERCULES kernel,
cuda_toolkit/src/beamformer/kernels/templated_beamformer.cuh:102-216, with a plane-wave
transmit along z): a point scatterer p echoes on (transmit row t, receive column c) at
    tau = (p.z + sqrt((x_c - p.x)^2 + (y_t - p.y)^2 + p.z^2)) / c_sound
with x_c, y_t the element centres. Each echo is a 2-cycle Gaussian-windowed tone at fc.
Transmits are encoded as enc[t] = sum_k H[t, k] * echo_k with the order-T Hadamard matrix,
noise is added at the requested SNR, the result is scaled to 0.8 * 32767 and rounded to
int16, and receive channel c is stored at raw channel map[c] (a seeded permutation), in
the channel-slowest layout raw[channel][t * S + s].
"""
import dataclasses
import math

import numpy as np

from .params import (ApoType, CudaBeamformerParameters, EncodingMatrix, InputDataTypes, RCAOrientation,
                     SampleType, SequenceId)

C_SOUND = 1540.0
FC = 5.0e6
FS = 20.0e6
PITCH = 0.3e-3


@dataclasses.dataclass
class Workload:
    name: str
    T: int
    C: int
    S: int
    X: int
    Y: int
    Z: int
    scatterers: int
    cubic: bool
    cf: float
    filter_taps: int = 0
    encoding: int = EncodingMatrix.HADAMARD
    box_xy: float = 9e-3
    z_range: tuple = (10e-3, 40e-3)
    snr_db: float = 40.0


# The configurations the benchmark and the parity tests use.
CONFIGS = {
    # 64 transmits x 64 channels x 2048 samples -> 64 x 64 x 128, linear, no coherence factor.
    "small": Workload("small", 64, 64, 2048, 64, 64, 128, 30, cubic=False, cf=0.0),
    # 128 x 128 x 4096 -> 128 x 128 x 256, 64-tap chirp match filter, cubic + coherence factor.
    "full": Workload("full", 128, 128, 4096, 128, 128, 256, 200, cubic=True, cf=1.0, filter_taps=64),
    # 256 x 256 x 8192 -> 128 x 128 x 256.
    "precision": Workload("precision", 256, 256, 8192, 128, 128, 256, 30, cubic=False, cf=0.0),
}


def sequence_params(name, T=64, C=128, S=2048, X=256, Z=512):
    """The tilted-plane-wave and UFORCES workloads of the benchmark's sequence section: T transmits x
    C channels x S samples -> X x 1 x Z (x, y, z), cubic + coherence factor, receive Hann window of
    f-number 1, in the x-z plane (y-invariant). "tpw": plane waves at angles linspace(-0.25, 0.25)
    rad; "uforces": transmit t on element 2t, focus at 30 mm (transmit 0 is the flash). The plain
    names span the whole aperture in x (0.15 mm steps: the staged windows of a 32-voxel-wide tile
    overflow); "_fine" spans x in +-4.8 mm (0.038 mm steps), on the staged engine."""
    half = (C * PITCH / 2) if not name.endswith("_fine") else 4.8e-3
    bp = make_params(Workload(name, T, C, S, X, 1, Z, 0, cubic=True, cf=1.0))
    bp.tx_orientation = bp.rx_orientation  # x-z plane
    bp.output_min_coordinate[0], bp.output_max_coordinate[0] = -half, half
    bp.fn_rx = 1.0
    if name.startswith("tpw"):
        bp.das_shader_id = int(SequenceId.RCA_TPW)
        for t, ang in enumerate(np.linspace(-0.25, 0.25, T)):
            bp.foci[3 * t + 2] = float(ang)
    elif name.startswith("uforces"):
        bp.das_shader_id = int(SequenceId.UFORCES)
        bp.foci[2] = 30e-3
        for t in range(T):
            bp.sparse_elements[t] = 2 * t
    else:
        raise ValueError(f"unknown sequence workload {name!r}")
    return bp


def chirp_taps(n, f0=3e6, f1=7e6, fs=FS):
    """Linear chirp f0 -> f1 over n samples with a Hann taper, unit energy."""
    t = np.arange(n) / fs
    dur = n / fs
    phase = 2 * np.pi * (f0 * t + 0.5 * (f1 - f0) / dur * t * t)
    h = np.cos(phase) * np.hanning(n)
    return (h / np.sqrt(np.sum(h * h))).astype(np.float32)


def make_params(w: Workload, data_type=InputDataTypes.TYPE_I16, channel_map=None, raw_padding=0):
    bp = CudaBeamformerParameters()
    bp.xdc_transform[12] = w.C * PITCH / 2
    bp.xdc_transform[13] = w.T * PITCH / 2
    bp.xdc_transform[15] = 1.0
    bp.xdc_element_pitch[0] = PITCH
    bp.xdc_element_pitch[1] = PITCH
    bp.rf_raw_dim[0] = w.T * w.S + raw_padding
    bp.rf_raw_dim[1] = w.C
    bp.dec_data_dim[0] = w.S
    bp.dec_data_dim[1] = w.C
    bp.dec_data_dim[2] = w.T
    bp.decode = int(w.encoding)
    bp.das_shader_id = SequenceId.HERCULES
    bp.time_offset = 0.0
    bp.output_points[0] = w.X
    bp.output_points[1] = w.Y
    bp.output_points[2] = w.Z
    bp.output_points[3] = 1
    bp.output_min_coordinate[0] = -w.box_xy
    bp.output_min_coordinate[1] = -w.box_xy
    bp.output_min_coordinate[2] = w.z_range[0]
    bp.output_max_coordinate[0] = w.box_xy
    bp.output_max_coordinate[1] = w.box_xy
    bp.output_max_coordinate[2] = w.z_range[1]
    bp.sampling_frequency = FS
    bp.center_frequency = FC
    bp.speed_of_sound = C_SOUND
    bp.fn_tx = 0.0
    bp.fn_rx = 0.0
    bp.interpolate = bool(w.cubic)
    bp.coherency_weighting = float(w.cf)
    cmap = np.arange(w.C) if channel_map is None else channel_map
    for c in range(w.C):
        bp.channel_mapping[c] = int(cmap[c])
    bp.foci[0] = 0.0
    bp.foci[1] = 0.0
    bp.foci[2] = math.inf
    bp.tx_orientation = RCAOrientation.ORIENT_ROWS
    bp.rx_orientation = RCAOrientation.ORIENT_COLS
    bp.readi_group_count = 0
    bp.readi_group_id = 0
    if w.filter_taps:
        taps = chirp_taps(w.filter_taps)
        bp.filter_length = len(taps)
        for i, v in enumerate(taps):
            bp.rf_filter[i] = float(v)
    bp.data_type = int(data_type)
    bp.apo_type = ApoType.RX_HANN
    bp.to_power = 1
    bp.sample_type = SampleType.SAMPLE_NORMAL
    return bp


def sylvester(n):
    h = np.ones((1, 1))
    while h.shape[0] < n:
        h = np.block([[h, h], [h, -h]])
    return h


def scatterer_field(w: Workload, rng):
    n = w.scatterers
    pos = np.stack([rng.uniform(-w.box_xy, w.box_xy, n), rng.uniform(-w.box_xy, w.box_xy, n),
                    rng.uniform(w.z_range[0], w.z_range[1], n)], axis=1)
    amp = rng.uniform(0.5, 1.0, n)
    return pos, amp


def echoes(w: Workload, pos, amp, half_width=16):
    """Unencoded echoes echo[t][c][s] (float32) of the scatterers."""
    T, C, S = w.T, w.C, w.S
    xc = -C * PITCH / 2 + PITCH / 2 + np.arange(C) * PITCH
    yt = -T * PITCH / 2 + PITCH / 2 + np.arange(T) * PITCH
    sigma = (2.0 / FC) / 2.3548 * FS          # envelope FWHM = 2 cycles, in samples
    offs = np.arange(-half_width, half_width + 1)
    out = np.zeros(T * C * S, dtype=np.float32)
    row = (np.arange(T)[:, None] * C + np.arange(C)[None, :]) * S
    for (px, py, pz), a in zip(pos, amp):
        d = pz + np.sqrt((xc[None, :] - px) ** 2 + (yt[:, None] - py) ** 2 + pz * pz)
        pos_s = d / C_SOUND * FS                              # [T][C] fractional sample
        base = np.floor(pos_s).astype(np.int64)
        n = base[:, :, None] + offs[None, None, :]
        u = n - pos_s[:, :, None]
        val = a * np.exp(-0.5 * (u / sigma) ** 2) * np.cos(2 * np.pi * FC / FS * u)
        ok = (n >= 0) & (n < S)
        lin = (row[:, :, None] + n)[ok]
        out[lin] += val[ok].astype(np.float32)
    return out.reshape(T, C, S)


def synth_frame(w: Workload, seed: int, channel_map=None):
    """Returns (raw int16 [C][T*S], channel_map, scatterer positions, amplitudes).
    channel_map: raw channel of each receive channel; a seeded permutation when None."""
    rng = np.random.default_rng(seed)
    pos, amp = scatterer_field(w, rng)
    e = echoes(w, pos, amp)
    T, C, S = w.T, w.C, w.S
    if w.encoding == EncodingMatrix.NONE:
        enc = e.reshape(T, C * S).astype(np.float64)
    else:
        enc = sylvester(T) @ e.reshape(T, C * S).astype(np.float64)
    rms = np.sqrt(np.mean(enc * enc))
    enc += rng.normal(0.0, rms * 10 ** (-w.snr_db / 20), enc.shape)
    enc *= 0.8 * 32767 / np.max(np.abs(enc))
    q = np.rint(enc).astype(np.int16).reshape(T, C, S)
    cmap = rng.permutation(C).astype(np.int16)
    if channel_map is not None:
        cmap = np.asarray(channel_map, dtype=np.int16)
    raw = np.empty((C, T, S), dtype=np.int16)
    raw[cmap] = q.transpose(1, 0, 2)
    return raw.reshape(C, T * S), cmap, pos, amp


def frame(name: str, seed: int = None, data_type=InputDataTypes.TYPE_I16, channel_map=None):
    """(raw, params) for a named configuration; seed defaults to a fixed per-config value."""
    w = CONFIGS[name]
    if seed is None:
        seed = 1000 * (list(CONFIGS).index(name) + 1)
    raw, cmap, _, _ = synth_frame(w, seed, channel_map)
    bp = make_params(w, data_type=data_type, channel_map=cmap)
    if data_type == InputDataTypes.TYPE_F32:
        raw = raw.astype(np.float32)
    return raw, bp


def phantom(rng, n_points, n_speckle=0, speckle_sigma=0.05, box_xy=9e-3, z_range=(10e-3, 40e-3)):
    """Scatterers as float32 [n][4] (x, y, z, amplitude): n_points point targets with U(0.5, 1)
    amplitudes plus n_speckle weak scatterers with N(0, speckle_sigma) amplitudes, all uniform
    in the box."""
    n = n_points + n_speckle
    out = np.empty((n, 4), dtype=np.float32)
    out[:, 0] = rng.uniform(-box_xy, box_xy, n)
    out[:, 1] = rng.uniform(-box_xy, box_xy, n)
    out[:, 2] = rng.uniform(z_range[0], z_range[1], n)
    out[:n_points, 3] = rng.uniform(0.5, 1.0, n_points)
    out[n_points:, 3] = rng.normal(0.0, speckle_sigma, n_speckle)
    return out


def speckle_frames(seed, width, height, shifts, noise=2.0, sigma=1.4, pad=24):
    """8-bit B-mode-like frames [F][height][width] (uint8): the envelope of one band-limited complex
    speckle field, frame k translated by shifts[k] = (dx, dy) pixels (Fourier shift, so sub-pixel
    shifts are exact band-limited translations), plus Gaussian noise. Inputs of the image
    correlation and motion-detection entry points."""
    rng = np.random.default_rng(seed)
    H, W = height + 2 * pad, width + 2 * pad
    field = rng.standard_normal((H, W)) + 1j * rng.standard_normal((H, W))
    ky = np.fft.fftfreq(H)[:, None]
    kx = np.fft.fftfreq(W)[None, :]
    spec = np.fft.fft2(field) * np.exp(-2 * (np.pi * sigma) ** 2 * (kx ** 2 + ky ** 2))
    frames = []
    for dx, dy in shifts:
        env = np.abs(np.fft.ifft2(spec * np.exp(-2j * np.pi * (kx * dx + ky * dy))))[pad:pad + height, pad:pad + width]
        frames.append(env)
    frames = np.stack(frames)
    frames = frames / np.percentile(frames, 99.5) * 230.0 + rng.normal(0.0, noise, frames.shape)
    return np.clip(np.rint(frames), 0, 255).astype(np.uint8)


def motion_workload(frames=16, size=512, patch=32, spacing=16, grid=32, margin=16, seed=2024):
    """The motion-detection benchmark case: `frames` speckle frames of size x size, frame k > 0
    translated by a seeded shift of up to 10 px from frame 0; patch / grid / search as given, every
    frame against frame 0. Returns (frames float32 [F][H][W], NccMotionParameters)."""
    from .params import NccMotionParameters
    rng = np.random.default_rng(77)
    shifts = [(0.0, 0.0)] + [tuple(rng.uniform(-10, 10, 2)) for _ in range(frames - 1)]
    f = speckle_frames(seed, size, size, shifts).astype(np.float32)
    p = NccMotionParameters.make(frame_count=frames, image_dims=(size, size), patch_size=patch,
                                 motion_grid_spacing=spacing, motion_grid_dims=(grid, grid),
                                 search_margins=(margin, margin), abs_cor_threshold=0.3, rel_cor_threshold=0.0,
                                 min_patch_variance=0.0, use_subpixel=True, reference_frame=0,
                                 neighbour_compare=False)
    return f, p
