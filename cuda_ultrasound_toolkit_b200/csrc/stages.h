// Internal interfaces between the plan (plan.cu) and the stage kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "../../include/cuda_beamformer_parameters.h"

namespace cutb {

// ---- convert + reorder + decode (decode.cu) ------------------------------------------
struct DecodeArgs {
    uint64_t R0;               // raw row length in elements (samples*transmits + padding)
    uint32_t S, C, T;          // samples, receive channels, transmits
    uint32_t L, G;             // transmit lanes per sample group, sample groups per warp (32 / L)
    const int16_t* map;        // device: raw channel of each receive channel (C entries)
    const uint16_t* out_row;   // device: natural decode row -> output row (T entries)
    float alpha;               // fl32(1 / T), or 1 when not decoding
};

struct DecodeSetup {
    DecodeArgs args{};
    int encoding = NONE;       // NONE, HADAMARD or WALSH
    unsigned base = 1, R = 1;  // base matrix order, transmits held in registers
};

bool plan_decode_split(unsigned T, unsigned base, unsigned& R, unsigned& L);

// Tensor-core (int8 hi/lo byte split) decode of int16 input (decode_tc.cu).
struct DecodeTcArgs {
    uint64_t R0;
    uint32_t S, C, T;
    const int16_t* map;
    float alpha;
    float* out;
    int* status;
};
bool decode_tc_supported(uint32_t T, uint32_t S, uint64_t R0);
// Canonical shared-memory image of the encoding matrix H (row-major T x T, +-1) for the kernel.
bool build_decode_tc_image(const int8_t* H, uint32_t T, std::vector<int8_t>& image);
bool launch_decode_tc(const DecodeTcArgs& a, const int8_t* image, const void* raw, unsigned out_stride,
                      cudaStream_t st);
bool launch_decode(const DecodeSetup& d, const void* raw, int data_type, float* out, unsigned out_stride,
                   cudaStream_t st);

// ---- bandpass IQ demodulation + time-domain filter (bandpass.cu) ----------------------------
struct DemodArgs {
    uint64_t rows;             // T * C rows of S complex samples (2 S decoded reals in)
    int S, L;                  // complex samples per row, filter taps
    const float* taps;         // device, L entries (null when L == 0)
    double fd_over_fs;         // demodulation frequency / sampling frequency
};
bool launch_demod_fir(const DemodArgs& a, const float* in, void* out, bool bf16, cudaStream_t st);

// ---- analytic signal (hilbert.cu) --------------------------------------------------------
constexpr unsigned kMaxHilbertLength = 131072;

struct HilbertArgs {
    uint64_t rows;             // T * C rows of n samples
    uint32_t n;                // samples per row
    uint32_t log_n;            // FFT length 2^log_n = hilbert_fft_length(n): n, or >= 2 n - 1 for other lengths
    uint32_t in_stride;        // 1: packed floats, 2: real part of complex input
    const float* twiddle;      // device: 2^log_n complex exp(-2 pi i m / 2^log_n)
    const float* weight;       // device: per bin k < 2^log_n, (Ge.re, Go.re, Ge.im, Go.im): the Hermitian-even
                               // part of the spectral weight and the Hermitian-odd part divided by i
};

// FFT length for rows of n samples: n itself for powers of two from 16, else the power of two
// >= max(16, 2 n - 1) (zero-padded circular convolution); 0 when above kMaxHilbertLength.
unsigned hilbert_fft_length(unsigned n);
bool hilbert_supported_length(unsigned n);
bool build_hilbert_tables(unsigned n, const float* taps, unsigned ntaps, std::vector<float>& twiddle,
                          std::vector<float>& weight);
bool launch_hilbert(const HilbertArgs& a, const float* in, void* out, bool bf16, cudaStream_t st);

// ---- delay and sum (das.cu) ----------------------------------------------------------------
struct DasArgs {
    int S, C, T, G;            // samples, channels, transmits, READI sub-signals (>= 1)
    int X, Y, Z;               // output grid
    int seq;                   // HERCULES or FORCES
    int focus;                 // YZ_PLANE (2) or YZ_FOCUS (4) for HERCULES
    int encoding;              // READI sub-signal ordering: HADAMARD or WALSH
    int cubic;                 // 1: Catmull-Rom, 0: linear
    int apo_type;              // ApoType
    int use_apo;               // 0: every apodization weight is exactly 1
    int apply_cf;              // multiply by the coherence factor
    float spm;                 // samples per metre, fs / c
    float px, py;              // element pitch
    float xmin_x, xmin_y;      // first element centre
    float xmax_x, xmax_y;      // last element centre
    float delay;               // (int)(time_offset * fs)
    float vmin_x, vmin_y, vmin_z;
    float res_x, res_y, res_z;
    float fz;                  // focal depth (0 for plane waves)
    float fn_rx, fn_tx;
    float cf_power;            // coherence exponent in [0, 1]
    float to_power;            // sine apodization exponent
    unsigned long long readi_row;  // bit g set: sub-signal g negated
    const float* angles;       // RCA_TPW: device plane-wave angles (foci[t][2]), T entries
    const short* elems;        // UFORCES: device transmit element indices (sparse_elements), T entries
    float fc_over_fs;          // RCA_TPW: centre / sampling frequency (IQ rotation)
    double fc_fs;              // the same ratio formed in FP64 from the FP32 frequencies
    int tile;                  // 0 chosen from the grid, 1 = 4 x 8 x 32, 2 = 8 x 8 x 16 (HERCULES, TPW in a
                               // y-z plane), 3 = one thread per voxel (TPW, UFORCES)
    int schedule;              // 0: split partial last wave / small 2-D volumes, 1: one CTA per tile, 2: stream-K
    int rows_per_stage;        // staged engine: receive channels per stage, 1 .. 8 (0: 8)
    const int* tiles;          // optional device list of tile ids (z-major); null = every tile
    int ntiles;
    int splits;                // > 1: stages split across CTAs, partial sums added atomically
    int* status;               // device word: bit 0 set when a bounded wait gave up
    float4* sk_partials;       // stream-K scratch: 2 x kTileVoxels partial sums per pair of CTAs (null: off)
    int* sk_counters;          // stream-K: arrivals per pair of CTAs, zeroed before each launch
    int sk_capacity;           // pairs the scratch holds
    int z_tile0, z_tiles;      // z-slab: tiles z_tile0 .. z_tile0 + z_tiles - 1 along z only (z_tiles 0: all)
    int z_out0;                // voxel z of the output buffer's first plane (the slab's start)
    long long wait_limit;      // cycles a bounded wait spins before giving up (0: about 0.2 s)
    int debug_skip;            // test hook: stage debug_skip - 1 is never issued (0: off)
};

// One frame of a persistent batched delay-and-sum: its constants and device buffers.
struct DasFrame {
    DasArgs a;
    const void* iq;
    float2* vol;
};
constexpr int kDasBatchMaxFrames = 96;
// Passed by value as the kernel's parameter table (< 32 KiB of kernel parameters).
struct DasBatchParams {
    DasFrame f[kDasBatchMaxFrames];
};
static_assert(sizeof(DasBatchParams) <= 32000, "batched delay-and-sum parameter table too large");

// Launches the persistent delay-and-sum over `nitems` (frame, tile id) items of frames that share
// sequence, interpolation, coherence, apodization, storage and tile shape with `like`, on `grid`
// CTAs; `counter` must be zero. With grid <= 0 it only prepares the kernel and reports its resident
// CTAs per SM (call that once, outside any stream capture).
bool launch_das_batch(const DasBatchParams* P, const int2* items, int nitems, int* counter, const DasArgs& like,
                      bool iq_bf16, bool short_tile, int grid, int* per_sm, cudaStream_t st);
bool das_uses_short_tile(const DasArgs& a);
// True when the delay-and-sum of `a` runs on the staged (TMA window) engine with bounded waits.
bool das_staged(const DasArgs& a);
// Tiles along x, y, z of the delay-and-sum grid for these arguments.
void das_grid_tiles(const DasArgs& a, int counts[3]);

// Derives the delay-and-sum constants from the parameter block, applying the same
// validation as the upstream dispatcher (beamformer.cu:17-197).
bool derive_das(const CudaBeamformerParameters& bp, DasArgs& a);
bool launch_das(const DasArgs& a, const void* iq, bool iq_bf16, void* volume, cudaStream_t st, int* launches);
// Sets the shared-memory attributes of the kernels `a` will launch on the current device and
// caches their wave sizes, without launching (call outside stream capture, e.g. at plan creation).
bool prepare_das(const DasArgs& a, bool iq_bf16);
// Stream-K scratch for a device with `sms` SMs: pairs and bytes of the partial sums.
constexpr int kStreamPairsPerSm = 4;
constexpr size_t kStreamTileVoxels = 1024;
// Tilted-plane-wave and UFORCES delay-and-sum (das_direct.cu).
bool launch_das_direct(const DasArgs& a, const void* iq, bool iq_bf16, void* volume, cudaStream_t st);
// Tile shape (x, y, z voxels) the delay-and-sum kernel uses for these arguments.
void das_tile_shape(const DasArgs& a, int shape[3]);

// ---- image correlation and block matching (motion.cu) --------------------------------------
struct MotionArgs {
    const float* frames;  // F images of W x H (x fastest)
    float* maps;          // F x gy x gx float4
    int W, H, F, patch, spacing, gx, gy, mx, my, ref, neighbour, subpixel;
    float abs_thr, rel_thr, sharp_thr;
    int tw_max, th_max, sw_max, sh_max, cw_max, ch_max;  // set by launch_block_match
};
bool launch_block_match(const MotionArgs& a, cudaStream_t st);
bool launch_corr_images(const float* tpl, int tw, int th, const float* src, int sw, int sh, float* out,
                        cudaStream_t st);

}  // namespace cutb
