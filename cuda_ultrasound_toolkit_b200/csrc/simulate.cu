// GPU RF simulator: int16 raw frames of point-scatterer phantoms for a row-column array, in the
// raw layout the beamforming pipeline reads (channel-slowest [raw channel][transmit * S + s]).
//
// Model (the delay model of the upstream HERCULES kernel,
// cuda_toolkit/src/beamformer/kernels/templated_beamformer.cuh:102-216, with a plane-wave
// transmit along z): transmit rows lie along y at y_r = -R p / 2 + p / 2 + r p (R rows),
// receive columns along x at x_c = -C p / 2 + p / 2 + c p. Transmit event t fires rows
// t * stride + offset + k, k < rows_per_transmit. A scatterer at (x, y, z) with
// amplitude a echoes on (row r, column c) at the sample position
//     pos = (z + sqrt((x_c - x)^2 + (y_r - y)^2 + z^2)) / c_sound * fs
// with a 2-cycle Gaussian-windowed tone a exp(-u^2 / (2 sigma^2)) cos(2 pi fc / fs u),
// u = n - pos, on the 33 samples n = floor(pos) - 16 .. floor(pos) + 16. The echo of a
// transmit event is the sum over the rows it fires.
// Transmit events are Hadamard encoded (enc[t] = sum_k H[t][k] echo[k], Sylvester H), white
// Gaussian noise at the requested SNR (relative to the encoded signal's RMS) is added, the
// frame is scaled to 0.8 * 32767 / max |enc| and rounded to int16, and receive channel c is
// stored at raw channel map[c].
//
// Noise: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC 2011) keyed by the frame seed, one counter per encoded sample, Box-Muller on
// the first two output words; a CPU restatement reproduces the same stream.
//
// Kernels: one CTA per (transmit, channel) row accumulates all echoes in shared memory (the
// pulse is advanced by a two-term recurrence, so a sample costs a few FMAs and one shared
// atomic); encoding runs the fast Walsh-Hadamard transform over 32-sample column tiles in
// shared memory and accumulates the signal energy; a noise pass tracks max |enc|; a final
// pass quantises and scatters through the channel map.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "../../include/cuda_toolkit_b200_learn.h"

namespace cutb {
namespace {

constexpr int kHalfWidth = 16;
constexpr float kTwoPi = 6.283185307179586f;

struct SimGeom {
    int T, G, C, S, R, stride, offset;
    float pitch, fs, fc, c_sound;
    float inv_two_sigma2;   // 1 / (2 sigma^2), sigma in samples
    float q;                // exp(-1 / sigma^2)
    float omega;            // 2 pi fc / fs
};

__global__ void echo_kernel(const float4* __restrict__ scat, int n, SimGeom g, float* __restrict__ echo)
{
    extern __shared__ float row[];
    const int c = blockIdx.x, t = blockIdx.y;
    for (int s = threadIdx.x; s < g.S; s += blockDim.x) row[s] = 0.f;
    __syncthreads();
    const int R = g.R;
    const float xc = -g.C * g.pitch * 0.5f + g.pitch * 0.5f + c * g.pitch;
    const float k_pos = g.fs / g.c_sound;
    float crot, srot;
    sincosf(g.omega, &srot, &crot);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 p = scat[i];
        if (p.w == 0.f) continue;
        const float dx = xc - p.x, dx2z2 = dx * dx + p.z * p.z;
        for (int k = 0; k < g.G; ++k) {
            const int r = t * g.stride + g.offset + k;
            const float yr = -R * g.pitch * 0.5f + g.pitch * 0.5f + r * g.pitch;
            const float dy = yr - p.y;
            const float pos = (p.z + sqrtf(dx2z2 + dy * dy)) * k_pos;
            const int base = (int)floorf(pos);
            const float u0 = (float)(base - kHalfWidth) - pos;
            // envelope e(u) = exp(-u^2 / (2 s^2)); e(u + 1) = e(u) * m(u), m(u + 1) = m(u) * q
            float env = p.w * expf(-u0 * u0 * g.inv_two_sigma2);
            float mul = expf(-(2.f * u0 + 1.f) * g.inv_two_sigma2);
            float cs, sn;
            sincosf(g.omega * u0, &sn, &cs);
#pragma unroll 1
            for (int j = 0; j <= 2 * kHalfWidth; ++j) {
                const int s = base - kHalfWidth + j;
                if (s >= 0 && s < g.S) atomicAdd(&row[s], env * cs);
                env *= mul;
                mul *= g.q;
                const float c2 = cs * crot - sn * srot;
                sn = sn * crot + cs * srot;
                cs = c2;
            }
        }
    }
    __syncthreads();
    float* dst = echo + ((size_t)t * g.C + c) * g.S;
    for (int s = threadIdx.x; s < g.S; s += blockDim.x) dst[s] = row[s];
}

// FWHT over transmits for 32-sample column tiles; accumulates sum(enc^2) in double.
__global__ void encode_kernel(float* __restrict__ echo, int T, int C, int S, int hadamard, double* __restrict__ sumsq)
{
    extern __shared__ float tile[];  // [T][32]
    const int s0 = blockIdx.x * 32, c = blockIdx.y;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const bool ok = s0 + lane < S;
    for (int t = w; t < T; t += nw) tile[t * 32 + lane] = ok ? echo[((size_t)t * C + c) * S + s0 + lane] : 0.f;
    __syncthreads();
    if (hadamard) {
        for (int h = 1; h < T; h <<= 1) {
            for (int pair = w; pair < T / 2; pair += nw) {
                const int lo = (pair / h) * 2 * h + pair % h, hi = lo + h;
                const float a = tile[lo * 32 + lane], b = tile[hi * 32 + lane];
                tile[lo * 32 + lane] = a + b;
                tile[hi * 32 + lane] = a - b;
            }
            __syncthreads();
        }
    }
    double acc = 0.0;
    for (int t = w; t < T; t += nw) {
        const float v = tile[t * 32 + lane];
        if (ok) {
            echo[((size_t)t * C + c) * S + s0 + lane] = v;
            acc += (double)v * v;
        }
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) atomicAdd(sumsq, acc);
}

__device__ __forceinline__ void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
    const unsigned long long p = (unsigned long long)a * b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

// Philox4x32 with 10 rounds; returns the first two output words.
__device__ __forceinline__ uint2 philox2(unsigned long long counter, unsigned long long key)
{
    uint32_t c0 = (uint32_t)counter, c1 = (uint32_t)(counter >> 32), c2 = 0, c3 = 0;
    uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53u, c0, hi0, lo0);
        mulhilo(0xCD9E8D57u, c2, hi1, lo1);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0;
        c1 = n1;
        c2 = n2;
        c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return make_uint2(c0, c1);
}

__global__ void noise_kernel(float* __restrict__ enc, size_t count, const double* __restrict__ sumsq, float rel_sigma,
                             unsigned long long seed, unsigned* __restrict__ maxabs_bits)
{
    const float sigma = (float)sqrt(*sumsq / (double)count) * rel_sigma;
    float m = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        float v = enc[i];
        if (rel_sigma > 0.f) {
            const uint2 r = philox2(i, seed);
            const float u1 = ((float)r.x + 0.5f) * 2.3283064365386963e-10f;  // (0, 1)
            const float u2 = (float)r.y * 2.3283064365386963e-10f;
            v += sigma * sqrtf(-2.f * logf(u1)) * cosf(kTwoPi * u2);
            enc[i] = v;
        }
        m = fmaxf(m, fabsf(v));
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxabs_bits, __float_as_uint(m));
}

__global__ void quantize_kernel(const float* __restrict__ enc, int T, int C, int S, const int16_t* __restrict__ map,
                                const unsigned* __restrict__ maxabs_bits, int16_t* __restrict__ raw,
                                float* __restrict__ gain_out)
{
    const float mx = __uint_as_float(*maxabs_bits);
    const float gain = mx > 0.f ? 0.8f * 32767.f / mx : 0.f;
    if (blockIdx.x == 0 && threadIdx.x == 0 && gain_out) *gain_out = gain;
    const size_t count = (size_t)T * C * S;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const int s = (int)(i % S);
        const size_t tc = i / S;
        const int c = (int)(tc % C), t = (int)(tc / C);
        raw[(size_t)map[c] * ((size_t)T * S) + (size_t)t * S + s] = (int16_t)rintf(enc[i] * gain);
    }
}

}  // namespace
}  // namespace cutb

using namespace cutb;

struct cutb_sim {
    cutb_sim_config cfg{};
    float* echo = nullptr;
    double* sumsq = nullptr;
    unsigned* maxabs = nullptr;
    int16_t* map = nullptr;
    ~cutb_sim()
    {
        device_free(echo);
        device_free(sumsq);
        device_free(maxabs);
        device_free(map);
    }
};

extern "C" {

CUTB_API cutb_sim* cutb_sim_create(const cutb_sim_config* cfg)
{
    if (!cfg) {
        set_error(CUTB_ERR_INVALID_ARGUMENT, "Null simulator configuration.");
        return nullptr;
    }
    const cutb_sim_config& c = *cfg;
    if (c.transmits < 1 || c.transmits > 1024 || c.rows_per_transmit < 1 || c.rows_per_transmit > 64 ||
        c.channels < 1 || c.channels > 1024 || c.samples < 32 || c.samples > 16384 ||
        (c.encoding == 1 && !is_pow2(c.transmits)) || c.encoding < 0 || c.encoding > 1 || !(c.pitch > 0.f) ||
        !(c.sampling_frequency > 0.f) || !(c.center_frequency > 0.f) || !(c.speed_of_sound > 0.f)) {
        set_error(CUTB_ERR_INVALID_ARGUMENT,
                  "Simulator configuration out of range (T %u x %u rows, C %u, S %u, encoding %d).", c.transmits,
                  c.rows_per_transmit, c.channels, c.samples, c.encoding);
        return nullptr;
    }
    const uint stride = c.row_stride ? c.row_stride : c.rows_per_transmit;
    const uint rows = c.array_rows ? c.array_rows : c.transmits * stride;
    if ((unsigned long long)(c.transmits - 1) * stride + c.row_offset + c.rows_per_transmit > rows || rows > 65536) {
        set_error(CUTB_ERR_INVALID_ARGUMENT, "Simulator: transmit rows exceed the %u-row array.", rows);
        return nullptr;
    }
    auto* sim = new cutb_sim();
    sim->cfg = c;
    sim->cfg.row_stride = stride;
    sim->cfg.array_rows = rows;
    const size_t n = (size_t)c.transmits * c.channels * c.samples;
    if (device_alloc((void**)&sim->echo, n * 4) != cudaSuccess || device_alloc((void**)&sim->sumsq, 8) != cudaSuccess ||
        device_alloc((void**)&sim->maxabs, 4) != cudaSuccess ||
        device_alloc((void**)&sim->map, 2 * c.channels) != cudaSuccess) {
        set_error(CUTB_ERR_ALLOCATION, "Simulator: device allocation failed.");
        delete sim;
        return nullptr;
    }
    return sim;
}

CUTB_API void cutb_sim_destroy(cutb_sim* sim) { delete sim; }

// Copies the encoded, noisy FP32 frame [T][C][S] of the last run (before quantisation).
CUTB_API bool cutb_sim_copy_signal(const cutb_sim* sim, float* d_dst, void* stream)
{
    CUTB_REQUIRE(sim && d_dst, CUTB_ERR_INVALID_ARGUMENT, "cutb_sim_copy_signal: null argument.");
    const size_t n = (size_t)sim->cfg.transmits * sim->cfg.channels * sim->cfg.samples;
    CUTB_CUDA_OK(cudaMemcpyAsync(d_dst, sim->echo, n * 4, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return true;
}

CUTB_API bool cutb_sim_run(cutb_sim* sim, const float* d_scatterers, unsigned count, const int16_t* channel_map,
                           unsigned long long noise_seed, void* d_raw, float* d_gain, void* stream)
{
    CUTB_REQUIRE(sim && channel_map && d_raw && (count == 0 || d_scatterers), CUTB_ERR_INVALID_ARGUMENT,
                 "cutb_sim_run: null argument.");
    const cutb_sim_config& c = sim->cfg;
    for (unsigned i = 0; i < c.channels; ++i)
        CUTB_REQUIRE(channel_map[i] >= 0 && (unsigned)channel_map[i] < c.channels, CUTB_ERR_INVALID_ARGUMENT,
                     "Channel map entry %u = %d outside 0..%u.", i, channel_map[i], c.channels - 1);
    cudaStream_t st = (cudaStream_t)stream;
    const int T = (int)c.transmits, C = (int)c.channels, S = (int)c.samples;
    const size_t n = (size_t)T * C * S;
    CUTB_CUDA_OK(cudaMemcpyAsync(sim->map, channel_map, 2 * C, cudaMemcpyHostToDevice, st));
    SimGeom g{};
    g.T = T;
    g.G = (int)c.rows_per_transmit;
    g.R = (int)c.array_rows;
    g.stride = (int)c.row_stride;
    g.offset = (int)c.row_offset;
    g.C = C;
    g.S = S;
    g.pitch = c.pitch;
    g.fs = c.sampling_frequency;
    g.fc = c.center_frequency;
    g.c_sound = c.speed_of_sound;
    // envelope FWHM = 2 cycles: sigma = (2 / fc) / (2 sqrt(2 ln 2)) seconds, in samples
    const double sigma = (2.0 / c.center_frequency) / 2.3548 * c.sampling_frequency;
    g.inv_two_sigma2 = (float)(1.0 / (2.0 * sigma * sigma));
    g.q = (float)std::exp(-1.0 / (sigma * sigma));
    g.omega = (float)(2.0 * M_PI * c.center_frequency / c.sampling_frequency);
    const size_t smem = (size_t)S * 4;
    CUTB_CUDA_OK(cudaFuncSetAttribute(echo_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    echo_kernel<<<dim3(C, T), 256, smem, st>>>((const float4*)d_scatterers, (int)count, g, sim->echo);
    CUTB_CUDA_OK(cudaGetLastError());
    CUTB_CUDA_OK(cudaMemsetAsync(sim->sumsq, 0, 8, st));
    CUTB_CUDA_OK(cudaMemsetAsync(sim->maxabs, 0, 4, st));
    const size_t tile_smem = (size_t)T * 32 * 4;
    CUTB_REQUIRE(tile_smem <= 200 * 1024, CUTB_ERR_UNSUPPORTED, "Too many transmits for the encoder.");
    CUTB_CUDA_OK(cudaFuncSetAttribute(encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem));
    encode_kernel<<<dim3(div_up(S, 32), C), 256, tile_smem, st>>>(sim->echo, T, C, S, c.encoding == 1, sim->sumsq);
    CUTB_CUDA_OK(cudaGetLastError());
    const float rel_sigma = c.snr_db >= 1000.f ? 0.f : (float)std::pow(10.0, -c.snr_db / 20.0);
    noise_kernel<<<148 * 8, 256, 0, st>>>(sim->echo, n, sim->sumsq, rel_sigma, noise_seed, sim->maxabs);
    CUTB_CUDA_OK(cudaGetLastError());
    quantize_kernel<<<148 * 8, 256, 0, st>>>(sim->echo, T, C, S, sim->map, sim->maxabs, (int16_t*)d_raw, d_gain);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

}  // extern "C"
