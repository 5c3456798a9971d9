// Bandpass-sampled input: IQ demodulation and time-domain filter, the analytic-signal stage of a
// plan whose parameter block says SAMPLE_BANDPASS.
//
// Upstream (RfProcessor::convert_demod, rf_processor.cpp:225-246; DataConverter::convert_and_demod,
// data_converter.cu:63-131; kernels data_conversion_kernels.cuh:14-20, 46-102): every two raw
// samples of a transmit are one IQ pair, sample s of row (t, c) is
//     z[s] = (x[2s], -x[2s + 1]) * exp(-i 2 pi s fd / fs)
// and the filter is a correlation with the reversed taps normalised by the number of taps that
// fall inside the row,
//     y[s] = sum_{i < L, 0 <= s + i - L/2 < S} z[s + i - L/2] h[L - 1 - i] / (number of such i).
// Upstream has no caller of that path (cuda_toolkit::beamform rejects bandpass data); here the
// plan runs it after the transmit decode, which is applied exactly to the raw IQ pairs (it is
// linear in the samples, so it commutes with the demodulation), and the delay-and-sum follows.
//
// One CTA per (t, c) row: the demodulated row and the taps sit in shared memory; the phase is
// formed as 2 pi frac(s fd / fs) from an FP64 product, so it stays exact for long rows (upstream
// multiplies the FP32 sample index into the angle, ~1e-4 rad off at the end of a 4096-sample row).
//
// Filter: a thread produces kOut consecutive outputs. For outputs whose taps all fall inside the
// row it slides a register window of 2 kOut samples through the taps, kOut taps at a time, so a
// block of kOut taps costs kOut new samples and two 16-byte tap loads for kOut^2 complex MACs
// (one sample and one tap load per MAC before: the loop was shared-memory bound). Each output
// still sums its taps in ascending order with one fmaf each, so the result is unchanged; outputs
// near the row ends take the per-output loop. Sample s sits at s + s / kOut in shared memory: the
// lanes of a warp then read samples kOut apart without bank conflicts.
#include <cuda_bf16.h>

#include "common.cuh"
#include "stages.h"

namespace cutb {
namespace {

constexpr int kThreads = 256;
constexpr int kOut = 8;  // consecutive outputs per thread in the filter

__host__ __device__ __forceinline__ int pad_index(int s) { return s + s / kOut; }
__host__ __device__ __forceinline__ int padded_len(int S) { return (pad_index(S) + 2) & ~1; }  // 16-byte multiple

// Packed FP32x2: a complex sample times a real tap in one instruction, element-wise the same
// rounding as two fmaf.
typedef unsigned long long f2x;
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c)
{
    f2x d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2x splat2(float h)
{
    f2x r;
    asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(h));
    return r;
}
__device__ __forceinline__ float2 unpack2(f2x v)
{
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}

// Samples b + 0 .. b + kOut - 1 of the padded row. ALIGNED: b is a multiple of kOut, so they sit
// at consecutive slots after pad_index(b) (constant offsets from one address).
template <bool ALIGNED>
__device__ __forceinline__ void load_block(const float2* row, int b, f2x (&w)[kOut])
{
    const f2x* r = reinterpret_cast<const f2x*>(row);
    if constexpr (ALIGNED) {
        const f2x* q = r + pad_index(b);
#pragma unroll
        for (int j = 0; j < kOut; ++j) w[j] = q[j];
    } else {
#pragma unroll
        for (int j = 0; j < kOut; ++j) w[j] = r[pad_index(b + j)];
    }
}

// acc[k] += sum_t win(t + k) h[t] for t = 0 .. kOut - 1, taps ascending per output; win(j) is
// lo[j] for j < kOut and hi[j - kOut] above.
__device__ __forceinline__ void mac_block(f2x (&acc)[kOut], const f2x (&lo)[kOut], const f2x (&hi)[kOut],
                                          const float* trev)
{
    float h[kOut];
    if ((reinterpret_cast<uintptr_t>(trev) & 15) == 0) {
        const float4 h0 = *reinterpret_cast<const float4*>(trev);
        const float4 h1 = *reinterpret_cast<const float4*>(trev + 4);
        h[0] = h0.x, h[1] = h0.y, h[2] = h0.z, h[3] = h0.w;
        h[4] = h1.x, h[5] = h1.y, h[6] = h1.z, h[7] = h1.w;
    } else {
#pragma unroll
        for (int t = 0; t < kOut; ++t) h[t] = trev[t];
    }
#pragma unroll
    for (int t = 0; t < kOut; ++t) {
        const f2x hh = splat2(h[t]);
#pragma unroll
        for (int k = 0; k < kOut; ++k) acc[k] = fma2(t + k < kOut ? lo[t + k] : hi[t + k - kOut], hh, acc[k]);
    }
}

// Interior outputs s0 .. s0 + kOut - 1: all L taps inside the row. The window slides kOut
// samples per block of kOut taps, alternating which half holds the newer samples.
template <bool ALIGNED>
__device__ __forceinline__ void fir_interior(const float2* row, const float* trev, int L, int b, f2x (&acc)[kOut])
{
    f2x lo[kOut], hi[kOut];
    load_block<ALIGNED>(row, b, lo);
    int i = 0;
    // Loads reach sample b + i + 2 kOut - 1 <= b + L + kOut - 1 <= S: inside the padded row
    // (padded_len(S) > pad_index(S)); the sample at S, if loaded, is not used.
    for (; i + 2 * kOut <= L; i += 2 * kOut) {
        load_block<ALIGNED>(row, b + i + kOut, hi);
        mac_block(acc, lo, hi, trev + i);
        load_block<ALIGNED>(row, b + i + 2 * kOut, lo);
        mac_block(acc, hi, lo, trev + i + kOut);
    }
    if (i + kOut <= L) {
        load_block<ALIGNED>(row, b + i + kOut, hi);
        mac_block(acc, lo, hi, trev + i);
        i += kOut;
    }
    const f2x* r = reinterpret_cast<const f2x*>(row);
    for (; i < L; ++i) {  // remaining taps (L not a multiple of kOut)
        const f2x hh = splat2(trev[i]);
#pragma unroll
        for (int k = 0; k < kOut; ++k) acc[k] = fma2(r[pad_index(b + i + k)], hh, acc[k]);
    }
}

template <class OutT>
__device__ __forceinline__ void store(OutT* out, size_t i, float2 v);
template <>
__device__ __forceinline__ void store<float2>(float2* out, size_t i, float2 v) { out[i] = v; }
template <>
__device__ __forceinline__ void store<__nv_bfloat162>(__nv_bfloat162* out, size_t i, float2 v)
{
    out[i] = __floats2bfloat162_rn(v.x, v.y);
}

template <class OutT>
__global__ void __launch_bounds__(kThreads) demod_fir_kernel(const float* __restrict__ in, OutT* __restrict__ out,
                                                             DemodArgs a)
{
    extern __shared__ float2 row[];  // S demodulated samples (padded), then the L taps reversed
    float* trev = reinterpret_cast<float*>(row + padded_len(a.S));
    const size_t r = blockIdx.x;
    const float2* src = reinterpret_cast<const float2*>(in) + r * a.S;
    for (int i = threadIdx.x; i < a.L; i += kThreads) trev[i] = a.taps[a.L - 1 - i];
    // kLoads loads in flight per thread before the phase arithmetic that consumes them.
    constexpr int kLoads = 8;
    for (int s1 = threadIdx.x; s1 < a.S; s1 += kThreads * kLoads) {
        float2 xs[kLoads];
#pragma unroll
        for (int k = 0; k < kLoads; ++k) {
            const int s = s1 + k * kThreads;
            xs[k] = s < a.S ? __ldcs(src + s) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < kLoads; ++k) {
            const int s = s1 + k * kThreads;
            if (s >= a.S) break;
            const float2 x = xs[k];
            const double ph = (double)s * a.fd_over_fs;
            float sn, cs;
            sincospif(2.f * (float)(ph - floor(ph)), &sn, &cs);
            // (x.x - i x.y) * (cs - i sn)
            row[pad_index(s)] = make_float2(x.x * cs - x.y * sn, -x.x * sn - x.y * cs);
        }
    }
    __syncthreads();
    OutT* dst = out + r * a.S;
    if (a.L == 0) {
        for (int s = threadIdx.x; s < a.S; s += kThreads) store(dst, s, row[pad_index(s)]);
        return;
    }
    const int half = a.L / 2, L = a.L;
    for (int s0 = threadIdx.x * kOut; s0 < a.S; s0 += kThreads * kOut) {
        // Interior: every output s0 .. s0 + kOut - 1 exists and has all L taps inside the row
        // (s >= half and s + L - 1 - half <= S - 1).
        if (s0 >= half && s0 + kOut - 1 <= a.S + half - L && s0 + kOut <= a.S) {
            const int b = s0 - half;  // sample under tap 0 of output s0
            f2x acc[kOut];
#pragma unroll
            for (int k = 0; k < kOut; ++k) acc[k] = 0ull;
            if (half % kOut == 0)  // every block starts on a multiple of kOut
                fir_interior<true>(row, trev, L, b, acc);
            else
                fir_interior<false>(row, trev, L, b, acc);
            const float inv = 1.f / (float)L;
#pragma unroll
            for (int k = 0; k < kOut; ++k) {
                const float2 v = unpack2(acc[k]);
                store(dst, s0 + k, make_float2(v.x * inv, v.y * inv));
            }
        } else {
            for (int s = s0; s < min(s0 + kOut, a.S); ++s) {
                const int i0 = max(0, half - s), i1 = min(L, a.S + half - s);
                float2 acc = make_float2(0.f, 0.f);
                for (int i = i0; i < i1; ++i) {
                    const float2 z = row[pad_index(s + i - half)];
                    const float h = trev[i];
                    acc.x = fmaf(z.x, h, acc.x);
                    acc.y = fmaf(z.y, h, acc.y);
                }
                const float inv = 1.f / (float)(i1 - i0);
                store(dst, s, make_float2(acc.x * inv, acc.y * inv));
            }
        }
    }
}

}  // namespace

bool launch_demod_fir(const DemodArgs& a, const float* in, void* out, bool bf16, cudaStream_t st)
{
    CUTB_REQUIRE(a.rows > 0 && a.S > 0 && a.L >= 0 && (a.L == 0 || a.taps), CUTB_ERR_INVALID_ARGUMENT,
                 "Demodulation: bad arguments.");
    const size_t smem = (size_t)padded_len(a.S) * sizeof(float2) + (size_t)a.L * sizeof(float);
    CUTB_REQUIRE(smem <= 200 * 1024, CUTB_ERR_UNSUPPORTED, "Bandpass rows of %d samples do not fit one CTA.", a.S);
    CUTB_REQUIRE(a.rows <= 0x7fffffffull, CUTB_ERR_UNSUPPORTED, "Too many rows.");
    if (bf16) {
        CUTB_CUDA_OK(cudaFuncSetAttribute(demod_fir_kernel<__nv_bfloat162>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        demod_fir_kernel<__nv_bfloat162><<<(unsigned)a.rows, kThreads, smem, st>>>(in, (__nv_bfloat162*)out, a);
    } else {
        CUTB_CUDA_OK(cudaFuncSetAttribute(demod_fir_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        demod_fir_kernel<float2><<<(unsigned)a.rows, kThreads, smem, st>>>(in, (float2*)out, a);
    }
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

}  // namespace cutb
