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
#include <cuda_bf16.h>

#include "common.cuh"
#include "stages.h"

namespace cutb {
namespace {

constexpr int kThreads = 256;

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
    extern __shared__ float2 row[];  // S demodulated samples, then L taps (as float2.x)
    float* taps = reinterpret_cast<float*>(row + a.S);
    const size_t r = blockIdx.x;
    const float2* src = reinterpret_cast<const float2*>(in) + r * a.S;
    for (int i = threadIdx.x; i < a.L; i += kThreads) taps[i] = a.taps[i];
    for (int s = threadIdx.x; s < a.S; s += kThreads) {
        const float2 x = __ldcs(src + s);
        const double ph = (double)s * a.fd_over_fs;
        float sn, cs;
        sincospif(2.f * (float)(ph - floor(ph)), &sn, &cs);
        // (x.x - i x.y) * (cs - i sn)
        row[s] = make_float2(x.x * cs - x.y * sn, -x.x * sn - x.y * cs);
    }
    __syncthreads();
    OutT* dst = out + r * a.S;
    if (a.L == 0) {
        for (int s = threadIdx.x; s < a.S; s += kThreads) store(dst, s, row[s]);
        return;
    }
    const int half = a.L / 2;
    for (int s = threadIdx.x; s < a.S; s += kThreads) {
        const int i0 = max(0, half - s), i1 = min(a.L, a.S + half - s);
        float2 acc = make_float2(0.f, 0.f);
        for (int i = i0; i < i1; ++i) {
            const float2 z = row[s + i - half];
            const float h = taps[a.L - 1 - i];
            acc.x = fmaf(z.x, h, acc.x);
            acc.y = fmaf(z.y, h, acc.y);
        }
        const float inv = 1.f / (float)(i1 - i0);
        store(dst, s, make_float2(acc.x * inv, acc.y * inv));
    }
}

}  // namespace

bool launch_demod_fir(const DemodArgs& a, const float* in, void* out, bool bf16, cudaStream_t st)
{
    CUTB_REQUIRE(a.rows > 0 && a.S > 0 && a.L >= 0 && (a.L == 0 || a.taps), CUTB_ERR_INVALID_ARGUMENT,
                 "Demodulation: bad arguments.");
    const size_t smem = (size_t)a.S * sizeof(float2) + (size_t)a.L * sizeof(float);
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
