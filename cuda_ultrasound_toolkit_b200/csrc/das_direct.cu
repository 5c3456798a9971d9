// Delay-and-sum for the tilted-plane-wave (RCA_TPW) and UFORCES sequences.
//
// Restates the upstream kernels beamformer_kernels.cu:490-550 (tpw_beamform) and :93-172
// (uforces_beamform); both are 2-D synthetic apertures in the x-z plane:
//   TPW      receive element c at xdc_mins.x + pitch/2 + c*pitch, path sqrt(rx^2 + z^2); transmit
//            plane wave at angle a_t (foci[t][2]): lat*sin(a_t) + z*cos(a_t), lat = y for a YZ
//            plane, x otherwise; Hann receive window, values below 0.1 skipped; every sample is
//            rotated by exp(i 2 pi fc/fs idx) after the clamp to [1, S-2]; CF always applied.
//   UFORCES  transmit row 0 is a discarded flash: transmit t < T-1 reads row t+1 from the
//            element at xdc_mins.x + pitch/2 + (elem[t] - elem[0])*pitch; path |rx| + |tx|; index
//            clamped to [0, S-2] (the tap below sample 0 reads 0 here, upstream reads outside the
//            row); first used transmit scaled by 1/sqrt(128); Hann receive window; CF applied.
// In both the incoherent sum takes the windowed values, as upstream.
//
// One thread per voxel; a voxel's distances to every element are formed in FP64 once and scaled
// to samples, so the FP32 sample index carries only its own rounding (~1e-5 samples). UFORCES
// keeps the transmit distances of 32 transmits at a time in shared memory and walks the
// channels; TPW walks channels outside and transmits inside with the angles' sines and cosines
// in shared memory. Voxels that do not depend on y (UFORCES, TPW in an XZ plane) are computed
// once per (x, z) and written to every y.
#include <cmath>

#include <cuda_bf16.h>

#include "common.cuh"
#include "stages.h"

namespace cutb {
namespace {

constexpr int kThreads = 128;
constexpr int kTChunk = 32;
constexpr float kPi = 3.141592654f;

__device__ __forceinline__ float2 to_f2(float2 v) { return v; }
__device__ __forceinline__ float2 to_f2(__nv_bfloat162 v) { return __bfloat1622float2(v); }

// Row sample at fractional index idx (already clamped), taps outside [0, n) read as 0.
template <bool CUBIC, class IQ>
__device__ __forceinline__ float2 sample_row(const IQ* __restrict__ row, float idx, int n)
{
    const int i = __float2int_rd(idx);
    const float t = idx - (float)i;
    auto tap = [&](int k) -> float2 {
        return (k >= 0 && k < n) ? to_f2(__ldg(row + k)) : make_float2(0.f, 0.f);
    };
    const float2 p0 = tap(i), p1 = tap(i + 1);
    if constexpr (!CUBIC) return make_float2(fmaf(p1.x - p0.x, t, p0.x), fmaf(p1.y - p0.y, t, p0.y));
    const float2 pm1 = tap(i - 1), p2 = tap(i + 2);
    const float t2 = t * t;
    const float h00 = fmaf(fmaf(2.f, t, -3.f), t2, 1.f);
    const float h10 = fmaf(t - 2.f, t2, t);
    const float h01 = fmaf(-2.f, t, 3.f) * t2;
    const float h11 = (t - 1.f) * t2;
    const float m0x = 0.5f * (p1.x - pm1.x), m0y = 0.5f * (p1.y - pm1.y);
    const float m1x = 0.5f * (p2.x - p0.x), m1y = 0.5f * (p2.y - p0.y);
    return make_float2(h00 * p0.x + h01 * p1.x + h10 * m0x + h11 * m1x, h00 * p0.y + h01 * p1.y + h10 * m0y + h11 * m1y);
}

// f-number Hann window, beamformer_utils.cuh:142-154.
__device__ __forceinline__ float hann(float lateral, float depth, float fnum)
{
    const float a = fminf(fnum * (lateral / depth) / 2.f, 0.5f);
    const float c = __cosf(kPi * a);
    return c * c;
}

template <int SEQ, bool CUBIC, bool CF, class IQ>
__global__ void __launch_bounds__(kThreads) das_direct_kernel(const IQ* __restrict__ iq, float2* __restrict__ vol,
                                                              DasArgs a, int ny)
{
    __shared__ float tx_s[kTChunk][kThreads];
    __shared__ float sin_s[256], cos_s[256];
    const long long gid = (long long)blockIdx.x * kThreads + threadIdx.x;
    const long long total_vox = (long long)a.X * ny * a.Z;
    if (SEQ == RCA_TPW) {
        for (int t = threadIdx.x; t < a.T; t += kThreads) {
            sin_s[t] = sinf(a.angles[t]);
            cos_s[t] = cosf(a.angles[t]);
        }
        __syncthreads();
    }
    const bool live = gid < total_vox;
    const int x = (int)(gid % a.X), y = (int)((gid / a.X) % ny), z = (int)(gid / ((long long)a.X * ny));
    const float vx = fmaf((float)x, a.res_x, a.vmin_x);
    const float vy = fmaf((float)y, a.res_y, a.vmin_y);
    const float vz = fmaf((float)(live ? z : 0), a.res_z, a.vmin_z);
    const double dvz2 = (double)vz * vz;
    const float hpx = a.px * 0.5f;
    // receive element 0 relative to the voxel (upstream: xdc_mins.x - vox.x + pitch/2)
    const double rx0 = (double)(a.xmin_x - vx + hpx);
    float2 total = make_float2(0.f, 0.f);
    float inc = 0.f;

    if (SEQ == UFORCES) {
        const double fx = (double)(a.xmin_x + hpx);
        const int e0 = a.elems[0];
        for (int t0 = 0; t0 + 1 < a.T; t0 += kTChunk) {
            const int nt = min(kTChunk, a.T - 1 - t0);
            __syncthreads();
            for (int j = 0; j < nt; ++j) {
                const double txx = fx + (double)(a.elems[t0 + j] - e0) * (double)a.px - (double)vx;
                tx_s[j][threadIdx.x] = (float)(sqrt(txx * txx + dvz2) * (double)a.spm);
            }
            __syncthreads();
            if (!live) continue;
            for (int c = 0; c < a.C; ++c) {
                const double rxx = rx0 + (double)c * (double)a.px;
                const float rs = (float)(sqrt(rxx * rxx + dvz2) * (double)a.spm);
                const float apo = hann(fabsf((float)rxx), vz, a.fn_rx);
                for (int j = 0; j < nt; ++j) {
                    const int t = t0 + j;
                    float idx = rs + tx_s[j][threadIdx.x] + a.delay;
                    idx = fminf(fmaxf(idx, 0.f), (float)(a.S - 2));
                    const IQ* row = iq + ((size_t)(t + 1) * a.C + c) * a.S;
                    float2 v = sample_row<CUBIC>(row, idx, a.S);
                    const float w = (t == 0 ? 0.088388347648318f : 1.f) * apo;
                    v.x *= w;
                    v.y *= w;
                    total.x += v.x;
                    total.y += v.y;
                    inc = fmaf(v.x, v.x, fmaf(v.y, v.y, inc));
                }
            }
        }
    } else {
        if (!live) return;
        const float lat = a.focus == 2 ? vy : vx;
        const float two_r = 2.f * a.fc_over_fs;
        for (int c = 0; c < a.C; ++c) {
            const double rxx = rx0 + (double)c * (double)a.px;
            const float apo = hann(fabsf((float)rxx), vz, a.fn_rx);
            if (apo < 0.1f) continue;
            const float rs = (float)(sqrt(rxx * rxx + dvz2) * (double)a.spm) + a.delay;
            const IQ* base = iq + (size_t)c * a.S;
            for (int t = 0; t < a.T; ++t) {
                const float tx = fmaf(lat, sin_s[t], vz * cos_s[t]);
                float idx = fmaf(tx, a.spm, rs);
                idx = fminf(fmaxf(idx, 1.f), (float)(a.S - 2));
                float2 v = sample_row<CUBIC>(base + (size_t)t * a.C * a.S, idx, a.S);
                float sn, cs;
                sincospif(two_r * idx, &sn, &cs);  // exp(i 2 pi fc/fs idx)
                const float rx = v.x * cs - v.y * sn, ry = v.x * sn + v.y * cs;
                v = make_float2(rx * apo, ry * apo);
                total.x += v.x;
                total.y += v.y;
                inc = fmaf(v.x, v.x, fmaf(v.y, v.y, inc));
            }
        }
    }
    if (!live) return;
    if (CF) {
        float cf = powf((total.x * total.x + total.y * total.y) / inc, a.cf_power);
        if (isnan(cf)) cf = 0.f;
        total.x *= cf;
        total.y *= cf;
    }
    if (ny == a.Y) {
        vol[((size_t)z * a.Y + y) * a.X + x] = total;
    } else {
        for (int yy = 0; yy < a.Y; ++yy) vol[((size_t)z * a.Y + yy) * a.X + x] = total;
    }
}

template <int SEQ, class IQ>
bool launch_t(const DasArgs& a, const void* iq, void* volume, cudaStream_t st)
{
    const bool y_invariant = SEQ == UFORCES || a.focus != 2;
    const int ny = y_invariant ? 1 : a.Y;
    const long long n = (long long)a.X * ny * a.Z;
    const unsigned blocks = (unsigned)div_up(n, (long long)kThreads);
    // the coherence factor is always applied by these sequences (its exponent may be 0)
    if (a.cubic)
        das_direct_kernel<SEQ, true, true, IQ><<<blocks, kThreads, 0, st>>>((const IQ*)iq, (float2*)volume, a, ny);
    else
        das_direct_kernel<SEQ, false, true, IQ><<<blocks, kThreads, 0, st>>>((const IQ*)iq, (float2*)volume, a, ny);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

}  // namespace

bool launch_das_direct(const DasArgs& a, const void* iq, bool iq_bf16, void* volume, cudaStream_t st)
{
    CUTB_REQUIRE(a.seq == RCA_TPW || a.seq == UFORCES, CUTB_ERR_UNSUPPORTED, "Not a direct delay-and-sum sequence.");
    CUTB_REQUIRE(a.seq != RCA_TPW || a.angles, CUTB_ERR_NOT_INITIALIZED, "TPW angles not uploaded.");
    CUTB_REQUIRE(a.seq != UFORCES || a.elems, CUTB_ERR_NOT_INITIALIZED, "UFORCES elements not uploaded.");
    CUTB_REQUIRE((long long)a.X * a.Y * a.Z < (1ll << 40), CUTB_ERR_UNSUPPORTED, "Output grid too large.");
    if (a.seq == RCA_TPW)
        return iq_bf16 ? launch_t<RCA_TPW, __nv_bfloat162>(a, iq, volume, st) : launch_t<RCA_TPW, float2>(a, iq, volume, st);
    return iq_bf16 ? launch_t<UFORCES, __nv_bfloat162>(a, iq, volume, st) : launch_t<UFORCES, float2>(a, iq, volume, st);
}

}  // namespace cutb
