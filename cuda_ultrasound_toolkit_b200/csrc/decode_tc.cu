// Convert + reorder + Hadamard/Walsh decode as an exact int8 tensor-core contraction.
//
// Upstream decodes with one FP32 GEMM, dec[t'][c][s] = fl32(1/T) * sum_t H[t'][t] * x[t][c][s]
// (hadamard_decoder.cpp:49-78). Every raw sample is an int16, x = 256 * hi + lo with hi the
// signed high byte and lo the unsigned low byte, so
//     sum_t H[t'][t] x[t] = 256 * (H . x_hi)[t'] + (H . x_lo)[t']
// and both products are int8 MMAs (tcgen05 kind::i8, int32 accumulation) with H in {-1, +1}.
// |H . x_hi| <= 128 T and |H . x_lo| <= 255 T, so for T <= 256 the combination is exact in int32
// and, scaled by fl32(1/T), bit-identical to the FWHT path and to upstream's FP32 GEMM.
//
// Persistent CTAs (two per SM, 256 TMEM columns each) walk the (receive channel c, N-sample
// tile) items. A = H (M = 128 output rows per tile, K = transmits, K-major, rows beyond T zero)
// comes from a prebuilt canonical image by one bulk copy per CTA. Per item the threads load the
// int16 tile [T][N] of raw channel map[c] with 16-byte loads, split it into a signed-high and an
// unsigned-low byte plane in the MN-major operand layout (16 samples x 8 transmits per core
// matrix), and one thread issues the MMAs: per 32 transmits one for each plane into its own TMEM
// accumulator. Planes and accumulators are double-buffered, so an item's MMAs and the next
// item's loads run during the previous item's epilogue, which combines hi and lo, scales, and
// stores rows t' of [T][C][S] through a per-warp staging tile as whole-row segments.
#include <algorithm>

#include "common.cuh"
#include "stages.h"
#include "tc05.cuh"

namespace cutb {
namespace {

using namespace tc;

constexpr int kThreads = 128;

// Canonical A image: M tile m, row r (t' = 128 m + r), transmit k at
//   m * 128 * T + (r / 8) * (T / 16) * 128 + (k / 16) * 128 + (r % 8) * 16 + (k % 16).
__host__ __device__ constexpr size_t a_offset(int T, int m, int r, int k)
{
    return (size_t)m * 128 * T + (size_t)(r / 8) * (T / 16) * 128 + (size_t)(k / 16) * 128 + (r % 8) * 16 + (k % 16);
}

template <int MT, int N>
struct DecCfg {
    static constexpr uint32_t kSetCols = 2u * MT * N;     // hi and lo accumulators per M tile
    static constexpr uint32_t kTmemCols = 2u * kSetCols;  // two sets: one tile's MMAs, the last one's epilogue
    static_assert(kTmemCols <= 256, "two CTAs per SM");
    static constexpr uint32_t kLboB = (N / 16) * 128;     // stride of 8-transmit groups in a plane
    static constexpr int kMaxVec = 8;                     // 16-byte raw vectors per thread and tile
    static_assert((MT * 128) * N / 8 / kThreads <= kMaxVec, "tile load per thread");
    // Epilogue staging per warp: 32 output rows of SC samples, rows padded by 4 floats (stride
    // 4 mod 8 words: conflict-free writes, whole-row reads); 32 columns when two CTAs still fit
    // beside the 64 KB encoding image of T > 128, else 16.
    static constexpr int SC = MT == 1 ? 32 : 16;
    static_assert(N % SC == 0, "staged columns");
    static constexpr int kStageRow = SC + 4;
    static constexpr int kLanesPerRow = SC / 4;            // float4 per staged row
    static constexpr int kRowsPerStore = 32 / kLanesPerRow;
    static constexpr uint32_t kStageBytes = 4u * 32 * kStageRow * sizeof(float);
};

// Persistent CTAs (two per SM) over (channel, sample-tile) items, item = c * ntiles + tile. Per
// iteration j:
//   1. the prefetched raw vectors of item j become the byte planes of buffer j % 2;
//   2. one thread issues item j's MMAs into TMEM set j % 2 and commits them;
//   3. the raw vectors of item j + 1 are loaded (in flight during step 4);
//   4. item j - 1's accumulators (set (j - 1) % 2) are combined, scaled and stored.
// Buffer and set j % 2 are rewritten in iteration j + 2, after step 4 of iteration j + 1 waited
// for their MMAs and the barrier of step 1 ordered every TMEM read before the next MMAs. All
// waits are bounded; a wait that gives up sets bit 2 of the status word.
template <int MT, int N, int OSTRIDE>
__global__ void __launch_bounds__(kThreads, 2) decode_tc_kernel(const int16_t* __restrict__ raw,
                                                                const int8_t* __restrict__ a_image, DecodeTcArgs a)
{
    using C = DecCfg<MT, N>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t a_full, mma_done[2];
    __shared__ uint32_t tmem_base_s;
    const int T = (int)a.T;
    const uint32_t a_bytes = (uint32_t)MT * 128 * T;
    const uint32_t plane = (uint32_t)T * N;
    uint8_t* A = smem;
    uint8_t* planes = smem + a_bytes;  // buffer b: hi at 2 b plane, lo at (2 b + 1) plane
    float* stage = reinterpret_cast<float*>(planes + 4 * plane);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = (int)((a.S + N - 1) / N);
    const long long items = (long long)a.C * ntiles;
    if (tid == 0) {
        mbar_init(&a_full, 1);
        mbar_init(&mma_done[0], 1);
        mbar_init(&mma_done[1], 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(&tmem_base_s, C::kTmemCols);
        tmem_relinquish();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base_s;
    if (tid == 0) {
        mbar_arrive_expect_tx(&a_full, a_bytes);
        bulk_load(A, a_image, a_bytes, &a_full);
    }

    constexpr int kVecPerRow = N / 8;
    const int nvec = T * kVecPerRow;
    uint4 x[C::kMaxVec];
    auto load = [&](long long item) {
        const int c = (int)(item / ntiles), s0 = (int)(item % ntiles) * N;
        const int16_t* src = raw + (size_t)a.map[c] * a.R0;
#pragma unroll
        for (int k = 0; k < C::kMaxVec; ++k) {
            const int v = tid + k * kThreads;
            x[k] = make_uint4(0, 0, 0, 0);
            if (v < nvec) {
                const int t = v / kVecPerRow, s = s0 + 8 * (v % kVecPerRow);
                if (s < (int)a.S) x[k] = __ldcs(reinterpret_cast<const uint4*>(src + (size_t)t * a.S + s));
            }
        }
    };
    auto split = [&](int b) {
        uint8_t* Bhi = planes + 2 * b * plane;
        uint8_t* Blo = Bhi + plane;
#pragma unroll
        for (int k = 0; k < C::kMaxVec; ++k) {
            const int v = tid + k * kThreads;
            if (v >= nvec) continue;
            const int t = v / kVecPerRow, j = v % kVecPerRow;
            const uint32_t w[4] = {x[k].x, x[k].y, x[k].z, x[k].w};
            uint32_t hi[2], lo[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                // bytes of samples 4h..4h+3: low bytes and high bytes of the four int16 values
                lo[h] = __byte_perm(w[2 * h], w[2 * h + 1], 0x6420);
                hi[h] = __byte_perm(w[2 * h], w[2 * h + 1], 0x7531);
            }
            const uint32_t off = (t / 8) * C::kLboB + ((8 * j) / 16) * 128 + (t % 8) * 16 + (8 * j) % 16;
            *reinterpret_cast<uint2*>(Bhi + off) = make_uint2(hi[0], hi[1]);
            *reinterpret_cast<uint2*>(Blo + off) = make_uint2(lo[0], lo[1]);
        }
    };
    auto epilogue = [&](long long item, int set) {
        const int c = (int)(item / ntiles), s0 = (int)(item % ntiles) * N;
        const uint32_t lane_addr = tmem + set * C::kSetCols + ((uint32_t)(32 * warp) << 16);
        for (int m = 0; m < MT; ++m) {
            if (OSTRIDE == 1) {
                // A lane holds one output row, but a store instruction should cover few rows:
                // SC samples of the warp's 32 rows go through its staging tile and leave as
                // whole-row segments (4 rows x 128 bytes or 8 rows x 64 bytes per store
                // instruction) instead of 32 rows x 16 bytes.
                float* tile = stage + warp * (32 * C::kStageRow);
#pragma unroll 1
                for (int qs = 0; qs < N / C::SC; ++qs) {
                    const int s = s0 + C::SC * qs;
#pragma unroll
                    for (int qq = 0; qq < C::SC / 8; ++qq) {
                        int h[8], l[8];
                        tmem_ld8_i32(lane_addr + (2 * m) * N + C::SC * qs + 8 * qq, h);
                        tmem_ld8_i32(lane_addr + (2 * m + 1) * N + C::SC * qs + 8 * qq, l);
                        tmem_wait_ld();
                        float f[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i) f[i] = __fmul_rn((float)(h[i] * 256 + l[i]), a.alpha);
                        float4* row = reinterpret_cast<float4*>(tile + lane * C::kStageRow + 8 * qq);
                        row[0] = make_float4(f[0], f[1], f[2], f[3]);
                        row[1] = make_float4(f[4], f[5], f[6], f[7]);
                    }
                    __syncwarp();
                    const int col = 4 * (lane % C::kLanesPerRow);
                    if (s + col < (int)a.S) {  // S is a multiple of 8: a float4 is all in or out
#pragma unroll
                        for (int k = 0; k < 32 / C::kRowsPerStore; ++k) {
                            const int rr = C::kRowsPerStore * k + lane / C::kLanesPerRow;
                            const int tr = m * 128 + 32 * warp + rr;
                            if (tr < T)
                                __stcs(reinterpret_cast<float4*>(a.out + ((size_t)tr * a.C + c) * a.S + s + col),
                                       *reinterpret_cast<const float4*>(tile + rr * C::kStageRow + col));
                        }
                    }
                    __syncwarp();
                }
            } else {
                const int tp = m * 128 + 32 * warp + lane;  // output row
#pragma unroll 1
                for (int q = 0; q < N / 8; ++q) {
                    int h[8], l[8];
                    tmem_ld8_i32(lane_addr + (2 * m) * N + 8 * q, h);
                    tmem_ld8_i32(lane_addr + (2 * m + 1) * N + 8 * q, l);
                    tmem_wait_ld();
                    const int s = s0 + 8 * q;
                    if (tp >= T || s >= (int)a.S) continue;
                    float f[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) f[i] = __fmul_rn((float)(h[i] * 256 + l[i]), a.alpha);
                    float* o = a.out + (((size_t)tp * a.C + c) * a.S + s) * OSTRIDE;
#pragma unroll
                    for (int i = 0; i < 8; i += 2)
                        reinterpret_cast<float4*>(o)[i / 2] = make_float4(f[i], 0.f, f[i + 1], 0.f);
                }
            }
        }
    };

    long long item = blockIdx.x;
    bool ok = true;
    if (item < items) load(item);
    if (tid == 0 && !mbar_wait(&a_full, 0)) ok = false;
    ok = __syncthreads_and(ok);
    int j = 0;
    for (; ok && item < items; item += gridDim.x, ++j) {
        const int b = j & 1;
        split(b);
        fence_proxy_async_shared();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (tid == 0) {
            constexpr uint32_t id_hi = idesc_i8(128, N, true, true, false, true);
            constexpr uint32_t id_lo = idesc_i8(128, N, true, false, false, true);
            const uint32_t sa = saddr(A), shi = saddr(planes + 2 * b * plane), slo = shi + plane;
            const uint32_t sbo_a = (uint32_t)(T / 16) * 128;
            const uint32_t d = tmem + b * C::kSetCols;
            for (int m = 0; m < MT; ++m)
                for (int ks = 0; ks < T / 32; ++ks) {
                    const uint64_t ad = smem_desc(sa + m * 128 * T + ks * 256, 128, sbo_a);
                    const uint64_t bh = smem_desc(shi + ks * 4 * C::kLboB, C::kLboB, 128);
                    const uint64_t bl = smem_desc(slo + ks * 4 * C::kLboB, C::kLboB, 128);
                    mma_i8(d + (2 * m) * N, ad, bh, id_hi, ks > 0);
                    mma_i8(d + (2 * m + 1) * N, ad, bl, id_lo, ks > 0);
                }
            mma_commit(&mma_done[b]);
        }
        if (item + gridDim.x < items) load(item + gridDim.x);
        if (j > 0) {
            const int pb = (j - 1) & 1;
            __syncwarp();
            if (!__all_sync(0xffffffffu, mbar_wait(&mma_done[pb], ((j - 1) >> 1) & 1))) ok = false;
            fence_after_sync();
            if (ok) epilogue(item - gridDim.x, pb);
            fence_before_sync();
        }
        ok = __syncthreads_and(ok);
    }
    if (ok && j > 0) {  // the last item's accumulators
        const int pb = (j - 1) & 1;
        if (!__all_sync(0xffffffffu, mbar_wait(&mma_done[pb], ((j - 1) >> 1) & 1))) ok = false;
        fence_after_sync();
        if (ok) epilogue(item - gridDim.x, pb);
        fence_before_sync();
    }
    ok = __syncthreads_and(ok);
    if (!ok) {
        if (tid == 0 && a.status) atomicOr(a.status, 2);
        // let MMAs and copies in flight finish (bounded) before TMEM and shared memory are released
        if (tid == 0) {
            mbar_wait(&a_full, 0);
            mbar_wait(&mma_done[0], 0), mbar_wait(&mma_done[0], 1);
            mbar_wait(&mma_done[1], 0), mbar_wait(&mma_done[1], 1);
        }
    }
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, C::kTmemCols);
}

template <int MT, int N, int OSTRIDE>
bool launch_tc(const int16_t* raw, const int8_t* image, const DecodeTcArgs& a, cudaStream_t st)
{
    auto k = decode_tc_kernel<MT, N, OSTRIDE>;
    const uint32_t used = (uint32_t)MT * 128 * a.T + 4u * a.T * N + DecCfg<MT, N>::kStageBytes;
    // at most two CTAs per SM, so that their TMEM (2 x 256 columns) always fits
    const uint32_t smem = used > 80u * 1024 ? used : 80u * 1024;
    CUTB_CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 148;
    CUTB_CUDA_OK(cudaGetDevice(&dev));
    CUTB_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long long items = (long long)a.C * ((a.S + N - 1) / N);
    const unsigned grid = (unsigned)std::min<long long>(items, 2ll * sms);
    k<<<grid, kThreads, smem, st>>>(raw, image, a);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

}  // namespace

bool decode_tc_supported(uint32_t T, uint32_t S, uint64_t R0)
{
    return T >= 32 && T <= 256 && T % 32 == 0 && S % 8 == 0 && R0 % 8 == 0;
}

bool build_decode_tc_image(const int8_t* H, uint32_t T, std::vector<int8_t>& image)
{
    const int MT = T > 128 ? 2 : 1;
    image.assign((size_t)MT * 128 * T, 0);
    for (int m = 0; m < MT; ++m)
        for (int r = 0; r < 128; ++r) {
            const int tp = m * 128 + r;
            if (tp >= (int)T) continue;
            for (int k = 0; k < (int)T; ++k) image[a_offset((int)T, m, r, k)] = H[(size_t)tp * T + k];
        }
    return true;
}

bool launch_decode_tc(const DecodeTcArgs& a, const int8_t* image, const void* raw, unsigned out_stride,
                      cudaStream_t st)
{
    CUTB_REQUIRE(decode_tc_supported(a.T, a.S, a.R0), CUTB_ERR_UNSUPPORTED,
                 "Tensor-core decode needs 32..256 transmits in steps of 32 and 8-sample aligned rows.");
    CUTB_REQUIRE(((uintptr_t)raw & 15) == 0 && ((uintptr_t)a.out & 15) == 0 && ((uintptr_t)image & 15) == 0,
                 CUTB_ERR_INVALID_ARGUMENT, "Tensor-core decode needs 16-byte aligned buffers.");
    const int16_t* r = (const int16_t*)raw;
    if (a.T > 128)
        return out_stride == 1 ? launch_tc<2, 32, 1>(r, image, a, st) : launch_tc<2, 32, 2>(r, image, a, st);
    return out_stride == 1 ? launch_tc<1, 64, 1>(r, image, a, st) : launch_tc<1, 64, 2>(r, image, a, st);
}

}  // namespace cutb
