// Implicit-GEMM 3x3x3 convolutions on the 5th-generation tensor cores (see conv3d.h).
//
// Forward (also the input gradient, with the flipped/transposed filter): a CTA owns
// 128 * MT output voxels, a box of TX x TY x TZ voxels. For each of the 27 taps one TMA
// tiled load brings the input box shifted by the tap's offset -- all channel blocks -- into
// shared memory; coordinates outside the volume read zeros, which is the "same" padding.
// The box lands as [channel block][voxel][8 channels], which is the no-swizzle K-major
// operand layout (8 voxels x 16 bytes per core matrix), so the MMA reads it directly:
//   D[voxel][cout] += A[voxel][cin of the tap] * Wtap[cout][cin]^T
// M = 128 voxels per instruction, N = cout, K = 16 input channels per instruction; the
// accumulators (MT x cout FP32 columns) stay in TMEM for all 27 taps. One thread issues TMA
// loads, one thread issues MMAs, a 4-stage mbarrier ring couples them, and all four warps run
// the epilogue (TMEM -> registers -> bias/ReLU/mask/loss -> BF16 C8 stores, 16 bytes per voxel).
//
// Weight gradient: dW[cout][tap][cin] = sum over voxels of dout[v][cout] * in[v + tap][cin].
// Rows of D are (tap, cin) pairs -- 16 channel blocks, i.e. 16 / (cin / 8) taps, per CTA --,
// columns are cout and K runs over voxels. Both operands come from the same C8 boxes, read
// as MN-major operands (the 8 channels of a voxel are contiguous along M/N, voxels along K).
// CTAs split the voxels; each adds its partial sums to the FP32 gradient with atomics.
#include <mutex>

#include <cudaTypedefs.h>

#include "common.cuh"
#include "conv3d.h"
#include "tc05.cuh"

namespace cutb {
namespace {

using namespace tc;

constexpr int kThreads = 128;
constexpr uint32_t kPlane = 128 * 16;  // one channel block of a 128-voxel box, bytes

enum ConvFail : int { kFailNone = 0, kFailProducer = 0x100, kFailMma = 0x200, kFailEpilogue = 0x300 };

__device__ __forceinline__ void record_failure(int* status, int code)
{
    if (status) atomicCAS(status, 0, code);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ void unpack_bf16x8(const uint4& u, float (&f)[8])
{
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        f[2 * i] = __uint_as_float(w[i] << 16);
        f[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
    }
}
__device__ __forceinline__ uint4 pack_bf16x8(const float (&f)[8])
{
    return make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                      pack_bf16x2(f[6], f[7]));
}

// After a timed-out wait, give bulk copies that were already issued time to land before the
// CTA releases its shared memory (they complete within microseconds).
__device__ __forceinline__ void drain_after_abort()
{
    for (int i = 0; i < 64; ++i) __nanosleep(1000);
}

constexpr uint32_t tmem_cols_for(int cols)
{
    return cols <= 32 ? 32 : cols <= 64 ? 64 : cols <= 128 ? 128 : cols <= 256 ? 256 : 512;
}

// Epilogue of one output voxel (one TMEM lane): reads the COUT accumulator columns starting at
// `col_addr` (a warp-collective tcgen05.ld per 8 columns, so every lane calls it) and applies the
// requested epilogue; `valid` guards the memory accesses of voxels outside the volume.
template <int COUT>
__device__ __forceinline__ void conv_epilogue_voxel(const ConvFwdArgs& a, uint32_t col_addr, int n, size_t vox,
                                                    bool valid, size_t plane, float& loss)
{
    if (a.epilogue == kEpiComplexOut || a.epilogue == kEpiLossGrad) {
        float v[8];
        tmem_ld8(col_addr, v);
        tmem_wait_ld();
        if (!valid) return;
        const float f0 = v[0] + (a.bias ? a.bias[0] : 0.f), f1 = v[1] + (a.bias ? a.bias[1] : 0.f);
        const size_t e = (size_t)n * plane + vox;
        const float2 in = a.res[e];
        const float s = a.scale[n];
        if (a.epilogue == kEpiComplexOut) {
            a.out_c[e] = make_float2(in.x + s * f0, in.y + s * f1);
        } else {
            const float2 tg = a.target[e];
            const float inv = 1.f / s;
            const float d0 = in.x * inv + f0 - tg.x * inv, d1 = in.y * inv + f1 - tg.y * inv;
            loss += d0 * d0 + d1 * d1;
            float g[8] = {a.grad_scale * d0, a.grad_scale * d1, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            uint4* o = reinterpret_cast<uint4*>(a.out) + ((size_t)n * a.out_cb_total + a.out_cb_offset) * plane + vox;
            o[0] = pack_bf16x8(g);
            for (int q = 1; q < COUT / 8; ++q) o[(size_t)q * plane] = make_uint4(0, 0, 0, 0);
        }
        return;
    }
#pragma unroll 1
    for (int q = 0; q < COUT / 8; ++q) {
        float v[8];
        tmem_ld8(col_addr + q * 8, v);
        tmem_wait_ld();
        if (!valid) continue;
        if (a.epilogue == kEpiMask) {
            const uint4 m =
                reinterpret_cast<const uint4*>(a.mask)[((size_t)n * a.mask_cb_total + a.mask_cb_offset + q) * plane + vox];
            float mf[8];
            unpack_bf16x8(m, mf);
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = mf[i] > 0.f ? v[i] : 0.f;
        } else {
            if (a.bias) {
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] += __ldg(a.bias + q * 8 + i);
            }
            if (a.epilogue == kEpiBiasRelu) {
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] = fmaxf(v[i], 0.f);
            }
        }
        reinterpret_cast<uint4*>(a.out)[((size_t)n * a.out_cb_total + a.out_cb_offset + q) * plane + vox] =
            pack_bf16x8(v);
    }
}

__device__ __forceinline__ void flush_loss(const ConvFwdArgs& a, float loss, int lane)
{
    if (a.epilogue != kEpiLossGrad) return;
#pragma unroll
    for (int o = 16; o; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) atomicAdd(a.loss, loss);
}

// ---- forward ---------------------------------------------------------------------------------
template <int CB_IN, int COUT, int MT>
struct FwdCfg {
    static constexpr int kRows = 128 * MT;
    static constexpr uint32_t kABytes = 16u * kRows * CB_IN;
    static constexpr uint32_t kBBytes = 16u * CB_IN * COUT;
    static constexpr uint32_t kStageBytes = kABytes + kBBytes;
    static constexpr int kStages = kStageBytes * 4 <= 150u * 1024 ? 4 : (kStageBytes * 3 <= 200u * 1024 ? 3 : 2);
    static constexpr uint32_t kTmemCols = tmem_cols_for(MT * COUT);
    static constexpr uint32_t kSmemUsed = kStages * kStageBytes;
    // Pad the shared-memory request so that the CTAs one SM can hold never ask for more
    // than the 512 TMEM columns together.
    static constexpr uint32_t kMaxCtas = 512 / kTmemCols;
    static constexpr uint32_t kSmemFloor = kMaxCtas >= 16 ? 0u : (228u * 1024) / (kMaxCtas + 1) + 1024;
    static constexpr uint32_t kSmem = kSmemUsed > kSmemFloor ? kSmemUsed : kSmemFloor;
    static_assert(kStages * kStageBytes <= 220u * 1024, "stage ring too large");
    static_assert(COUT % 16 == 0 && COUT >= 16 && COUT <= 256, "MMA N");
    static_assert(CB_IN % 2 == 0, "K step of 16 channels");
};

template <int CB_IN, int COUT, int MT>
__global__ void __launch_bounds__(kThreads) conv_fwd_kernel(const __grid_constant__ CUtensorMap tmap,
                                                            const ConvFwdArgs a, int TX, int TY, int TZ)
{
    using C = FwdCfg<CB_IN, COUT, MT>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t full[C::kStages], empty[C::kStages], accum;
    __shared__ uint32_t tmem_base_s;
    __shared__ int abort_s;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int X = a.shape.X, Y = a.shape.Y, Z = a.shape.Z;
    const int tiles_x = X / TX, tiles_y = Y / TY, tiles_z = div_up(Z, TZ);
    int b = blockIdx.x;
    const int ix = b % tiles_x;
    b /= tiles_x;
    const int iy = b % tiles_y;
    b /= tiles_y;
    const int iz = b % tiles_z;
    const int n = b / tiles_z;
    const int x0 = ix * TX, y0 = iy * TY, z0 = iz * TZ;

    if (tid == 0) {
        for (int s = 0; s < C::kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accum, 1);
        abort_s = 0;
        fence_mbar_init();
        prefetch_tensormap(&tmap);
    }
    if (warp == 0) {
        tmem_alloc(&tmem_base_s, C::kTmemCols);
        tmem_relinquish();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base_s;

    if (warp == 0 && lane == 0) {
        for (int t = 0; t < 27; ++t) {
            const int s = t % C::kStages;
            if (t >= C::kStages && !mbar_wait(&empty[s], ((t / C::kStages) - 1) & 1)) {
                record_failure(a.status, kFailProducer | t);
                abort_s = 1;
                break;
            }
            uint8_t* A = smem + s * C::kStageBytes;
            mbar_arrive_expect_tx(&full[s], C::kStageBytes);
            const int kz = t / 9, ky = (t / 3) % 3, kx = t % 3;
            tma_load_5d(A, &tmap, 0, x0 + kx - 1, y0 + ky - 1, z0 + kz - 1, n * CB_IN, &full[s]);
            bulk_load(A + C::kABytes, a.wf + (size_t)t * CB_IN * COUT * 8, C::kBBytes, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(128, COUT, false, false);
        for (int t = 0; t < 27; ++t) {
            const int s = t % C::kStages;
            if (!mbar_wait(&full[s], (t / C::kStages) & 1)) {
                record_failure(a.status, kFailMma | t);
                abort_s = 1;
                break;
            }
            fence_after_sync();
            const uint32_t a_base = saddr(smem + s * C::kStageBytes);
            const uint32_t b_base = a_base + C::kABytes;
#pragma unroll
            for (int j = 0; j < MT; ++j)
#pragma unroll
                for (int ks = 0; ks < CB_IN / 2; ++ks) {
                    const uint64_t ad = smem_desc(a_base + j * 2048 + ks * 2 * (16 * C::kRows), 16 * C::kRows, 128);
                    const uint64_t bd = smem_desc(b_base + ks * 2 * (16 * COUT), 16 * COUT, 128);
                    mma_bf16(tmem + j * COUT, ad, bd, idesc, (t | ks) != 0);
                }
            mma_commit(&empty[s]);
        }
        mma_commit(&accum);
    }
    __syncwarp();
    __syncthreads();
    const bool ok = __all_sync(0xffffffffu, mbar_wait(&accum, 0));
    fence_after_sync();
    if (!ok) {
        if (lane == 0) record_failure(a.status, kFailEpilogue);
    } else if (!abort_s) {
        const size_t plane = (size_t)X * Y * Z;
        const int row = 32 * warp + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
        float loss = 0.f;
#pragma unroll 1
        for (int j = 0; j < MT; ++j) {
            const int r = j * 128 + row;
            const int x = x0 + r % TX, y = y0 + (r / TX) % TY, z = z0 + r / (TX * TY);
            const size_t vox = ((size_t)z * Y + y) * X + x;
            // a box may extend past a volume smaller than 128 voxels
            conv_epilogue_voxel<COUT>(a, lane_addr + j * COUT, n, vox, z < Z, plane, loss);
        }
        flush_loss(a, loss, lane);
    }
    if (abort_s) drain_after_abort();
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, C::kTmemCols);
}

// ---- forward, 128-voxel lines with a shared halo --------------------------------------------
// For volumes 128 voxels wide. A tile is 2 x 2 (y, z) lines of 128 voxels: four M = 128 MMAs per
// tap. One TMA box brings the tile's halo -- 130 x 4 x 4 voxels (x, y, z) of two input channel
// blocks -- into shared memory, and all 27 taps read that one box at voxel offsets
// ((z + kz) * 4 + y + ky) * 130 + kx (every row stays 16-byte aligned and the 8-row core-matrix
// stride stays 128 bytes), so an input voxel crosses L2 4x per layer instead of 27x. A stage is
// (tile, pair of input channel blocks): the halo plus that pair's weights for all taps. Warp 4
// issues the TMA loads, warp 5 the MMAs, warps 0-3 run the epilogue and hand the accumulators
// back through a TMEM-empty barrier; CTAs are persistent over tiles.
template <int CB_IN, int COUT>
struct LineCfg {
    static constexpr int kTY = 2, kTZ = 2, kMT = kTY * kTZ;
    static constexpr int kHX = 130, kHY = kTY + 2, kHZ = kTZ + 2;
    static constexpr uint32_t kHaloPlane = 16u * kHX * kHY * kHZ;  // one channel block
    static constexpr uint32_t kHaloBytes = 2 * kHaloPlane;
    static constexpr uint32_t kWTap = 2u * COUT * 16;                // one tap, two channel blocks
    static constexpr uint32_t kWBytes = 27 * kWTap;
    static constexpr uint32_t kStageBytes = kHaloBytes + kWBytes;
    static constexpr int kStages = 2;
    static constexpr int kKSteps = CB_IN / 2;
    static constexpr uint32_t kTmemCols = tmem_cols_for(kMT * COUT);
    static constexpr uint32_t kSmem = kStages * kStageBytes;
    static constexpr int kThreads = 192;
    static_assert(kSmem <= 220u * 1024, "stage ring too large");
    static_assert(CB_IN % 2 == 0 && COUT % 16 == 0 && kMT * COUT <= 256, "shape");
};

template <int CB_IN, int COUT>
__global__ void __launch_bounds__(192, 1) conv_fwd_line_kernel(const __grid_constant__ CUtensorMap tmap,
                                                               const ConvFwdArgs a, int ntiles)
{
    using C = LineCfg<CB_IN, COUT>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t full[C::kStages], empty[C::kStages], accum_full, tmem_empty;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Y = a.shape.Y, Z = a.shape.Z;
    const int tiles_y = Y / C::kTY, tiles_z = Z / C::kTZ;

    if (tid == 0) {
        for (int s = 0; s < C::kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accum_full, 1);
        mbar_init(&tmem_empty, 128);
        abort_s = 0;
        fence_mbar_init();
        prefetch_tensormap(&tmap);
    }
    if (warp == 0) {
        tmem_alloc(&tmem_base_s, C::kTmemCols);
        tmem_relinquish();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base_s;

    if (warp == 4) {
        if (lane == 0) {
            int g = 0;
            for (int tile = blockIdx.x; tile < ntiles && !abort_s; tile += gridDim.x) {
                int t = tile;
                const int iy = t % tiles_y;
                t /= tiles_y;
                const int iz = t % tiles_z;
                const int n = t / tiles_z;
                for (int ks = 0; ks < C::kKSteps; ++ks, ++g) {
                    const int slot = g % C::kStages;
                    if (g >= C::kStages && !mbar_wait(&empty[slot], ((g / C::kStages) - 1) & 1)) {
                        record_failure(a.status, kFailProducer | 0x40);
                        abort_s = 1;
                        break;
                    }
                    uint8_t* st = smem + slot * C::kStageBytes;
                    mbar_arrive_expect_tx(&full[slot], C::kStageBytes);
                    tma_load_5d(st, &tmap, 0, -1, iy * C::kTY - 1, iz * C::kTZ - 1, n * CB_IN + 2 * ks, &full[slot]);
                    for (int tap = 0; tap < 27; ++tap)
                        bulk_load(st + C::kHaloBytes + tap * C::kWTap, a.wf + ((size_t)tap * CB_IN + 2 * ks) * COUT * 8,
                                  C::kWTap, &full[slot]);
                }
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(128, COUT, false, false);
            int g = 0, i = 0;
            for (int tile = blockIdx.x; tile < ntiles && !abort_s; tile += gridDim.x, ++i) {
                if (i > 0 && !mbar_wait(&tmem_empty, (i - 1) & 1)) {
                    record_failure(a.status, kFailMma | 0x41);
                    abort_s = 1;
                    break;
                }
                fence_after_sync();
                for (int ks = 0; ks < C::kKSteps; ++ks, ++g) {
                    const int slot = g % C::kStages;
                    if (!mbar_wait(&full[slot], (g / C::kStages) & 1)) {
                        record_failure(a.status, kFailMma | 0x40);
                        abort_s = 1;
                        break;
                    }
                    fence_after_sync();
                    const uint32_t halo = saddr(smem + slot * C::kStageBytes);
                    const uint32_t wts = halo + C::kHaloBytes;
                    for (int tap = 0; tap < 27; ++tap) {
                        const int kz = tap / 9, ky = (tap / 3) % 3, kx = tap % 3;
                        const uint64_t bd = smem_desc(wts + tap * C::kWTap, 16 * COUT, 128);
#pragma unroll
                        for (int j = 0; j < C::kMT; ++j) {
                            const int zl = j / C::kTY, yl = j % C::kTY;
                            const uint32_t start = halo + (((zl + kz) * C::kHY + (yl + ky)) * C::kHX + kx) * 16;
                            const uint64_t ad = smem_desc(start, C::kHaloPlane, 128);
                            mma_bf16(tmem + j * COUT, ad, bd, idesc, (ks | tap) != 0);
                        }
                    }
                    mma_commit(&empty[slot]);
                }
                if (abort_s) break;
                mma_commit(&accum_full);
            }
        }
    } else {
        // epilogue: warps 0-3, TMEM lanes 32 * warp + lane = x of a 128-voxel line
        const size_t plane = (size_t)128 * Y * Z;
        const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
        const int x = 32 * warp + lane;
        float loss = 0.f;
        int i = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&accum_full, i & 1));
            if (!ok || abort_s) {
                if (lane == 0 && !ok) record_failure(a.status, kFailEpilogue | 0x40);
                abort_s = 1;
                break;
            }
            fence_after_sync();
            int t = tile;
            const int iy = t % tiles_y;
            t /= tiles_y;
            const int iz = t % tiles_z;
            const int n = t / tiles_z;
#pragma unroll 1
            for (int j = 0; j < C::kMT; ++j) {
                const int z = iz * C::kTZ + j / C::kTY, y = iy * C::kTY + j % C::kTY;
                conv_epilogue_voxel<COUT>(a, lane_addr + j * COUT, n, ((size_t)z * Y + y) * 128 + x, true, plane, loss);
            }
            fence_before_sync();
            mbar_arrive(&tmem_empty);
        }
        flush_loss(a, loss, lane);
    }
    __syncwarp();
    __syncthreads();
    if (abort_s) drain_after_abort();
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, C::kTmemCols);
}

// ---- weight gradient -------------------------------------------------------------------------
template <int CB_IN, int COUT>
struct WgradCfg {
    static constexpr int kTapsPerBlock = 16 / CB_IN;
    static constexpr uint32_t kABytes = 16 * kPlane;
    static constexpr uint32_t kBBytes = (COUT / 8) * kPlane;
    static constexpr uint32_t kStageBytes = kABytes + kBBytes;
    static constexpr int kStages = kStageBytes * 4 <= 200u * 1024 ? 4 : 3;
    static constexpr uint32_t kTmemCols = tmem_cols_for(COUT);
    static constexpr uint32_t kMaxCtas = 512 / kTmemCols;
    static constexpr uint32_t kSmemUsed = kStages * kStageBytes;
    static constexpr uint32_t kSmemFloor = kMaxCtas >= 16 ? 0u : (228u * 1024) / (kMaxCtas + 1) + 1024;
    static constexpr uint32_t kSmem = kSmemUsed > kSmemFloor ? kSmemUsed : kSmemFloor;
    static_assert(16 % CB_IN == 0, "channel blocks per tap must divide 16");
    static_assert(COUT % 16 == 0 && COUT <= 256, "MMA N");
};

template <int CB_IN, int COUT>
__global__ void __launch_bounds__(kThreads) conv_wgrad_kernel(const __grid_constant__ CUtensorMap tin,
                                                              const __grid_constant__ CUtensorMap tdout,
                                                              const ConvWgradArgs a, int TX, int TY, int TZ,
                                                              int boxes_per_cta)
{
    using C = WgradCfg<CB_IN, COUT>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t full[C::kStages], empty[C::kStages], accum;
    __shared__ uint32_t tmem_base_s;
    __shared__ int abort_s;

    const int X = a.shape.X, Y = a.shape.Y, Z = a.shape.Z;
    const int tiles_x = X / TX, tiles_y = Y / TY, tiles_z = div_up(Z, TZ);
    const int total = a.shape.NB * tiles_x * tiles_y * tiles_z;
    const int box0 = blockIdx.y * boxes_per_cta;
    const int nbox = min(total - box0, boxes_per_cta);
    if (nbox <= 0) return;
    const int tap0 = blockIdx.x * C::kTapsPerBlock;
    const int ntaps = min(C::kTapsPerBlock, 27 - tap0);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < C::kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accum, 1);
        abort_s = 0;
        fence_mbar_init();
        prefetch_tensormap(&tin);
        prefetch_tensormap(&tdout);
    }
    if (warp == 0) {
        tmem_alloc(&tmem_base_s, C::kTmemCols);
        tmem_relinquish();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base_s;

    if (warp == 0 && lane == 0) {
        const uint32_t bytes = ntaps * CB_IN * kPlane + C::kBBytes;
        for (int t = 0; t < nbox; ++t) {
            const int s = t % C::kStages;
            if (t >= C::kStages && !mbar_wait(&empty[s], ((t / C::kStages) - 1) & 1)) {
                record_failure(a.status, kFailProducer | 0x80);
                abort_s = 1;
                break;
            }
            int bx = box0 + t;
            const int ix = bx % tiles_x;
            bx /= tiles_x;
            const int iy = bx % tiles_y;
            bx /= tiles_y;
            const int iz = bx % tiles_z;
            const int n = bx / tiles_z;
            const int x0 = ix * TX, y0 = iy * TY, z0 = iz * TZ;
            uint8_t* A = smem + s * C::kStageBytes;
            mbar_arrive_expect_tx(&full[s], bytes);
            for (int tp = 0; tp < ntaps; ++tp) {
                const int tap = tap0 + tp, kz = tap / 9, ky = (tap / 3) % 3, kx = tap % 3;
                tma_load_5d(A + tp * CB_IN * kPlane, &tin, 0, x0 + kx - 1, y0 + ky - 1, z0 + kz - 1, n * CB_IN,
                            &full[s]);
            }
            tma_load_5d(A + C::kABytes, &tdout, 0, x0, y0, z0, n * (COUT / 8), &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(128, COUT, true, true);
        for (int t = 0; t < nbox; ++t) {
            const int s = t % C::kStages;
            if (!mbar_wait(&full[s], (t / C::kStages) & 1)) {
                record_failure(a.status, kFailMma | 0x80);
                abort_s = 1;
                break;
            }
            fence_after_sync();
            const uint32_t a_base = saddr(smem + s * C::kStageBytes);
            const uint32_t b_base = a_base + C::kABytes;
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                const uint64_t ad = smem_desc(a_base + kk * 256, 128, kPlane);
                const uint64_t bd = smem_desc(b_base + kk * 256, 128, kPlane);
                mma_bf16(tmem, ad, bd, idesc, (t | kk) != 0);
            }
            mma_commit(&empty[s]);
        }
        mma_commit(&accum);
    }
    __syncwarp();
    __syncthreads();
    const bool ok = __all_sync(0xffffffffu, mbar_wait(&accum, 0));
    fence_after_sync();
    if (!ok) {
        if (lane == 0) record_failure(a.status, kFailEpilogue | 0x80);
    } else if (!abort_s) {
        const int row = 32 * warp + lane;
        const int ql = row >> 3, c = row & 7;
        const int tp = ql / CB_IN, cb = ql % CB_IN;
        const int tap = tap0 + tp, ci = cb * 8 + c;
        const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
        const int cin = CB_IN * 8;
#pragma unroll 1
        for (int q = 0; q < COUT / 8; ++q) {
            float v[8];
            tmem_ld8(lane_addr + q * 8, v);
            tmem_wait_ld();
            if (tp < ntaps) {
#pragma unroll
                for (int i = 0; i < 8; ++i) atomicAdd(a.dw + ((size_t)(q * 8 + i) * 27 + tap) * cin + ci, v[i]);
            }
        }
    }
    if (abort_s) drain_after_abort();
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, C::kTmemCols);
}

// ---- host: tensor maps and dispatch ----------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
bool g_force_tap_kernel = false;  // test hook: always use the per-tap forward kernel
std::mutex g_encode_mutex;

bool encode_fn(PFN_cuTensorMapEncodeTiled_v12000* out)
{
    std::lock_guard<std::mutex> lock(g_encode_mutex);
    if (!g_encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        CUTB_CUDA_OK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        CUTB_REQUIRE(fn && q == cudaDriverEntryPointSuccess, CUTB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable.");
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    *out = g_encode;
    return true;
}

// Map of a whole C8 buffer ([n * cb][z][y][x][8] BF16) with boxes of (TX, TY, TZ) voxels and
// `box_cb` channel blocks.
bool c8_tensor_map(CUtensorMap* map, const void* base, VolumeShape s, int cb, int TX, int TY, int TZ, int box_cb)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc;
    if (!encode_fn(&enc)) return false;
    CUTB_REQUIRE(((uintptr_t)base & 15) == 0, CUTB_ERR_INVALID_ARGUMENT, "C8 volume not 16-byte aligned.");
    const cuuint64_t dims[5] = {8, (cuuint64_t)s.X, (cuuint64_t)s.Y, (cuuint64_t)s.Z, (cuuint64_t)s.NB * cb};
    const cuuint64_t strides[4] = {16, 16ull * s.X, 16ull * s.X * s.Y, 16ull * s.X * s.Y * s.Z};
    const cuuint32_t box[5] = {8, (cuuint32_t)TX, (cuuint32_t)TY, (cuuint32_t)TZ, (cuuint32_t)box_cb};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    CUTB_REQUIRE(r == CUDA_SUCCESS, CUTB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d).", (int)r);
    return true;
}

// Box of `rows` voxels: x first, then y, then z. A volume smaller than the box is covered by
// one box whose extra z-planes read zeros and are not written.
bool tile_shape(VolumeShape s, int rows, int* TX, int* TY, int* TZ)
{
    const int tx = s.X < rows ? s.X : rows;
    const int ty = s.Y < rows / tx ? s.Y : rows / tx;
    const int tz = rows / (tx * ty);
    if (tx * ty * tz != rows || s.X % tx || s.Y % ty || tx > 256 || ty > 256 || tz > 256) return false;
    if (tz > s.Z ? (tx != s.X || ty != s.Y) : (s.Z % tz != 0)) return false;
    *TX = tx;
    *TY = ty;
    *TZ = tz;
    return true;
}

bool valid_shape(VolumeShape s)
{
    return s.X > 0 && s.Y > 0 && s.Z > 0 && s.NB > 0 && is_pow2(s.X) && is_pow2(s.Y) && is_pow2(s.Z);
}

template <int CB_IN, int COUT, int MT>
bool launch_fwd(const ConvFwdArgs& a, cudaStream_t st)
{
    using C = FwdCfg<CB_IN, COUT, MT>;
    int TX, TY, TZ;
    CUTB_REQUIRE(tile_shape(a.shape, C::kRows, &TX, &TY, &TZ), CUTB_ERR_UNSUPPORTED,
                 "conv3d: no %d-voxel tile for a %d x %d x %d volume.", C::kRows, a.shape.X, a.shape.Y, a.shape.Z);
    CUtensorMap map;
    if (!c8_tensor_map(&map, a.in, a.shape, CB_IN, TX, TY, TZ, CB_IN)) return false;
    auto k = conv_fwd_kernel<CB_IN, COUT, MT>;
    CUTB_CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::kSmem));
    const long long grid = (long long)a.shape.NB * (a.shape.X / TX) * (a.shape.Y / TY) * div_up(a.shape.Z, TZ);
    k<<<(unsigned)grid, kThreads, C::kSmem, st>>>(map, a, TX, TY, TZ);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

template <int CB_IN, int COUT>
bool launch_fwd_line(const ConvFwdArgs& a, cudaStream_t st)
{
    using C = LineCfg<CB_IN, COUT>;
    CUtensorMap map;
    if (!c8_tensor_map(&map, a.in, a.shape, CB_IN, C::kHX, C::kHY, C::kHZ, 2)) return false;
    auto k = conv_fwd_line_kernel<CB_IN, COUT>;
    CUTB_CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::kSmem));
    const int ntiles = a.shape.NB * (a.shape.Y / C::kTY) * (a.shape.Z / C::kTZ);
    int sms = 148;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const int grid = ntiles < sms ? ntiles : sms;
    k<<<grid, C::kThreads, C::kSmem, st>>>(map, a, ntiles);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

// The halo kernel serves 128-wide volumes whose weights for all taps of two channel blocks fit
// its stage (cout <= 32); everything else uses the per-tap kernel.
template <int CB_IN, int COUT>
constexpr bool line_kernel_fits()
{
    return COUT <= 32 && CB_IN % 2 == 0 && CB_IN <= 8;
}

template <int CB_IN, int COUT>
bool dispatch_fwd_mt(const ConvFwdArgs& a, cudaStream_t st)
{
    if constexpr (line_kernel_fits<CB_IN, COUT>())
        if (a.shape.X == 128 && a.shape.Y % 2 == 0 && a.shape.Z % 2 == 0 && !g_force_tap_kernel)
            return launch_fwd_line<CB_IN, COUT>(a, st);
    const long long vox = (long long)a.shape.X * a.shape.Y * a.shape.Z;
    int TX, TY, TZ;
    if constexpr (4 * COUT <= 256 && 16u * 512 * CB_IN <= 64u * 1024)
        if (vox >= 512 && tile_shape(a.shape, 512, &TX, &TY, &TZ)) return launch_fwd<CB_IN, COUT, 4>(a, st);
    if constexpr (2 * COUT <= 256 && 16u * 256 * CB_IN <= 64u * 1024)
        if (vox >= 256 && tile_shape(a.shape, 256, &TX, &TY, &TZ)) return launch_fwd<CB_IN, COUT, 2>(a, st);
    return launch_fwd<CB_IN, COUT, 1>(a, st);
}

template <int CB_IN, int COUT>
bool launch_wgrad(const ConvWgradArgs& a, cudaStream_t st)
{
    using C = WgradCfg<CB_IN, COUT>;
    int TX, TY, TZ;
    CUTB_REQUIRE(tile_shape(a.shape, 128, &TX, &TY, &TZ), CUTB_ERR_UNSUPPORTED, "conv3d: unsupported volume shape.");
    CUtensorMap tin, tdout;
    if (!c8_tensor_map(&tin, a.in, a.shape, CB_IN, TX, TY, TZ, CB_IN)) return false;
    if (!c8_tensor_map(&tdout, a.dout, a.shape, COUT / 8, TX, TY, TZ, COUT / 8)) return false;
    const int total = a.shape.NB * (a.shape.X / TX) * (a.shape.Y / TY) * div_up(a.shape.Z, TZ);
    const int mblocks = div_up(27 * CB_IN, 16);
    int splits = div_up(4 * 148, mblocks);
    if (splits > total) splits = total;
    const int per = div_up(total, splits);
    splits = div_up(total, per);
    auto k = conv_wgrad_kernel<CB_IN, COUT>;
    CUTB_CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::kSmem));
    k<<<dim3(mblocks, splits), kThreads, C::kSmem, st>>>(tin, tdout, a, TX, TY, TZ, per);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

// ---- elementwise helpers ---------------------------------------------------------------------
__global__ void avgpool2_kernel(const uint4* __restrict__ in, int in_cb_total, int in_cb_offset, int cb,
                                VolumeShape lo, uint4* __restrict__ out)
{
    const size_t nlo = (size_t)lo.X * lo.Y * lo.Z;
    const size_t total = (size_t)lo.NB * cb * nlo;
    const int HX = 2 * lo.X, HY = 2 * lo.Y;
    const size_t nhi = nlo * 8;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t v = i % nlo, nc = i / nlo;  // nc = n * cb + c
        const int x = v % lo.X, y = (v / lo.X) % lo.Y, z = v / ((size_t)lo.X * lo.Y);
        const size_t n = nc / cb, c = nc % cb;
        const uint4* src = in + (n * in_cb_total + in_cb_offset + c) * nhi;
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const size_t hv = ((size_t)(2 * z + (d >> 2)) * HY + 2 * y + ((d >> 1) & 1)) * HX + 2 * x + (d & 1);
            float f[8];
            unpack_bf16x8(src[hv], f);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += f[k];
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] *= 0.125f;
        out[nc * nlo + v] = pack_bf16x8(acc);
    }
}

__global__ void upsample2_kernel(const uint4* __restrict__ in, int cb, VolumeShape lo, uint4* __restrict__ out,
                                 int out_cb_total, int out_cb_offset)
{
    const int HX = 2 * lo.X, HY = 2 * lo.Y, HZ = 2 * lo.Z;
    const size_t nhi = (size_t)HX * HY * HZ, nlo = (size_t)lo.X * lo.Y * lo.Z;
    const size_t total = (size_t)lo.NB * cb * nhi;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t v = i % nhi, nc = i / nhi;
        const int x = v % HX, y = (v / HX) % HY, z = v / ((size_t)HX * HY);
        const size_t lv = ((size_t)(z >> 1) * lo.Y + (y >> 1)) * lo.X + (x >> 1);
        const size_t n = nc / cb, c = nc % cb;
        out[(n * out_cb_total + out_cb_offset + c) * nhi + v] = in[nc * nlo + lv];
    }
}

__global__ void pool_backward_kernel(const uint4* __restrict__ skip, int skip_cb_total, int skip_cb_offset,
                                     const uint4* __restrict__ act, int act_cb_total, int act_cb_offset,
                                     const uint4* __restrict__ dlow, int cb, VolumeShape hi, uint4* __restrict__ out)
{
    const size_t nhi = (size_t)hi.X * hi.Y * hi.Z, nlo = nhi / 8;
    const int LX = hi.X / 2, LY = hi.Y / 2;
    const size_t total = (size_t)hi.NB * cb * nhi;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t v = i % nhi, nc = i / nhi;
        const size_t n = nc / cb, c = nc % cb;
        const int x = v % hi.X, y = (v / hi.X) % hi.Y, z = v / ((size_t)hi.X * hi.Y);
        const size_t lv = ((size_t)(z >> 1) * LY + (y >> 1)) * LX + (x >> 1);
        float s[8], m[8], d[8];
        unpack_bf16x8(skip[(n * skip_cb_total + skip_cb_offset + c) * nhi + v], s);
        unpack_bf16x8(act[(n * act_cb_total + act_cb_offset + c) * nhi + v], m);
        unpack_bf16x8(dlow[nc * nlo + lv], d);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] += m[k] > 0.f ? 0.125f * d[k] : 0.f;
        out[nc * nhi + v] = pack_bf16x8(s);
    }
}

__global__ void upsample_backward_kernel(const uint4* __restrict__ dhigh, int dh_cb_total, int dh_cb_offset, int cb,
                                         VolumeShape hi, uint4* __restrict__ out)
{
    const size_t nhi = (size_t)hi.X * hi.Y * hi.Z, nlo = nhi / 8;
    const int LX = hi.X / 2, LY = hi.Y / 2;
    const size_t total = (size_t)hi.NB * cb * nlo;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t v = i % nlo, nc = i / nlo;
        const size_t n = nc / cb, c = nc % cb;
        const int x = v % LX, y = (v / LX) % LY, z = v / ((size_t)LX * LY);
        const uint4* src = dhigh + (n * dh_cb_total + dh_cb_offset + c) * nhi;
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const size_t hv = ((size_t)(2 * z + (d >> 2)) * hi.Y + 2 * y + ((d >> 1) & 1)) * hi.X + 2 * x + (d & 1);
            float f[8];
            unpack_bf16x8(src[hv], f);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += f[k];
        }
        out[nc * nlo + v] = pack_bf16x8(acc);
    }
}

// db[c * 8 + k] += sum over n, voxels. Grid: (blocks, cb); a block reduces a voxel range of
// every volume for one channel block.
__global__ void bias_grad_kernel(const uint4* __restrict__ g, int cb, VolumeShape s, float* __restrict__ db)
{
    const size_t nv = (size_t)s.X * s.Y * s.Z;
    const int c = blockIdx.y;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int n = 0; n < s.NB; ++n) {
        const uint4* src = g + ((size_t)n * cb + c) * nv;
        for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
            float f[8];
            unpack_bf16x8(src[v], f);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += f[k];
        }
    }
    __shared__ float red[8][32];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float x = acc[k];
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        float x = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += red[threadIdx.x][w];
        atomicAdd(db + c * 8 + threadIdx.x, x);
    }
}

__global__ void sumsq_kernel(const float2* __restrict__ in, size_t nv, float* __restrict__ sumsq)
{
    const int n = blockIdx.y;
    const float2* src = in + (size_t)n * nv;
    float acc = 0.f;
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
        const float2 z = src[v];
        acc += z.x * z.x + z.y * z.y;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sumsq + n, acc);
}

__global__ void pack_input_kernel(const float2* __restrict__ in, size_t nv, int nb, const float* __restrict__ sumsq,
                                  float* __restrict__ scale, uint4* __restrict__ out)
{
    const size_t total = (size_t)nb * nv;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t n = i / nv, v = i % nv;
        const float s = sqrtf(sumsq[n] / (float)nv) + 1e-30f;
        if (v == 0) scale[n] = s;
        const float inv = 1.f / s;
        const float2 z = in[i];
        float f[8] = {z.x * inv, z.y * inv, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        out[(n * 2) * nv + v] = pack_bf16x8(f);
        out[(n * 2 + 1) * nv + v] = make_uint4(0, 0, 0, 0);
    }
}

unsigned grid_for(size_t work, int threads = 256)
{
    size_t b = div_up(work, (size_t)threads);
    const size_t cap = 148 * 16;
    return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

void conv3d_force_tap_kernel(bool on) { g_force_tap_kernel = on; }

bool conv3d_forward(const ConvFwdArgs& a, cudaStream_t st)
{
    CUTB_REQUIRE(valid_shape(a.shape), CUTB_ERR_UNSUPPORTED, "conv3d: volume dimensions must be powers of two.");
    CUTB_REQUIRE(a.in && a.wf && (a.out || a.out_c), CUTB_ERR_INVALID_ARGUMENT, "conv3d: null buffer.");
    CUTB_REQUIRE(((uintptr_t)a.wf & 15) == 0 && (!a.out || ((uintptr_t)a.out & 15) == 0), CUTB_ERR_INVALID_ARGUMENT,
                 "conv3d: buffers must be 16-byte aligned.");
    CUTB_REQUIRE(a.epilogue != kEpiMask || a.mask, CUTB_ERR_INVALID_ARGUMENT, "conv3d: mask epilogue without mask.");
    CUTB_REQUIRE((a.epilogue != kEpiComplexOut && a.epilogue != kEpiLossGrad) || (a.res && a.scale),
                 CUTB_ERR_INVALID_ARGUMENT, "conv3d: complex epilogue without input/scale.");
    CUTB_REQUIRE(a.epilogue != kEpiLossGrad || (a.target && a.loss && a.out), CUTB_ERR_INVALID_ARGUMENT,
                 "conv3d: loss epilogue without target/loss/gradient buffers.");
    const int cbi = a.cin / 8;
#define CUTB_FWD(CBI, CO) \
    if (cbi == CBI && a.cout == CO) return dispatch_fwd_mt<CBI, CO>(a, st);
    CUTB_FWD(2, 16) CUTB_FWD(2, 32) CUTB_FWD(2, 64) CUTB_FWD(4, 16) CUTB_FWD(4, 32) CUTB_FWD(4, 64)
    CUTB_FWD(4, 128) CUTB_FWD(8, 16) CUTB_FWD(8, 32) CUTB_FWD(8, 64) CUTB_FWD(16, 32) CUTB_FWD(16, 64)
#undef CUTB_FWD
    set_error(CUTB_ERR_UNSUPPORTED, "conv3d: channel pair %d -> %d not instantiated.", a.cin, a.cout);
    return false;
}

bool conv3d_wgrad(const ConvWgradArgs& a, cudaStream_t st)
{
    CUTB_REQUIRE(valid_shape(a.shape), CUTB_ERR_UNSUPPORTED, "conv3d: volume dimensions must be powers of two.");
    CUTB_REQUIRE(a.in && a.dout && a.dw, CUTB_ERR_INVALID_ARGUMENT, "conv3d: null buffer.");
    const int cbi = a.cin / 8;
#define CUTB_WG(CBI, CO) \
    if (cbi == CBI && a.cout == CO) return launch_wgrad<CBI, CO>(a, st);
    CUTB_WG(2, 16) CUTB_WG(2, 32) CUTB_WG(2, 64) CUTB_WG(4, 16) CUTB_WG(4, 32) CUTB_WG(4, 64)
    CUTB_WG(4, 128) CUTB_WG(8, 16) CUTB_WG(8, 32) CUTB_WG(8, 64) CUTB_WG(16, 32) CUTB_WG(16, 64)
#undef CUTB_WG
    set_error(CUTB_ERR_UNSUPPORTED, "conv3d: channel pair %d -> %d not instantiated.", a.cin, a.cout);
    return false;
}

bool c8_avgpool2(const __nv_bfloat16* in, int in_cb_total, int in_cb_offset, int cb, VolumeShape s,
                 __nv_bfloat16* out, cudaStream_t st)
{
    VolumeShape lo{s.X / 2, s.Y / 2, s.Z / 2, s.NB};
    avgpool2_kernel<<<grid_for((size_t)lo.NB * cb * lo.X * lo.Y * lo.Z), 256, 0, st>>>(
        (const uint4*)in, in_cb_total, in_cb_offset, cb, lo, (uint4*)out);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

bool c8_upsample2(const __nv_bfloat16* in, int cb, VolumeShape s, __nv_bfloat16* out, int out_cb_total,
                  int out_cb_offset, cudaStream_t st)
{
    upsample2_kernel<<<grid_for((size_t)s.NB * cb * s.X * s.Y * s.Z * 8), 256, 0, st>>>(
        (const uint4*)in, cb, s, (uint4*)out, out_cb_total, out_cb_offset);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

bool c8_pool_backward(const __nv_bfloat16* skip, int skip_cb_total, int skip_cb_offset, const __nv_bfloat16* act,
                      int act_cb_total, int act_cb_offset, const __nv_bfloat16* dlow, int cb, VolumeShape hi,
                      __nv_bfloat16* out, cudaStream_t st)
{
    pool_backward_kernel<<<grid_for((size_t)hi.NB * cb * hi.X * hi.Y * hi.Z), 256, 0, st>>>(
        (const uint4*)skip, skip_cb_total, skip_cb_offset, (const uint4*)act, act_cb_total, act_cb_offset,
        (const uint4*)dlow, cb, hi, (uint4*)out);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

bool c8_upsample_backward(const __nv_bfloat16* dhigh, int dh_cb_total, int dh_cb_offset, int cb, VolumeShape hi,
                          __nv_bfloat16* out, cudaStream_t st)
{
    upsample_backward_kernel<<<grid_for((size_t)hi.NB * cb * hi.X * hi.Y * hi.Z / 8), 256, 0, st>>>(
        (const uint4*)dhigh, dh_cb_total, dh_cb_offset, cb, hi, (uint4*)out);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

bool c8_bias_grad(const __nv_bfloat16* g, int cb, VolumeShape s, float* db, cudaStream_t st)
{
    const size_t nv = (size_t)s.X * s.Y * s.Z;
    unsigned bx = (unsigned)div_up(nv, (size_t)256 * 8);
    if (bx > 148u * 4 / cb + 1) bx = 148u * 4 / cb + 1;
    bias_grad_kernel<<<dim3(bx, cb), 256, 0, st>>>((const uint4*)g, cb, s, db);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

bool c8_pack_input(const float2* in, VolumeShape s, float* scale, float* sumsq, __nv_bfloat16* out, cudaStream_t st)
{
    const size_t nv = (size_t)s.X * s.Y * s.Z;
    CUTB_CUDA_OK(cudaMemsetAsync(sumsq, 0, sizeof(float) * s.NB, st));
    unsigned bx = (unsigned)div_up(nv, (size_t)256 * 16);
    if (bx > 296) bx = 296;
    sumsq_kernel<<<dim3(bx, s.NB), 256, 0, st>>>(in, nv, sumsq);
    CUTB_CUDA_OK(cudaGetLastError());
    pack_input_kernel<<<grid_for((size_t)s.NB * nv), 256, 0, st>>>(in, nv, s.NB, sumsq, scale, (uint4*)out);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

}  // namespace cutb
