// 3-D delay-and-sum with interpolation and coherence weighting.
//
// Restates the live upstream kernels (cuda_toolkit/src/beamformer/):
//   hercules_beamform_new  kernels/templated_beamformer.cuh:102-216
//   forces_beamform_new    kernels/templated_beamformer.cuh:219-324
//   helpers                beamformer_utils.cuh:48-154, 207-213
// with the constants of Beamformer::_params_to_constants (beamformer.cu:17-98) and the
// dispatch rules of Beamformer::beamform (beamformer.cu:139-197, 223-413).
//
// Design: a CTA owns a tile of voxels and walks the [T][C] analytic-signal rows. For
// each row it stages only the window of samples that the tile can address (computed by
// interval arithmetic on the delay over the tile's bounding box) into shared memory, so
// the four-tap gathers of every voxel hit shared memory instead of L1/L2. Lanes of a warp
// are consecutive depths, whose delays differ by a few samples, which keeps the gathers
// free of bank conflicts. Delays are computed on the fly in FP32 from per-voxel bases.
//
// Choices where upstream is silent or self-contradictory (documented for users):
//   * interpolate == false -> linear, true -> cubic Catmull-Rom (upstream always cubic);
//   * HERCULES multiplies by the coherence factor when coherency_weighting > 0 (upstream
//     computes it but does not apply it); FORCES always applies it, as upstream;
//   * a single output point along x or z gets step 0 (upstream divides by zero);
//   * FORCES does not depend on y (upstream recomputes every y): one y-slice is computed
//     and written to every y.
#include <cmath>

#include <cuda_bf16.h>

#include "common.cuh"
#include "encoding.h"
#include "stages.h"

namespace cutb {
namespace {

constexpr int kDasThreads = 256;
constexpr int kVpt = 4;          // voxels per thread (along x)
constexpr int kCps = 8;          // channel rows staged per step
constexpr int kWinMax = 256;     // samples per staged window
constexpr int kWinStride = kWinMax + 4;
constexpr float kPi = 3.141592654f;  // value of CUDART_PI_F used upstream

struct Interval {
    float lo, hi;
};

__device__ __forceinline__ Interval sq_range(float a, float b)
{
    const float lo = (a <= 0.f && b >= 0.f) ? 0.f : fminf(a * a, b * b);
    return {lo, fmaxf(a * a, b * b)};
}

__device__ __forceinline__ float fast_sqrt(float x)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// f-number Hann window, beamformer_utils.cuh:142-154.
__device__ __forceinline__ float hann_apo(float lateral, float depth, float fnum)
{
    float a = fminf(fnum * (lateral / depth) / 2.f, 0.5f);
    const float c = __cosf(kPi * a);
    return c * c;
}

// Sine apodization to an integer power, templated_beamformer.cuh:86-99.
__device__ __forceinline__ float sin_apo(float loc, float centre, float power)
{
    float a = fminf(fmaxf(kPi * loc / centre, -kPi), kPi);
    a = sinf(a);
    float r = 1.f;
    for (unsigned i = 0; (float)i < power; ++i) r *= a;
    return r;
}

__device__ __forceinline__ float2 load_iq(const float2* p) { return __ldg(p); }
__device__ __forceinline__ float2 load_iq(const __nv_bfloat162* p) { return __bfloat1622float2(__ldg(p)); }

// Catmull-Rom (tangent 0.5*(p[i+1] - p[i-1])) at fractional position t in [i, i+1],
// beamformer_utils.cuh:99-125; or linear, :127-140.
template <bool CUBIC>
__device__ __forceinline__ float2 interp(float2 pm1, float2 p0, float2 p1, float2 p2, float t)
{
    if constexpr (CUBIC) {
        const float t2 = t * t;
        const float h00 = fmaf(fmaf(2.f, t, -3.f), t2, 1.f);
        const float h10 = fmaf(t - 2.f, t2, t);
        const float h01 = fmaf(-2.f, t, 3.f) * t2;
        const float h11 = (t - 1.f) * t2;
        const float m0x = 0.5f * (p1.x - pm1.x), m0y = 0.5f * (p1.y - pm1.y);
        const float m1x = 0.5f * (p2.x - p0.x), m1y = 0.5f * (p2.y - p0.y);
        return make_float2(fmaf(h00, p0.x, fmaf(h01, p1.x, fmaf(h10, m0x, h11 * m1x))),
                           fmaf(h00, p0.y, fmaf(h01, p1.y, fmaf(h10, m0y, h11 * m1y))));
    } else {
        return make_float2(fmaf(p1.x - p0.x, t, p0.x), fmaf(p1.y - p0.y, t, p0.y));
    }
}

// Sample of one row at (already clamped) position idx. `row` is either a staged window
// (every tap in range) or a global row of n samples whose taps past the end read as 0.
template <bool CUBIC, bool GUARD, class P>
__device__ __forceinline__ float2 sample(const P* row, float idx, int n)
{
    const int i = __float2int_rd(idx);
    const float t = idx - (float)i;
    auto tap = [&](int k) -> float2 {
        if constexpr (GUARD) return k < n ? load_iq(row + k) : make_float2(0.f, 0.f);
        else return row[k];
    };
    if constexpr (CUBIC) return interp<true>(tap(i - 1), tap(i), tap(i + 1), tap(i + 2), t);
    else return interp<false>(float2{}, tap(i), tap(i + 1), float2{}, t);
}

template <int SEQ, bool CUBIC, bool CF, class IQ>
__global__ void __launch_bounds__(kDasThreads)
das_kernel(const IQ* __restrict__ iq, float2* __restrict__ vol, DasArgs a)
{
    __shared__ float2 win[kCps][kWinStride];
    __shared__ int s_lo[kCps], s_len[kCps];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr bool HERC = SEQ == HERCULES;

    // ---- voxels of this thread and the tile box -------------------------------------
    const int x_base = HERC ? blockIdx.x * kVpt : blockIdx.x * (8 * kVpt) + warp * kVpt;
    const int y_idx = HERC ? blockIdx.y * 8 + warp : 0;
    const int z_idx = blockIdx.z * 32 + lane;
    const bool yz_ok = y_idx < a.Y && z_idx < a.Z;
    const float vy = fmaf((float)min(y_idx, a.Y - 1), a.res_y, a.vmin_y);
    const float vz = fmaf((float)min(z_idx, a.Z - 1), a.res_z, a.vmin_z);
    float vx[kVpt];
#pragma unroll
    for (int v = 0; v < kVpt; ++v) vx[v] = fmaf((float)min(x_base + v, a.X - 1), a.res_x, a.vmin_x);

    // Tile bounding box over the voxels that exist (uniform across the CTA).
    const int tx0 = HERC ? blockIdx.x * kVpt : blockIdx.x * 8 * kVpt;
    const int tx1 = min(tx0 + (HERC ? kVpt : 8 * kVpt), a.X) - 1;
    const int ty0 = HERC ? blockIdx.y * 8 : 0, ty1 = HERC ? min(ty0 + 8, a.Y) - 1 : 0;
    const int tz0 = blockIdx.z * 32, tz1 = min(tz0 + 32, a.Z) - 1;
    const float bx0 = fminf(fmaf((float)tx0, a.res_x, a.vmin_x), fmaf((float)tx1, a.res_x, a.vmin_x));
    const float bx1 = fmaxf(fmaf((float)tx0, a.res_x, a.vmin_x), fmaf((float)tx1, a.res_x, a.vmin_x));
    const float by0 = fminf(fmaf((float)ty0, a.res_y, a.vmin_y), fmaf((float)ty1, a.res_y, a.vmin_y));
    const float by1 = fmaxf(fmaf((float)ty0, a.res_y, a.vmin_y), fmaf((float)ty1, a.res_y, a.vmin_y));
    const float bz0 = fminf(fmaf((float)tz0, a.res_z, a.vmin_z), fmaf((float)tz1, a.res_z, a.vmin_z));
    const float bz1 = fmaxf(fmaf((float)tz0, a.res_z, a.vmin_z), fmaf((float)tz1, a.res_z, a.vmin_z));
    const Interval vz2 = sq_range(bz0, bz1);

    // Transmit distance (HERCULES; templated_beamformer.cuh:16-40, :136-147) and its range.
    float txd = vz;
    Interval txr = {bz0, bz1};
    if (HERC && a.focus == 4) {  // YZ_FOCUS
        const float dz = vz - a.fz;
        txd = copysignf(sqrtf(vy * vy + dz * dz), dz) + a.fz;
        const Interval vy2 = sq_range(by0, by1);
        const float dz0 = bz0 - a.fz, dz1 = bz1 - a.fz;
        const Interval dz2 = sq_range(dz0, dz1);
        const float rlo = sqrtf(vy2.lo + dz2.lo), rhi = sqrtf(vy2.hi + dz2.hi);
        txr.lo = (dz0 >= 0.f ? rlo : -rhi) + a.fz;
        txr.hi = (dz1 <= 0.f ? -rlo : rhi) + a.fz;
    }

    float2 total[kVpt];
    float inc[kVpt];
#pragma unroll
    for (int v = 0; v < kVpt; ++v) { total[v] = make_float2(0.f, 0.f); inc[v] = 0.f; }

    const float spm = a.spm;
    const float smax = (float)a.S - 2.f;

    for (int t = 0; t < a.T; ++t) {
        for (int c0 = 0; c0 < a.C; c0 += kCps) {
            const int nq = min(kCps, a.C - c0);
            // ---- window of samples the tile can address in each staged row -------------
            if (threadIdx.x < nq) {
                const int c = c0 + threadIdx.x;
                float imin = INFINITY, imax = -INFINITY;
                if (HERC) {
                    const float xc = fmaf((float)c, a.px, a.xmin_x);
                    const Interval rx2 = sq_range(xc - bx1, xc - bx0);
                    for (int g = 0; g < a.G; ++g) {
                        const float j = a.G > 1 ? (a.encoding == WALSH ? (float)(t * a.G + g) : (float)(g * a.T + t))
                                                : (float)t;
                        const float yj = fmaf(j, a.py, a.xmin_y);
                        const Interval ry2 = sq_range(yj - by1, yj - by0);
                        imin = fminf(imin, (txr.lo + sqrtf(rx2.lo + ry2.lo + vz2.lo) + a.fz) * spm + a.delay);
                        imax = fmaxf(imax, (txr.hi + sqrtf(rx2.hi + ry2.hi + vz2.hi) + a.fz) * spm + a.delay);
                    }
                } else {
                    const float ec = fmaf((float)c, a.px, a.xmin_x);
                    const Interval rx2 = sq_range(ec - bx1, ec - bx0);
                    const float rlo = sqrtf(rx2.lo + vz2.lo), rhi = sqrtf(rx2.hi + vz2.hi);
                    for (int g = 0; g < a.G; ++g) {
                        const float et = fmaf((float)(g * a.T + t), a.px, a.xmin_x);
                        const Interval tx2 = sq_range(bx0 - et, bx1 - et);
                        imin = fminf(imin, (sqrtf(tx2.lo + vz2.lo) + rlo) * spm + a.delay);
                        imax = fmaxf(imax, (sqrtf(tx2.hi + vz2.hi) + rhi) * spm + a.delay);
                    }
                }
                int lo = 0, len = 0;
                if (imin <= imax) {  // false for NaN bounds: use the guarded direct path
                    imin = fminf(fmaxf(imin, 1.f), smax);
                    imax = fminf(fmaxf(imax, 1.f), smax);
                    lo = max(0, (int)floorf(imin) - 3);
                    const int hi = min(a.S, (int)floorf(imax) + 4);  // index S is a zero tap
                    len = hi - lo + 1;
                    if (len > kWinMax) { lo = 0; len = 0; }
                }
                s_lo[threadIdx.x] = lo;
                s_len[threadIdx.x] = len;
            }
            __syncthreads();
            // ---- stage the windows ------------------------------------------------------
            for (int q = 0; q < nq; ++q) {
                const int len = s_len[q], lo = s_lo[q];
                const IQ* row = iq + ((size_t)t * a.C + c0 + q) * a.S;
                for (int i = threadIdx.x; i < len; i += kDasThreads)
                    win[q][i] = lo + i < a.S ? load_iq(row + lo + i) : make_float2(0.f, 0.f);
            }
            __syncthreads();
            // ---- accumulate ---------------------------------------------------------------
            for (int g = 0; g < a.G; ++g) {
                bool negate = false;
                float ry = 0.f, a2 = 0.f, et = 0.f, yj = 0.f;
                if (a.G > 1) {
                    int bit = g;
                    if (HERC && a.encoding == WALSH && (t & 1)) bit = a.G - 1 - g;
                    negate = (a.readi_row >> bit) & 1ull;
                }
                if (HERC) {
                    const float j = a.G > 1 ? (a.encoding == WALSH ? (float)(t * a.G + g) : (float)(g * a.T + t))
                                            : (float)t;
                    yj = fmaf(j, a.py, a.xmin_y);
                    ry = yj - vy;
                    a2 = fmaf(ry, ry, vz * vz);
                } else {
                    et = fmaf((float)(g * a.T + t), a.px, a.xmin_x);
                }
                for (int q = 0; q < nq; ++q) {
                    const int c = c0 + q;
                    const int len = s_len[q];
                    const bool staged = len > 0;
                    const float lo = (float)s_lo[q];
                    const float hiclamp = staged ? (float)(len - 3) : smax;
                    const float xc = fmaf((float)c, a.px, a.xmin_x);
                    const IQ* grow = iq + ((size_t)t * a.C + c) * a.S;
                    float rx_apo = 1.f, uni_apo = 1.f;
                    if (a.use_apo) {
                        if (HERC) {
                            if (a.apo_type == RX_TO_SIN)
                                uni_apo = sin_apo(xc, a.xmax_x, a.to_power) * sin_apo(yj, a.xmax_y, a.to_power);
                        } else {
                            if (a.apo_type == RX_TO_SIN || a.apo_type == BOTH_TO_SIN)
                                rx_apo = sin_apo(xc, a.xmax_x, a.to_power);
                            if (a.apo_type == TX_TO_SIN || a.apo_type == BOTH_TO_SIN)
                                uni_apo = sin_apo(et, a.xmax_x, a.to_power);
                        }
                    }
#pragma unroll
                    for (int v = 0; v < kVpt; ++v) {
                        const float rx = xc - vx[v];
                        float d, apo = 1.f;
                        if (HERC) {
                            d = txd + fast_sqrt(fmaf(rx, rx, a2));
                            if (a.use_apo) {
                                apo = a.apo_type == RX_TO_SIN ? uni_apo
                                                              : hann_apo(sqrtf(fmaf(rx, rx, ry * ry)), vz, a.fn_rx);
                                if (!(apo > 0.1f)) continue;
                            }
                            d += a.fz;
                        } else {
                            const float txx = vx[v] - et;
                            d = fast_sqrt(fmaf(txx, txx, vz * vz)) + fast_sqrt(fmaf(rx, rx, vz * vz));
                            if (a.use_apo) {
                                float ra = rx_apo;
                                if (!(a.apo_type == RX_TO_SIN || a.apo_type == BOTH_TO_SIN))
                                    ra = hann_apo(fabsf(rx), vz, a.fn_rx);
                                if (!(ra > 0.f)) continue;
                                const float ta = (a.apo_type == TX_TO_SIN || a.apo_type == BOTH_TO_SIN)
                                                     ? uni_apo
                                                     : hann_apo(fabsf(txx), vz, a.fn_tx);
                                apo = ra * ta;
                            }
                        }
                        float idx = fmaf(d, spm, a.delay) - lo;
                        idx = fminf(fmaxf(idx, 1.f), hiclamp);
                        const float2 val = staged ? sample<CUBIC, false>(win[q], idx, 0)
                                                  : sample<CUBIC, true>(grow, idx, a.S);
                        const float w = negate ? -apo : apo;
                        total[v].x = fmaf(w, val.x, total[v].x);
                        total[v].y = fmaf(w, val.y, total[v].y);
                        inc[v] = fmaf(val.x, val.x, fmaf(val.y, val.y, inc[v]));
                    }
                }
            }
            __syncthreads();
        }
    }

    if (!yz_ok) return;
#pragma unroll
    for (int v = 0; v < kVpt; ++v) {
        const int x = x_base + v;
        if (x >= a.X) continue;
        float2 out = total[v];
        if (CF) {
            float cf = powf((out.x * out.x + out.y * out.y) / inc[v], a.cf_power);
            if (isnan(cf)) cf = 0.f;
            out.x *= cf;
            out.y *= cf;
        }
        if (HERC) {
            vol[((size_t)z_idx * a.Y + y_idx) * a.X + x] = out;
        } else {
            for (int y = 0; y < a.Y; ++y) vol[((size_t)z_idx * a.Y + y) * a.X + x] = out;
        }
    }
}

template <int SEQ, bool CUBIC, bool CF, class IQ>
bool launch_das_t(const DasArgs& a, const void* iq, void* volume, cudaStream_t st)
{
    dim3 grid;
    if (SEQ == HERCULES) grid = dim3(div_up(a.X, kVpt), div_up(a.Y, 8), div_up(a.Z, 32));
    else grid = dim3(div_up(a.X, 8 * kVpt), 1, div_up(a.Z, 32));
    CUTB_REQUIRE(grid.y <= 65535 && grid.z <= 65535, CUTB_ERR_UNSUPPORTED, "Output grid too large.");
    das_kernel<SEQ, CUBIC, CF, IQ><<<grid, kDasThreads, 0, st>>>((const IQ*)iq, (float2*)volume, a);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

template <int SEQ, class IQ>
bool launch_das_s(const DasArgs& a, const void* iq, void* volume, cudaStream_t st)
{
    if (a.cubic) return a.apply_cf ? launch_das_t<SEQ, true, true, IQ>(a, iq, volume, st)
                                   : launch_das_t<SEQ, true, false, IQ>(a, iq, volume, st);
    return a.apply_cf ? launch_das_t<SEQ, false, true, IQ>(a, iq, volume, st)
                      : launch_das_t<SEQ, false, false, IQ>(a, iq, volume, st);
}

}  // namespace

bool derive_das(const CudaBeamformerParameters& bp, DasArgs& a)
{
    a = DasArgs{};
    a.S = (int)bp.dec_data_dim[0];
    a.C = (int)bp.dec_data_dim[1];
    a.T = (int)bp.dec_data_dim[2];
    a.X = (int)bp.output_points[0];
    a.Y = (int)bp.output_points[1];
    a.Z = (int)bp.output_points[2];
    CUTB_REQUIRE(bp.dec_data_dim[0] >= 4 && bp.dec_data_dim[1] > 0 && bp.dec_data_dim[2] > 0 &&
                     bp.dec_data_dim[0] < (1u << 30) && bp.dec_data_dim[1] <= 65535 && bp.dec_data_dim[2] <= 65535,
                 CUTB_ERR_INVALID_ARGUMENT, "Invalid decoded dimensions [%u, %u, %u].", bp.dec_data_dim[0],
                 bp.dec_data_dim[1], bp.dec_data_dim[2]);
    CUTB_REQUIRE(bp.output_points[0] > 0 && bp.output_points[1] > 0 && bp.output_points[2] > 0 &&
                     bp.output_points[0] < (1u << 24) && bp.output_points[1] < (1u << 19) &&
                     bp.output_points[2] < (1u << 21),
                 CUTB_ERR_INVALID_ARGUMENT, "Invalid output points [%u, %u, %u].", bp.output_points[0],
                 bp.output_points[1], bp.output_points[2]);
    a.seq = bp.das_shader_id;
    CUTB_REQUIRE(a.seq == HERCULES || a.seq == FORCES, CUTB_ERR_UNSUPPORTED,
                 "Beamformer: Unsupported sequence ID %d.", (int)bp.das_shader_id);

    // beamformer.cu:25-36
    a.spm = bp.sampling_frequency / bp.speed_of_sound;
    CUTB_REQUIRE(std::isfinite(a.spm) && a.spm > 0.f, CUTB_ERR_INVALID_ARGUMENT,
                 "Sampling frequency / speed of sound must be positive and finite.");
    a.px = bp.xdc_element_pitch[0];
    a.py = bp.xdc_element_pitch[1];
    const float hpx = a.px * 0.5f, hpy = a.py * 0.5f;
    a.xmin_x = -bp.xdc_transform[12] + hpx;
    a.xmin_y = -bp.xdc_transform[13] + hpy;
    a.xmax_x = bp.xdc_transform[12] - hpx;
    a.xmax_y = bp.xdc_transform[13] - hpy;
    a.delay = (float)(int)(bp.time_offset * bp.sampling_frequency);
    // beamformer.cu:39-49: lateral step reused for y.
    a.vmin_x = bp.output_min_coordinate[0];
    a.vmin_y = bp.output_min_coordinate[1];
    a.vmin_z = bp.output_min_coordinate[2];
    a.res_x = a.X > 1 ? (bp.output_max_coordinate[0] - bp.output_min_coordinate[0]) / (float)(a.X - 1) : 0.f;
    a.res_y = a.res_x;
    a.res_z = a.Z > 1 ? (bp.output_max_coordinate[2] - bp.output_min_coordinate[2]) / (float)(a.Z - 1) : 0.f;
    a.fn_rx = bp.fn_rx;
    a.fn_tx = bp.fn_tx;
    a.cf_power = fminf(fmaxf(bp.coherency_weighting, 0.f), 1.f);
    a.to_power = (float)bp.to_power;
    a.apo_type = bp.apo_type;
    CUTB_REQUIRE(a.apo_type >= RX_HANN && a.apo_type <= BOTH_TO_SIN, CUTB_ERR_INVALID_ARGUMENT,
                 "Invalid apodization type %d.", a.apo_type);
    a.cubic = bp.interpolate ? 1 : 0;
    a.encoding = bp.decode;

    // Focus type, beamformer.cu:64-83.
    a.fz = bp.foci[2];
    if (bp.tx_orientation == ORIENT_NONE) a.focus = 0;
    else if (std::isinf(bp.foci[2]) || bp.das_shader_id == RCA_TPW) {
        a.fz = 0.f;
        a.focus = bp.tx_orientation == bp.rx_orientation ? 1 : 2;
    } else {
        a.focus = bp.tx_orientation == bp.rx_orientation ? 3 : 4;
    }

    // READI sub-signals, beamformer.cu:56-61, 100-137, 235-251.
    a.G = (int)(uint8_t)bp.readi_group_count;
    if (a.G == 0) a.G = 1;
    a.readi_row = 0;
    if (a.G > 1) {
        CUTB_REQUIRE(bp.decode != NONE, CUTB_ERR_INVALID_ARGUMENT,
                     "READI groups (%d) require a Hadamard or Walsh encoding.", a.G);
        const unsigned id = (uint8_t)bp.readi_group_id;
        CUTB_REQUIRE((int)id < a.G, CUTB_ERR_INVALID_ARGUMENT, "READI group id %u >= group count %d.", id, a.G);
        EncodingInfo enc;
        if (!build_encoding((unsigned)a.G, bp.decode, enc)) return false;
        for (int k = 0; k < a.G; ++k)
            if (enc.matrix[(size_t)id * a.G + k] < 0) a.readi_row |= 1ull << k;
    }

    if (a.seq == HERCULES) {
        CUTB_REQUIRE(a.focus == 2 || a.focus == 4, CUTB_ERR_UNSUPPORTED, "Invalid focus for HERCULES.");
        CUTB_REQUIRE(a.G <= 32, CUTB_ERR_UNSUPPORTED,
                     "HERCULES supports at most 32 READI groups (upstream packs the row in 32 bits).");
        a.apply_cf = a.cf_power > 0.f;
        a.use_apo = a.apo_type == RX_TO_SIN || a.fn_rx != 0.f;
    } else {
        CUTB_REQUIRE(a.G <= 64, CUTB_ERR_UNSUPPORTED, "FORCES supports at most 64 READI groups.");
        CUTB_REQUIRE(a.G == 1 || bp.decode == HADAMARD, CUTB_ERR_UNSUPPORTED,
                     "FORCES only supports Hadamard encoding at this time.");
        a.apply_cf = 1;
        a.use_apo = !(a.apo_type == RX_HANN && a.fn_rx == 0.f && a.fn_tx == 0.f);
    }
    // A zero f-number still skips voxels at zero depth upstream (0 * inf -> NaN -> window 0):
    // keep the general path if the grid reaches z = 0.
    const float zlast = fmaf((float)(a.Z - 1), a.res_z, a.vmin_z);
    if (!a.use_apo && fminf(a.vmin_z, zlast) <= 0.f) a.use_apo = 1;
    return true;
}

bool launch_das(const DasArgs& a, const void* iq, bool iq_bf16, void* volume, cudaStream_t st, int* launches)
{
    bool ok;
    if (a.seq == HERCULES)
        ok = iq_bf16 ? launch_das_s<HERCULES, __nv_bfloat162>(a, iq, volume, st)
                     : launch_das_s<HERCULES, float2>(a, iq, volume, st);
    else
        ok = iq_bf16 ? launch_das_s<FORCES, __nv_bfloat162>(a, iq, volume, st)
                     : launch_das_s<FORCES, float2>(a, iq, volume, st);
    if (ok && launches) ++*launches;
    return ok;
}

}  // namespace cutb
