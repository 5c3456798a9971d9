// Image correlation and NCC block-matching motion detection.
//
// Upstream (image_processing/image_processor.cpp, kernels/block_match_kernels.cu) runs, for every
// frame and every grid point, one NPP valid normalised cross-correlation
// (nppiCrossCorrValid_NormLevel_32f_C1R) into a global map, one CUB block radix sort of the
// first 2048 map values for the 32 best candidates and one warp kernel that fits a quadratic
// surface to each candidate's 3 x 3 neighbourhood, rejects flat, saddle or weak peaks and keeps
// the best: three launches and a global round trip per grid point, issued from the host.
//
// Here one launch covers every (frame, grid point): a CTA stages its template and search window
// in shared memory, forms the whole correlation map there, selects the 32 candidates with the
// same order as a stable descending radix sort (value, then lower map index) and runs the fit and
// the tests in one warp, whose shuffle-down reduction keeps upstream's tie order. Only the float4
// vector leaves the SM.
//
// Correlation of template T (n pixels) and source window S at one position:
//     rho = sum (S - c) T' / sqrt(var_S * var_T),   T' = T - mean(T),  c = rint(mean(T))
// with the numerator in FP32 (as NPP), and the window moments sum S_c, sum S_c^2 in FP64 so that
// n * sum S_c^2 - (sum S_c)^2 is exact for 8-bit-valued images and a flat window is recognised
// exactly; such a position (or a flat template) yields FLT_MAX, which is what upstream's NPP call
// returns there.
#include <cfloat>
#include <cstdint>

#include <algorithm>

#include "../../include/cuda_toolkit_b200_motion.h"
#include "common.cuh"
#include "stages.h"

namespace cutb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kCandidates = 32;     // find_peaks_kernel keeps the first 32 ranks
constexpr int kPerThread = 8;       // ... of 256 threads x 8 loaded map values
constexpr double kFlatTol = 1e-11;  // relative size of n*var below which a window counts as flat
constexpr size_t kMaxSmem = 200 * 1024;

// cub's float radix order: larger keys are larger floats, -0 below +0.
__device__ __forceinline__ uint32_t radix_key(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Same value in every thread: warp shuffles, then a fixed-order sum of the warp partials.
__device__ double block_sum(double v, double* red)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += red[w];
    return s;
}

// num / sqrt(var_S * var_T) with d = n * sum (S - mean S)^2 and tvn = sum T'^2 / n; the flat test
// in FP64, the final scale in FP32 (~3e-7 relative) unless the product leaves the FP32 range.
__device__ __forceinline__ float ncc_value(float num, double s1, double s2, double n, double tvn)
{
    const double d = n * s2 - s1 * s1;
    if (tvn <= 0.0 || d <= kFlatTol * n * s2) return FLT_MAX;
    const double x = d * tvn;
    if (x > 1e-30 && x < 1e30) return num * rsqrtf((float)x);
    return (float)((double)num / sqrt(x));
}

// Quadratic-surface weights on the 3 x 3 grid (x, y in {-1, 0, 1}) for the coefficients of
// a x^2 + b y^2 + c xy + d x + e y + f, from the normal equations of the least-squares fit.
__device__ __forceinline__ float fit_weight(int coeff, int x, int y)
{
    switch (coeff) {
        case 0: return x ? 1.f / 6.f : -1.f / 3.f;
        case 1: return y ? 1.f / 6.f : -1.f / 3.f;
        case 2: return (float)(x * y) / 4.f;
        case 3: return (float)x / 6.f;
        case 4: return (float)y / 6.f;
        default: return (5.f - 3.f * (float)(x * x + y * y)) / 9.f;
    }
}

struct Window {
    int tl, tt, tw, th;  // template window in the template frame
    int sl, st, sw, sh;  // search window in the source frame
};

// _compare_images (image_processor.cpp:146-195): the patch around grid point (gx_i, gy_i) and the
// search window `margins` around it, both clipped to the image.
__device__ __forceinline__ Window cell_window(const MotionArgs& a, int col, int row)
{
    Window w;
    int tt = row * a.spacing - a.patch / 2, tb = tt + a.patch - 1;
    int tl = col * a.spacing - a.patch / 2, tr = tl + a.patch - 1;
    const int st = max(tt - a.my, 0), sb = min(tb + a.my, a.H - 1);
    const int sl = max(tl - a.mx, 0), sr = min(tr + a.mx, a.W - 1);
    tt = max(tt, 0);
    tb = min(tb, a.H - 1);
    tl = max(tl, 0);
    tr = min(tr, a.W - 1);
    w.tl = tl;
    w.tt = tt;
    w.tw = tr - tl + 1;
    w.th = tb - tt + 1;
    w.sl = sl;
    w.st = st;
    w.sw = sr - sl + 1;
    w.sh = sb - st + 1;
    return w;
}

// Correlation map of the staged template (centred, tsm, row stride tws, zero beyond tw) over the
// staged window (ssm, row stride sws, shifted by c, zero beyond sw). Leaves cmap complete (after
// a barrier); h1/h2 (sh x cw doubles each) are scratch.
//
// Warps 0-1 form the window moments while warps 2-7 accumulate the numerators into cmap; then
// every thread turns numerator and moments into the coefficient.
//
// Window moments: FP64 running sums along each row, then down each column in place, so that
// h1/h2[oy][ox] end as sum S_c and sum S_c^2 over the window at (ox, oy). Exact for
// integer-valued images; otherwise ~1e-15 relative.
//
// Numerator: each thread accumulates a strip of 8 consecutive map positions of one row; per 4
// template columns it loads 4 new window values and 4 template values as float4 and issues 32
// FMAs (the template-column loop is unrolled completely for 16- and 32-wide templates).
// Consecutive lanes take consecutive rows; the row stride is 4 (mod 8) words, so the 8 lanes of
// a 16-byte load phase hit 8 different bank quads.
constexpr int kStrip = 8;
constexpr int kMomentWarps = 2;
constexpr int kMomentThreads = 32 * kMomentWarps;

__device__ __forceinline__ void strip_fma(float (&acc)[kStrip], const float4& a, const float4& b, const float4& c,
                                          const float4& t)
{
    const float w[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    const float tv[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
    for (int qq = 0; qq < 4; ++qq)
#pragma unroll
        for (int k = 0; k < kStrip; ++k) acc[k] = fmaf(w[k + qq], tv[qq], acc[k]);
}

// QB = template float4 columns when known at compile time, 0 for any width.
template <int QB>
__device__ __forceinline__ void numerator_strips(const float* ssm, int sws, const float* tsm, int tws, int th, int cw,
                                                 int ch, int qblocks, float* cmap, int tid, int nthreads)
{
    const int nsx = (cw + kStrip - 1) / kStrip;
    for (int j = tid; j < nsx * ch; j += nthreads) {
        const int oy = j % ch, ox0 = (j / ch) * kStrip;
        float acc[kStrip];
#pragma unroll
        for (int k = 0; k < kStrip; ++k) acc[k] = 0.f;
        for (int r = 0; r < th; ++r) {
            const float4* srow = reinterpret_cast<const float4*>(ssm + (oy + r) * sws + ox0);
            const float4* trow = reinterpret_cast<const float4*>(tsm + r * tws);
            float4 a = srow[0], b = srow[1];
            if constexpr (QB > 0) {
#pragma unroll
                for (int qb = 0; qb < QB; ++qb) {
                    const float4 c = srow[qb + 2];
                    strip_fma(acc, a, b, c, trow[qb]);
                    a = b;
                    b = c;
                }
            } else {
                for (int qb = 0; qb < qblocks; ++qb) {
                    const float4 c = srow[qb + 2];
                    strip_fma(acc, a, b, c, trow[qb]);
                    a = b;
                    b = c;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kStrip; ++k)
            if (ox0 + k < cw) cmap[oy * cw + ox0 + k] = acc[k];
    }
}

__device__ void window_moments(const float* ssm, int sws, int tw, int th, int cw, int ch, double* h1, double* h2,
                               int tid)
{
    const int sh = ch + th - 1;
    for (int y = tid; y < sh; y += kMomentThreads) {
        const float* r = ssm + y * sws;
        double a = 0, b = 0;
        for (int q = 0; q < tw; ++q) {
            const double v = r[q];
            a += v;
            b = fma(v, v, b);
        }
        h1[y * cw] = a;
        h2[y * cw] = b;
        for (int ox = 1; ox < cw; ++ox) {
            const double vin = r[ox + tw - 1], vout = r[ox - 1];
            a += vin - vout;
            b += fma(vin, vin, -vout * vout);
            h1[y * cw + ox] = a;
            h2[y * cw + ox] = b;
        }
    }
    asm volatile("bar.sync 1, %0;" ::"n"(kMomentThreads) : "memory");
    for (int ox = tid; ox < cw; ox += kMomentThreads) {
        double a = 0, b = 0;
        for (int r = 0; r < th; ++r) {
            a += h1[r * cw + ox];
            b += h2[r * cw + ox];
        }
        for (int oy = 0; oy < ch; ++oy) {
            const int i = oy * cw + ox;
            double na = a, nb = b;
            if (oy + 1 < ch) {
                na += h1[i + th * cw] - h1[i];
                nb += h2[i + th * cw] - h2[i];
            }
            h1[i] = a;  // row oy is not read again by this column
            h2[i] = b;
            a = na;
            b = nb;
        }
    }
}

__device__ void corr_map_smem(const float* ssm, int sws, const float* tsm, int tws, int tw, int th, int cw, int ch,
                              double tvar, double* h1, double* h2, float* cmap)
{
    const int warp = threadIdx.x >> 5;
    if (warp < kMomentWarps) {
        window_moments(ssm, sws, tw, th, cw, ch, h1, h2, threadIdx.x);
    } else {
        const int tid = threadIdx.x - kMomentThreads, nt = kThreads - kMomentThreads;
        const int qblocks = tws / 4;
        if (qblocks == 8)
            numerator_strips<8>(ssm, sws, tsm, tws, th, cw, ch, qblocks, cmap, tid, nt);
        else if (qblocks == 4)
            numerator_strips<4>(ssm, sws, tsm, tws, th, cw, ch, qblocks, cmap, tid, nt);
        else
            numerator_strips<0>(ssm, sws, tsm, tws, th, cw, ch, qblocks, cmap, tid, nt);
    }
    __syncthreads();
    const double n = (double)tw * th, tvn = tvar / n;
    for (int i = threadIdx.x; i < cw * ch; i += kThreads) cmap[i] = ncc_value(cmap[i], h1[i], h2[i], n, tvn);
    __syncthreads();
}

// find_peaks_kernel (block_match_kernels.cu:8-61): the 32 largest of the first 2048 map values
// (-1 past the end of the map), larger value first, equal values by lower index; written to
// cand[0..31] as map indices. Keys are (radix order of the value, complement of the index), so the
// order is that of a 64-bit maximum and every key is unique. Two levels, one block barrier: each
// warp draws the 32 largest of its 256 keys (every thread keeps its 8 sorted and the owner of each
// warp maximum drops it), then warp 0 draws the 32 largest of the 8 sorted lists.
__device__ __forceinline__ unsigned long long warp_max64(unsigned long long v)
{
    // high words first, then low words among the lanes that hold the highest high word
    const uint32_t hi = (uint32_t)(v >> 32), lo = (uint32_t)v;
    const uint32_t mh = __reduce_max_sync(0xffffffffu, hi);
    const uint32_t ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
    return ((unsigned long long)mh << 32) | ml;
}

// 32 rounds: the warp maximum of the lanes' heads, dropped by its owner. Lane r receives the r-th.
template <int K>
__device__ __forceinline__ unsigned long long warp_top32(unsigned long long (&key)[K])
{
    const int lane = threadIdx.x & 31;
    unsigned long long mine = 0;
    for (int round = 0; round < kCandidates; ++round) {
        const unsigned long long m = warp_max64(key[0]);
        if (key[0] == m) {
#pragma unroll
            for (int i = 0; i + 1 < K; ++i) key[i] = key[i + 1];
            key[K - 1] = 0ull;
        }
        if (lane == round) mine = m;
    }
    return mine;
}

__device__ void select_candidates(const float* cmap, int n, int* cand, unsigned long long* lists)
{
    unsigned long long key[kPerThread];
#pragma unroll
    for (int i = 0; i < kPerThread; ++i) {
        const int idx = threadIdx.x * kPerThread + i;
        const float v = idx < n ? cmap[idx] : -1.0f;
        key[i] = ((unsigned long long)radix_key(v) << 32) | (0xFFFFFFFFu - (uint32_t)idx);
    }
#pragma unroll
    for (int i = 1; i < kPerThread; ++i)
#pragma unroll
        for (int j = kPerThread - 1; j >= i; --j)
            if (key[j] > key[j - 1]) {
                const unsigned long long t = key[j];
                key[j] = key[j - 1];
                key[j - 1] = t;
            }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    lists[warp * kCandidates + lane] = warp_top32(key);  // each list sorted, largest first
    __syncthreads();
    if (warp == 0) {
        // lane l holds entries 8 (l % 4) .. 8 (l % 4) + 7 of warp (l / 4)'s list: already sorted
        unsigned long long k[kPerThread];
#pragma unroll
        for (int i = 0; i < kPerThread; ++i) k[i] = lists[lane * kPerThread + i];
        const unsigned long long best = warp_top32(k);
        cand[lane] = (int)(0xFFFFFFFFu - (uint32_t)best);
    }
    __syncthreads();
}

// test_peaks (block_match_kernels.cu:64-188), one lane per candidate, on warp 0.
__device__ void test_candidates(const float* cmap, int cw, int ch, const int* cand, int nsx, int nsy,
                                const MotionArgs& a, float4* out)
{
    const int lane = threadIdx.x & 31;
    const int n = cw * ch;
    const int idx = cand[lane];
    float peak = idx < n ? cmap[idx] : -1.0f;
    const int px = idx % cw, py = idx / cw;
    float v[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int y = py + k / 3 - 1, x = px + k % 3 - 1;
        v[k] = (y >= 0 && y < ch && x >= 0 && x < cw) ? cmap[y * cw + x] : 0.f;
    }
    float c[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 9; ++k) s = fmaf(fit_weight(i, k % 3 - 1, k / 3 - 1), v[k], s);
        c[i] = s;
    }
    // Hessian eigenvalues (times 1/2) and the stationary point of the fitted surface.
    float r2 = c[0] * c[0];
    r2 = fmaf(c[1], c[1], r2);
    r2 = fmaf(c[2], c[2], r2);
    r2 = fmaf(-2.f * c[0], c[1], r2);
    const float root = sqrtf(r2);
    const float s0 = c[0] + c[1] + root, s1 = c[0] + c[1] - root;
    const float min_sharp = fminf(fabsf(s0), fabsf(s1));
    const float den = fmaf(c[2], c[2], -4.f * c[1] * c[0]);
    float ox = 0.f, oy = 0.f;
    if (den != 0.f) {
        ox = fmaf(2.f * c[1], c[3], -c[2] * c[4]) / den;
        oy = fmaf(2.f * c[0], c[4], -c[2] * c[3]) / den;
    }
    ox = a.subpixel ? fminf(fmaxf(ox, -1.f), 1.f) : 0.f;
    oy = a.subpixel ? fminf(fmaxf(oy, -1.f), 1.f) : 0.f;
    float tx = (ox + (float)px) - (float)nsx;
    float ty = (oy + (float)py) - (float)nsy;
    const float no_shift = cmap[nsy * cw + nsx];
    const float threshold = no_shift * (1.0f + a.rel_thr);
    if (min_sharp < a.sharp_thr || s0 >= 0.f || peak > 1.0f || peak < threshold) peak = -2.0f;
    // warp_reduce_max: shuffle-down tree, strict comparison (ties keep the lower half)
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float p2 = __shfl_down_sync(0xffffffffu, peak, o);
        const float x2 = __shfl_down_sync(0xffffffffu, tx, o);
        const float y2 = __shfl_down_sync(0xffffffffu, ty, o);
        if (p2 > peak) {
            peak = p2;
            tx = x2;
            ty = y2;
        }
    }
    if (lane == 0) {
        if (peak < a.abs_thr || peak <= no_shift) {
            tx = ty = 0.f;
            if (peak < threshold) peak = -1.0f;
        }
        *out = make_float4(tx, ty, peak, no_shift);
    }
}

struct MotionSmem {
    size_t h_off, s_off, t_off, c_off, bytes;
    int sws, tws;
};

// Window rows hold the strips' overrun (up to index sw + 10) at a stride of 4 (mod 8) words; template
// rows are padded to whole float4s.
__host__ __device__ inline MotionSmem motion_smem(const MotionArgs& a)
{
    MotionSmem m;
    const int sw = a.sw_max, sh = a.sh_max, cw = a.cw_max, ch = a.ch_max;
    const int base = sw + 11;  // strips read up to index sw + 10
    m.sws = base + (12 - base % 8) % 8;  // smallest stride >= base that is 4 (mod 8)
    m.tws = (a.tw_max + 3) / 4 * 4;
    m.h_off = 0;
    m.s_off = m.h_off + 2 * sizeof(double) * (size_t)sh * cw;
    m.t_off = m.s_off + sizeof(float) * (size_t)sh * m.sws;
    m.c_off = m.t_off + sizeof(float) * (size_t)m.tws * a.th_max;
    m.bytes = m.c_off + sizeof(float) * (size_t)cw * ch;
    return m;
}

__global__ void __launch_bounds__(kThreads, 3) block_match_kernel(MotionArgs a)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ double red[kWarps];
    __shared__ unsigned long long lists[kWarps * kCandidates];
    __shared__ int cand[kCandidates];

    const int cell = blockIdx.x, pair = blockIdx.y;
    const int col = cell % a.gx, row = cell / a.gx;
    // ncc_block_match (image_processor.cpp:25-44): every frame but the reference, against the
    // reference or, with neighbour_compare, against its neighbour towards the reference.
    const int f = pair < a.ref ? pair : pair + 1;
    const int tf = a.neighbour ? (a.ref > f ? f + 1 : f - 1) : a.ref;
    const Window w = cell_window(a, col, row);
    // An empty patch (grid point outside the image) fails upstream's correlation call before the
    // peak kernels run; the vector keeps the cleared value.
    if (w.tw < 1 || w.th < 1) return;
    const int cw = w.sw - w.tw + 1, ch = w.sh - w.th + 1;

    const MotionSmem L = motion_smem(a);
    double* h1 = reinterpret_cast<double*>(smem + L.h_off);
    double* h2 = h1 + (size_t)w.sh * cw;
    float* ssm = reinterpret_cast<float*>(smem + L.s_off);
    float* tsm = reinterpret_cast<float*>(smem + L.t_off);
    float* cmap = reinterpret_cast<float*>(smem + L.c_off);

    const size_t frame_px = (size_t)a.W * a.H;
    const float* T = a.frames + (size_t)tf * frame_px + (size_t)w.tt * a.W + w.tl;
    const float* S = a.frames + (size_t)f * frame_px + (size_t)w.st * a.W + w.sl;
    const int nt = w.tw * w.th, tws = (w.tw + 3) / 4 * 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double part = 0;
    for (int y = warp; y < w.th; y += kWarps)
        for (int x = lane; x < tws; x += 32) {
            const float v = x < w.tw ? __ldg(T + (size_t)y * a.W + x) : 0.f;
            tsm[y * tws + x] = v;
            part += v;
        }
    const double mean = block_sum(part, red) / (double)nt;
    const float shift = rintf((float)mean);
    part = 0;
    for (int y = warp; y < w.th; y += kWarps)
        for (int x = lane; x < w.tw; x += 32) {
            const float d = (float)((double)tsm[y * tws + x] - mean);
            tsm[y * tws + x] = d;
            part = fma((double)d, (double)d, part);
        }
    const double tvar = block_sum(part, red);
    for (int y = warp; y < w.sh; y += kWarps)
        for (int x = lane; x < L.sws; x += 32)
            ssm[y * L.sws + x] = x < w.sw ? __ldg(S + (size_t)y * a.W + x) - shift : 0.f;
    __syncthreads();
    corr_map_smem(ssm, L.sws, tsm, tws, w.tw, w.th, cw, ch, tvar, h1, h2, cmap);
    select_candidates(cmap, cw * ch, cand, lists);
    if (threadIdx.x < 32)
        test_candidates(cmap, cw, ch, cand, w.tl - w.sl, w.tt - w.st, a,
                        reinterpret_cast<float4*>(a.maps) + ((size_t)f * a.gx * a.gy + cell));
}

// ---- corr_images: template statistics, window row moments, tiled correlation ------------------

constexpr int kTileX = 64, kTileY = 16;   // outputs per CTA (256 threads x 4 along x)
constexpr int kTileStrip = 4;
constexpr int kChunkX = 32, kChunkY = 16; // template block staged per step

struct TplStats {
    double mean, tvar;
    float shift;
};

__global__ void __launch_bounds__(1024) template_stats_kernel(const float* __restrict__ tpl, int n, float* centred,
                                                              TplStats* st)
{
    __shared__ double red[32];
    auto sum = [&](double v) {
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        double s = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
        return s;
    };
    double p = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) p += tpl[i];
    const double mean = sum(p) / (double)n;
    p = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float d = (float)((double)tpl[i] - mean);
        centred[i] = d;
        p = fma((double)d, (double)d, p);
    }
    const double tvar = sum(p);
    if (threadIdx.x == 0) *st = TplStats{mean, tvar, rintf((float)mean)};
}

// h[y][ox] = sum_{q < tw} S_c[y][ox + q] and the sum of squares, FP64.
__global__ void __launch_bounds__(kThreads) row_moments_kernel(const float* __restrict__ src, int sw, int sh, int tw,
                                                               int cw, const TplStats* st, double2* __restrict__ h)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (i >= (long long)sh * cw) return;
    const int y = (int)(i / cw), ox = (int)(i - (long long)y * cw);
    const float c = st->shift;
    const float* r = src + (size_t)y * sw + ox;
    double a = 0, b = 0;
    for (int q = 0; q < tw; ++q) {
        const double v = __ldg(r + q) - c;
        a += v;
        b = fma(v, v, b);
    }
    h[i] = make_double2(a, b);
}

__global__ void __launch_bounds__(kThreads) corr_tile_kernel(const float* __restrict__ src, int sw, int sh,
                                                             const float* __restrict__ tc, int tw, int th,
                                                             const TplStats* st, const double2* __restrict__ h,
                                                             float* __restrict__ out)
{
    constexpr int kSW = kTileX + kChunkX - 1 + kTileStrip - 1;  // staged window width (with strip overrun)
    constexpr int kSH = kTileY + kChunkY - 1;
    __shared__ float ssm[kSH][kSW];
    __shared__ float tsm[kChunkY][kChunkX];
    const int cw = sw - tw + 1, ch = sh - th + 1;
    const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY;
    const int tx = threadIdx.x % (kTileX / kTileStrip), ty = threadIdx.x / (kTileX / kTileStrip);
    const float c = st->shift;
    float acc[kTileStrip] = {0.f, 0.f, 0.f, 0.f};
    for (int r0 = 0; r0 < th; r0 += kChunkY)
        for (int q0 = 0; q0 < tw; q0 += kChunkX) {
            const int rn = min(kChunkY, th - r0), qn = min(kChunkX, tw - q0);
            __syncthreads();
            for (int i = threadIdx.x; i < kChunkY * kChunkX; i += kThreads) {
                const int r = i / kChunkX, q = i % kChunkX;
                tsm[r][q] = (r < rn && q < qn) ? tc[(size_t)(r0 + r) * tw + q0 + q] : 0.f;
            }
            for (int i = threadIdx.x; i < kSH * kSW; i += kThreads) {
                const int y = i / kSW, x = i % kSW;
                const int sy = y0 + r0 + y, sx = x0 + q0 + x;
                ssm[y][x] = (sy < sh && sx < sw) ? __ldg(src + (size_t)sy * sw + sx) - c : 0.f;
            }
            __syncthreads();
            for (int r = 0; r < rn; ++r) {
                const float* srow = &ssm[ty + r][tx * kTileStrip];
                float s0 = srow[0], s1 = srow[1], s2 = srow[2];
                for (int q = 0; q < qn; ++q) {
                    const float s3 = srow[q + 3];
                    const float t = tsm[r][q];
                    acc[0] = fmaf(s0, t, acc[0]);
                    acc[1] = fmaf(s1, t, acc[1]);
                    acc[2] = fmaf(s2, t, acc[2]);
                    acc[3] = fmaf(s3, t, acc[3]);
                    s0 = s1;
                    s1 = s2;
                    s2 = s3;
                }
            }
        }
    const int oy = y0 + ty;
    if (oy >= ch) return;
    const double n = (double)tw * th, tvn = st->tvar / n;
#pragma unroll
    for (int k = 0; k < kTileStrip; ++k) {
        const int ox = x0 + tx * kTileStrip + k;
        if (ox >= cw) break;
        double m1 = 0, m2 = 0;
        for (int r = 0; r < th; ++r) {
            const double2 v = h[(size_t)(oy + r) * cw + ox];
            m1 += v.x;
            m2 += v.y;
        }
        out[(size_t)oy * cw + ox] = ncc_value(acc[k], m1, m2, n, tvn);
    }
}

}  // namespace

bool launch_block_match(const MotionArgs& args, cudaStream_t st)
{
    MotionArgs a = args;
    CUTB_REQUIRE(a.frames && a.maps, CUTB_ERR_INVALID_ARGUMENT, "Motion detection: null buffer.");
    CUTB_REQUIRE(((uintptr_t)a.maps & 15) == 0, CUTB_ERR_INVALID_ARGUMENT,
                 "Motion detection: the motion maps must be 16-byte aligned (float4 vectors).");
    CUTB_REQUIRE(a.W > 0 && a.H > 0 && a.F > 0 && a.patch > 0, CUTB_ERR_INVALID_ARGUMENT,
                 "Motion detection: image size, frame count and patch size must be positive.");
    CUTB_REQUIRE(a.ref >= 0 && a.ref < a.F, CUTB_ERR_INVALID_ARGUMENT,
                 "Motion detection: reference frame %d outside the %d frames.", a.ref, a.F);
    CUTB_REQUIRE(a.mx >= 0 && a.my >= 0 && a.spacing >= 0, CUTB_ERR_INVALID_ARGUMENT,
                 "Motion detection: negative margins or spacing.");
    const size_t cells = (size_t)a.gx * a.gy;
    CUTB_CUDA_OK(cudaMemsetAsync(a.maps, 0, cells * a.F * 4 * sizeof(float), st));
    if (cells == 0 || a.F == 1) return true;
    CUTB_REQUIRE(cells <= 0x7fffffffu && a.F - 1 <= 65535, CUTB_ERR_UNSUPPORTED,
                 "Motion detection: at most 2^31 grid points and 65536 frames.");
    // Largest windows any grid point can have (the clipped ones are smaller).
    a.tw_max = min(a.patch, a.W);
    a.th_max = min(a.patch, a.H);
    a.sw_max = (int)std::min<long long>((long long)a.patch + 2ll * a.mx, a.W);
    a.sh_max = (int)std::min<long long>((long long)a.patch + 2ll * a.my, a.H);
    a.cw_max = min(2 * a.mx + 1, a.sw_max);
    a.ch_max = min(2 * a.my + 1, a.sh_max);
    const MotionSmem L = motion_smem(a);
    CUTB_REQUIRE(L.bytes <= kMaxSmem, CUTB_ERR_UNSUPPORTED,
                 "Motion detection: a %d x %d search window with a %d-pixel patch needs %zu bytes of shared memory "
                 "(limit %zu).",
                 a.sw_max, a.sh_max, a.patch, L.bytes, kMaxSmem);
    CUTB_CUDA_OK(cudaFuncSetAttribute(block_match_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes));
    block_match_kernel<<<dim3((unsigned)cells, (unsigned)(a.F - 1)), kThreads, L.bytes, st>>>(a);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

bool launch_corr_images(const float* tpl, int tw, int th, const float* src, int sw, int sh, float* out,
                        cudaStream_t st)
{
    CUTB_REQUIRE(tpl && src && out, CUTB_ERR_INVALID_ARGUMENT, "corr_images: null buffer.");
    CUTB_REQUIRE(tw > 0 && th > 0 && sw > 0 && sh > 0, CUTB_ERR_INVALID_ARGUMENT,
                 "Invalid image dimensions for corr_images.");
    CUTB_REQUIRE(tw <= sw && th <= sh, CUTB_ERR_INVALID_ARGUMENT,
                 "Template dimensions must be <= source dimensions for corr_images.");
    const int cw = sw - tw + 1, ch = sh - th + 1;
    const size_t tbytes = sizeof(float) * (size_t)tw * th, hbytes = sizeof(double2) * (size_t)sh * cw;
    CUTB_REQUIRE(div_up((long long)ch, (long long)kTileY) <= 65535, CUTB_ERR_UNSUPPORTED,
                 "corr_images: correlation map too tall.");
    uint8_t* scratch = nullptr;
    const size_t stats_off = 0, tc_off = 256, h_off = tc_off + (tbytes + 255) / 256 * 256;
    CUTB_CUDA_OK(cudaMallocAsync((void**)&scratch, h_off + hbytes, st));
    TplStats* stats = reinterpret_cast<TplStats*>(scratch + stats_off);
    float* tc = reinterpret_cast<float*>(scratch + tc_off);
    double2* h = reinterpret_cast<double2*>(scratch + h_off);
    template_stats_kernel<<<1, 1024, 0, st>>>(tpl, tw * th, tc, stats);
    row_moments_kernel<<<(unsigned)div_up((long long)sh * cw, (long long)kThreads), kThreads, 0, st>>>(
        src, sw, sh, tw, cw, stats, h);
    corr_tile_kernel<<<dim3((unsigned)div_up(cw, kTileX), (unsigned)div_up(ch, kTileY)), kThreads, 0, st>>>(
        src, sw, sh, tc, tw, th, stats, h, out);
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(scratch, st);
    CUTB_CUDA_OK(e);
    return true;
}

}  // namespace cutb

using namespace cutb;

extern "C" {

CUTB_API bool cutb_corr_images(const float* d_template, const float* d_source, const uint tpl_dims[2],
                               const uint src_dims[2], float* d_corr, void* stream)
{
    CUTB_REQUIRE(tpl_dims && src_dims, CUTB_ERR_INVALID_ARGUMENT, "corr_images: null dimension array.");
    CUTB_REQUIRE(tpl_dims[0] <= 0x7fffffffu && tpl_dims[1] <= 0x7fffffffu && src_dims[0] <= 0x7fffffffu &&
                     src_dims[1] <= 0x7fffffffu,
                 CUTB_ERR_INVALID_ARGUMENT, "Invalid image dimensions for corr_images.");
    return launch_corr_images(d_template, (int)tpl_dims[0], (int)tpl_dims[1], d_source, (int)src_dims[0],
                              (int)src_dims[1], d_corr, (cudaStream_t)stream);
}

CUTB_API bool cutb_motion_detection(const float* d_frames, const NccMotionParameters* p, float* d_maps, void* stream)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Motion detection: null parameters.");
    for (uint v : {p->patch_size, p->motion_grid_spacing, p->motion_grid_dims[0], p->motion_grid_dims[1],
                   p->search_margins[0], p->search_margins[1], p->frame_count, p->image_dims[0], p->image_dims[1]})
        CUTB_REQUIRE(v <= 0x7fffffu, CUTB_ERR_INVALID_ARGUMENT, "Motion detection: parameter value %u too large.", v);
    MotionArgs a{};
    a.frames = d_frames;
    a.maps = d_maps;
    a.W = (int)p->image_dims[0];
    a.H = (int)p->image_dims[1];
    a.F = (int)p->frame_count;
    a.patch = (int)p->patch_size;
    a.spacing = (int)p->motion_grid_spacing;
    a.gx = (int)p->motion_grid_dims[0];
    a.gy = (int)p->motion_grid_dims[1];
    a.mx = (int)p->search_margins[0];
    a.my = (int)p->search_margins[1];
    a.ref = p->reference_frame <= 0x7fffffu ? (int)p->reference_frame : -1;
    a.neighbour = p->neighbour_compare ? 1 : 0;
    a.subpixel = p->use_subpixel ? 1 : 0;
    a.abs_thr = p->abs_cor_threshold;
    a.rel_thr = p->rel_cor_threshold;
    a.sharp_thr = p->min_patch_variance;
    return launch_block_match(a, (cudaStream_t)stream);
}

}  // extern "C"
