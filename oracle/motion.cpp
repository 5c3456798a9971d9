/*
 * ORACLE — CPU restatement of the upstream toolkit's image-correlation and NCC motion-detection
 * path. TEST INFRASTRUCTURE ONLY (see oracle.cpp): tests/ load it as the checker; the product
 * library never links, loads or calls it.
 *
 *   orc_corr_images       <- ImageProcessor::corr_images (image_processing/image_processor.cpp:
 *                            55-128): NPP nppiCrossCorrValid_NormLevel_32f_C1R, the zero-mean
 *                            normalised cross-correlation of a template at every fully
 *                            overlapping position of a source image.
 *   orc_motion_detection  <- ImageProcessor::ncc_block_match and _compare_images
 *                            (image_processor.cpp:9-52, 130-228) with block_match_pipeline,
 *                            find_peaks_kernel and test_peaks (kernels/block_match_kernels.cu).
 *
 * Correlations are formed in FP64 and rounded to FP32 (upstream's maps are FP32); the peak
 * selection, the quadratic fit and the tests run in FP64 on those FP32 values.
 *
 * Pinning: tests/golden/ncc.npz holds outputs of upstream's own pipeline (its sources compiled
 * unmodified for the GPU with NPP, oracle/Makefile.ref target `ncc`, driven by
 * tests/golden/make_ncc_golden.py); tests/test_golden.py checks this restatement against it.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/cuda_beamformer_parameters.h"

namespace {

// Quadratic-surface fit f = a x^2 + b y^2 + c xy + d x + e y + f0 over a 3 x 3 neighbourhood
// (row-major, y = -1..1 outer, x = -1..1 inner): least-squares weights of block_match_kernels.cuh
// P3, restated from the normal equations (coefficient order a, b, c, d, e, f0).
void fit3x3(const double v[9], double coeff[6])
{
    double sx2 = 0, sy2 = 0, sxy = 0, sx = 0, sy = 0, s = 0;
    for (int k = 0; k < 9; ++k) {
        const int y = k / 3 - 1, x = k % 3 - 1;
        s += v[k];
        sx += x * v[k];
        sy += y * v[k];
        sxy += x * y * v[k];
        sx2 += x * x * v[k];
        sy2 += y * y * v[k];
    }
    // Solution of the normal equations on the grid {-1, 0, 1}^2 in terms of the moments above.
    coeff[0] = (sx2 - 2.0 / 3.0 * s) / 2.0;
    coeff[1] = (sy2 - 2.0 / 3.0 * s) / 2.0;
    coeff[2] = sxy / 4.0;
    coeff[3] = sx / 6.0;
    coeff[4] = sy / 6.0;
    coeff[5] = (5.0 * s - 3.0 * (sx2 + sy2)) / 9.0;
}

// Order of cub's float radix sort: the IEEE bits with the sign flipped for positives and every
// bit flipped for negatives, so larger keys are larger floats (-0 < +0).
uint32_t radix_key(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

uint32_t bit_reverse5(uint32_t i)
{
    uint32_t r = 0;
    for (int b = 0; b < 5; ++b) r |= ((i >> b) & 1u) << (4 - b);
    return r;
}

// Zero-mean NCC of template t (tw x th) at every valid offset of source s (row stride ss), FP64.
// A position where the source window or the template has zero variance yields FLT_MAX, as NPP's
// nppiCrossCorrValid_NormLevel_32f_C1R does (observed on upstream's pipeline, tests/golden/ncc.npz).
constexpr float kZeroVariance = 3.402823466e38f;

void corr_valid(const float* t, int tw, int th, size_t ts, const float* s, int sw, int sh, size_t ss, float* out)
{
    const int cw = sw - tw + 1, ch = sh - th + 1;
    const double n = (double)tw * th;
    double tsum = 0;
    for (int y = 0; y < th; ++y)
        for (int x = 0; x < tw; ++x) tsum += t[y * ts + x];
    const double tmean = tsum / n;
    std::vector<double> tc((size_t)tw * th);
    double tvar = 0;
    for (int y = 0; y < th; ++y)
        for (int x = 0; x < tw; ++x) {
            tc[(size_t)y * tw + x] = t[y * ts + x] - tmean;
            tvar += tc[(size_t)y * tw + x] * tc[(size_t)y * tw + x];
        }
    for (int oy = 0; oy < ch; ++oy)
        for (int ox = 0; ox < cw; ++ox) {
            double ssum = 0;
            for (int y = 0; y < th; ++y)
                for (int x = 0; x < tw; ++x) ssum += s[(oy + y) * ss + ox + x];
            const double smean = ssum / n;
            double num = 0, svar = 0;
            for (int y = 0; y < th; ++y)
                for (int x = 0; x < tw; ++x) {
                    const double d = s[(oy + y) * ss + ox + x] - smean;
                    num += d * tc[(size_t)y * tw + x];
                    svar += d * d;
                }
            const double den = std::sqrt(svar * tvar);
            out[(size_t)oy * cw + ox] = den > 0 ? (float)(num / den) : kZeroVariance;
        }
}

struct Vec4 {
    float x, y, z, w;
};

// One grid point: block_match_pipeline (block_match_kernels.cu:190-241) on the corr map.
Vec4 match_point(const float* corr, int cw, int ch, int nsx, int nsy, const NccMotionParameters& p)
{
    const int n = cw * ch;
    // find_peaks_kernel: the first 2048 map values (256 threads x 8), -1 beyond the map, sorted
    // descending by a stable radix sort; the first 32 ranks are the candidates.
    constexpr int kLoad = 2048, kCand = 32;
    std::vector<std::pair<uint64_t, int>> keys(kLoad);
    for (int i = 0; i < kLoad; ++i) {
        const float v = i < n ? corr[i] : -1.0f;
        keys[i] = {((uint64_t)radix_key(v) << 32) | (uint32_t)(0xFFFFFFFFu - (uint32_t)i), i};
    }
    std::partial_sort(keys.begin(), keys.begin() + kCand, keys.end(),
                      [](const auto& a, const auto& b) { return a.first > b.first; });
    const float no_shift = corr[nsy * cw + nsx];
    const double threshold = (double)no_shift * (1.0 + (double)p.rel_cor_threshold);
    // test_peaks: one lane per candidate.
    double best = 0, bx = 0, by = 0;
    uint32_t best_rank = 0xFFFFFFFFu;
    for (int lane = 0; lane < kCand; ++lane) {
        const int idx = keys[lane].second;
        const float pk = idx < n ? corr[idx] : -1.0f;
        const int px = idx % cw, py = idx / cw;
        double v[9] = {0};
        for (int dy = -1; dy <= 1; ++dy) {
            if (py + dy < 0 || py + dy >= ch) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                if (px + dx < 0 || px + dx >= cw) continue;
                v[(dy + 1) * 3 + dx + 1] = corr[(py + dy) * cw + px + dx];
            }
        }
        double c[6];
        fit3x3(v, c);
        const double root = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2] - 2 * c[0] * c[1]);
        const double s0 = c[0] + c[1] + root, s1 = c[0] + c[1] - root;
        const double min_sharp = std::min(std::fabs(s0), std::fabs(s1));
        const double den = c[2] * c[2] - 4 * c[1] * c[0];
        double ox = 0, oy = 0;
        if (den != 0) {
            ox = (2 * c[1] * c[3] - c[2] * c[4]) / den;
            oy = (2 * c[0] * c[4] - c[2] * c[3]) / den;
        }
        ox = p.use_subpixel ? std::min(std::max(ox, -1.0), 1.0) : 0.0;
        oy = p.use_subpixel ? std::min(std::max(oy, -1.0), 1.0) : 0.0;
        double peak = pk;
        if (min_sharp < p.min_patch_variance || s0 >= 0 || peak > 1.0 || peak < threshold) peak = -2.0;
        // warp_reduce_max: a shuffle-down tree keeping the lower half on ties, so among equal
        // maxima the lane with the smallest bit-reversed index wins.
        const uint32_t rank = bit_reverse5((uint32_t)lane);
        if (best_rank == 0xFFFFFFFFu || peak > best || (peak == best && rank < best_rank)) {
            best = peak;
            best_rank = rank;
            bx = ox + px - nsx;
            by = oy + py - nsy;
        }
    }
    if (best < p.abs_cor_threshold || best <= no_shift) {
        bx = by = 0;
        if (best < threshold) best = -1.0;
    }
    return {(float)bx, (float)by, (float)best, no_shift};
}

}  // namespace

extern "C" {

// corr = (sw - tw + 1) x (sh - th + 1), row-major; images row-major with width the fast axis.
int orc_corr_images(const float* tpl, unsigned tw, unsigned th, const float* src, unsigned sw, unsigned sh, float* corr)
{
    if (!tw || !th || !sw || !sh || tw > sw || th > sh) return -1;
    corr_valid(tpl, (int)tw, (int)th, tw, src, (int)sw, (int)sh, sw, corr);
    return 0;
}

// images: frame_count frames of image_dims[0] x image_dims[1] (width fastest); maps:
// frame_count x motion_grid_dims[1] x motion_grid_dims[0] x (dx, dy, peak, no-shift peak).
int orc_motion_detection(const float* images, const NccMotionParameters* pp, float* maps, int nthreads)
{
    const NccMotionParameters& p = *pp;
    const int W = (int)p.image_dims[0], H = (int)p.image_dims[1];
    const int gx = (int)p.motion_grid_dims[0], gy = (int)p.motion_grid_dims[1];
    const int F = (int)p.frame_count, P = (int)p.patch_size, sp = (int)p.motion_grid_spacing;
    const int mx = (int)p.search_margins[0], my = (int)p.search_margins[1];
    if (F < 1 || W < 1 || H < 1 || P < 1 || p.reference_frame >= p.frame_count) return -1;
    std::memset(maps, 0, sizeof(float) * 4 * (size_t)F * gx * gy);
    struct Job {
        int frame, tframe, cell;
    };
    std::vector<Job> jobs;
    for (int f = 0; f < F; ++f) {
        int ref = (int)p.reference_frame;
        if (f == ref) continue;
        if (p.neighbour_compare) ref = ref > f ? f + 1 : f - 1;
        for (int c = 0; c < gx * gy; ++c) jobs.push_back({f, ref, c});
    }
    const size_t frame_px = (size_t)W * H;
    auto work = [&](size_t lo, size_t hi) {
        std::vector<float> corr;
        for (size_t j = lo; j < hi; ++j) {
            const Job& jb = jobs[j];
            const int i = jb.cell / gx, k = jb.cell % gx;
            int tt = i * sp - P / 2, tb = tt + P - 1, tl = k * sp - P / 2, tr = tl + P - 1;
            int st = std::max(tt - my, 0), sb = std::min(tb + my, H - 1);
            int sl = std::max(tl - mx, 0), sr = std::min(tr + mx, W - 1);
            tt = std::max(tt, 0);
            tb = std::min(tb, H - 1);
            tl = std::max(tl, 0);
            tr = std::min(tr, W - 1);
            const int tw = tr - tl + 1, th = tb - tt + 1, sw = sr - sl + 1, sh = sb - st + 1;
            // An empty window makes upstream's correlation call fail before the peak kernels;
            // the vector keeps its zero initialisation.
            if (tw < 1 || th < 1 || sw < tw || sh < th) continue;
            const float* T = images + (size_t)jb.tframe * frame_px + (size_t)tt * W + tl;
            const float* S = images + (size_t)jb.frame * frame_px + (size_t)st * W + sl;
            const int cw = sw - tw + 1, ch = sh - th + 1;
            corr.assign((size_t)cw * ch, 0.f);
            corr_valid(T, tw, th, W, S, sw, sh, W, corr.data());
            const Vec4 v = match_point(corr.data(), cw, ch, tl - sl, tt - st, p);
            float* o = maps + 4 * ((size_t)jb.frame * gx * gy + jb.cell);
            o[0] = v.x;
            o[1] = v.y;
            o[2] = v.z;
            o[3] = v.w;
        }
    };
    int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = (int)std::min<size_t>((size_t)nt, std::max<size_t>(jobs.size(), 1));
    std::vector<std::thread> pool;
    const size_t per = (jobs.size() + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const size_t lo = std::min(jobs.size(), t * per), hi = std::min(jobs.size(), lo + per);
        pool.emplace_back(work, lo, hi);
    }
    for (auto& th : pool) th.join();
    return 0;
}

}  // extern "C"
