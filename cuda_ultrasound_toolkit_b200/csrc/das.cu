// 3-D delay-and-sum with interpolation and coherence weighting.
//
// Restates the live upstream kernels (cuda_toolkit/src/beamformer/):
//   hercules_beamform_new  kernels/templated_beamformer.cuh:102-216
//   forces_beamform_new    kernels/templated_beamformer.cuh:219-324
//   helpers                beamformer_utils.cuh:48-154, 207-213
// with the constants of Beamformer::_params_to_constants (beamformer.cu:17-98) and the
// dispatch rules of Beamformer::beamform (beamformer.cu:139-197, 223-413).
//
// Design. A CTA of four warps owns a tile of voxels: 8 x 8 x 16 (x, y, z) by default for
// HERCULES, 4 x 8 x 32 for narrow volumes or on request, 32 x 1 x 32 for FORCES. The lanes of a
// warp are 4 x 8 (x, y) neighbours and each thread holds 8 consecutive depths, so the lanes'
// delays differ by a sample or two and their shared-memory reads fall in distinct banks. The CTA
// walks the analytic-signal rows (t, c) in stages of 8 channels. The window of samples the tile
// can address in each row follows from a Lipschitz bound on the path lengths; its metadata is
// computed in FP64 for 8 stages at a time by all threads, and lanes 0..7 of warp 0 then copy each
// row's window with one TMA bulk copy (cp.async.bulk) into one of three stage buffers completed
// through an mbarrier, keeping two stages of copies in flight. Once a stage has landed, all
// threads turn its windows into interpolation coefficients (cubic: four complex polynomial
// coefficients per interval; linear: value and slope) in shared memory, and every voxel then
// costs two 16-byte loads and a Horner evaluation per row, run on packed FP32x2 instructions for
// voxel pairs. Where the windows are short enough, the coefficients are double-buffered, so a
// stage needs one block barrier instead of two.
//
// Delays are formed relative to an FP64 origin at the tile centre: per row the FP64
// distance d0 from the tile centre to the element gives the absolute sample index of the
// centre; per voxel (offset delta from the centre, exact in FP32) the FP32 correction
// d - d0 = (d^2 - d0^2) / (d + d0) with d^2 - d0^2 = -2 (e - centre).delta + |delta|^2 keeps
// the index error near 1e-5 samples, instead of ~1e-4 for a direct FP32 sqrt of the
// ~5 cm path length.
//
// Choices where upstream is silent or self-contradictory (documented for users):
//   * interpolate == false -> linear, true -> cubic Catmull-Rom (upstream always cubic);
//   * HERCULES multiplies by the coherence factor when coherency_weighting > 0 (upstream
//     computes it but does not apply it); FORCES always applies it, as upstream;
//   * a single output point along x or z gets step 0 (upstream divides by zero);
//   * FORCES does not depend on y (upstream recomputes every y): one y-slice is computed
//     and written to every y.
#include <algorithm>
#include <cmath>

#include <cuda_bf16.h>

#include "common.cuh"
#include "encoding.h"
#include "stages.h"

namespace cutb {
namespace {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kVpt = 8;           // voxels per thread (along z)
constexpr int kRows = 8;          // rows (channels) per stage
constexpr int kStages = 3;        // raw stage buffers in flight
constexpr int kWinMax = 136;      // samples per staged window
constexpr int kWinShort = 88;     // ... for the double-buffered short-window form
constexpr int kBatch = 8;         // stages whose window metadata is computed together
constexpr int kSlots = 2 * kBatch;  // metadata ring: a batch never overwrites a stage still being issued
constexpr float kPi = 3.141592654f;  // value of CUDART_PI_F used upstream
constexpr long long kWaitLimitCycles = 400000000ll;  // ~0.2 s at 2 GHz

// Template code of tilted plane waves in a y-z plane: the plane-wave delay depends on y, so the
// tile spans y as for HERCULES. RCA_TPW itself stands for the x-z plane form (y-invariant).
constexpr int kTpwYz = 100 + RCA_TPW;

// Geometry of each sequence in the staged engine.
template <int SEQ>
struct Seq {
    static constexpr bool kTpw = SEQ == RCA_TPW || SEQ == kTpwYz;  // tilted plane waves, IQ rotation
    static constexpr bool kUf = SEQ == UFORCES;                    // sparse transmit elements after a flash
    static constexpr bool k3d = SEQ == HERCULES || SEQ == kTpwYz;  // voxels of a tile differ in y
};

// ---- PTX helpers: mbarrier + bulk copy (TMA) ----------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false if the phase did not complete within `limit` cycles.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long long limit)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - start > limit) return false;
    return true;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// f-number Hann window, beamformer_utils.cuh:142-154.
__device__ __forceinline__ float hann_apo(float lateral, float depth, float fnum)
{
    const float a = fminf(fnum * (lateral / depth) / 2.f, 0.5f);
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

__device__ __forceinline__ float2 to_f2(float2 v) { return v; }
__device__ __forceinline__ float2 to_f2(__nv_bfloat162 v) { return __bfloat1622float2(v); }

// Catmull-Rom (tangent 0.5*(p[i+1] - p[i-1])) at t in [0, 1) between p0 and p1,
// beamformer_utils.cuh:99-125; linear, :127-140.
__device__ __forceinline__ float2 catmull_rom(float2 pm1, float2 p0, float2 p1, float2 p2, float t)
{
    const float t2 = t * t;
    const float h00 = fmaf(fmaf(2.f, t, -3.f), t2, 1.f);
    const float h10 = fmaf(t - 2.f, t2, t);
    const float h01 = fmaf(-2.f, t, 3.f) * t2;
    const float h11 = (t - 1.f) * t2;
    const float m0x = 0.5f * (p1.x - pm1.x), m0y = 0.5f * (p1.y - pm1.y);
    const float m1x = 0.5f * (p2.x - p0.x), m1y = 0.5f * (p2.y - p0.y);
    return make_float2(fmaf(h00, p0.x, fmaf(h01, p1.x, fmaf(h10, m0x, h11 * m1x))),
                       fmaf(h00, p0.y, fmaf(h01, p1.y, fmaf(h10, m0y, h11 * m1y))));
}

// Guarded read of a global row: row[k] exists for k_min <= k < n; other taps read as zero.
template <bool CUBIC, class IQ>
__device__ __forceinline__ float2 interp_global(const IQ* row, float idx, int k_min, int n)
{
    const int i = __float2int_rd(idx);
    const float t = idx - (float)i;
    auto tap = [&](int k) -> float2 { return k >= k_min && k < n ? to_f2(__ldg(row + k)) : make_float2(0.f, 0.f); };
    if constexpr (CUBIC) return catmull_rom(tap(i - 1), tap(i), tap(i + 1), tap(i + 2), t);
    const float2 p0 = tap(i), p1 = tap(i + 1);
    return make_float2(fmaf(p1.x - p0.x, t, p0.x), fmaf(p1.y - p0.y, t, p0.y));
}

// Per-row stage metadata written by the issuing lane.
struct RowMeta {
    float base;     // sample index at the tile centre, relative to `lo`
    float d0;       // FP32 copy of the centre-to-receive-point distance
    float d0sq;     // its square
    float two_d0;   // 2 * d0
    float ex2;      // -2 * (receive point x - centre x)
    float rx_apo;   // sine receive apodization when it is uniform over the row, else 1
    float loclamp;  // clamp range of the window-relative index: the row's [1, S-2] ...
    float hiclamp;  // ... intersected with the staged window
    float xc;       // receive element x
    float rot_c, rot_s;  // TPW: exp(i 2 pi fc/fs lo), the IQ rotation at window index 0
    int lo;         // row sample of window index 0
    int len;        // staged samples; 0: the row is read from global memory
    int unclamped;  // staged, and no voxel of the tile can reach the clamp: the clamp is skipped
};

// Per-stage metadata (transmit t, sub-signal g, rows c0..c0+nq-1).
struct StageMeta {
    float ey2;      // HERCULES: -2 * (receive row y - centre y); FORCES: -2 * (tx element x - centre x)
    float tx_d0;    // FORCES: centre-to-transmit-element distance
    float tx_d0sq;
    float two_tx_d0;
    float sign;     // READI sign of this sub-signal
    float uni_apo;  // apodization factor uniform over the stage (sine types)
    float yj, et;   // receive row y (HERCULES) / transmit element x (FORCES, UFORCES)
    float s_t, c_t; // TPW: sine and cosine of the plane-wave angle
    int t, g, c0, nq;  // t: the analytic-signal transmit row (UFORCES: the used transmit + 1)
};

// Shared memory: NS raw windows per row (TMA destination) and, for NC > 0, one buffer of
// interpolation coefficients per row. Cubic (NC = 2): A[i] = (a, b), B[i] = (c, d) with
// value(t) = a + t (b + t (c + t d)) on [i, i + 1] (complex a..d), split so each is one 16-byte
// load. Linear (NC = 1): A[i] = (p[i], p[i + 1] - p[i]).
//
// DB: two coefficient buffers (stage j builds into buffer j % 2), so that a stage needs one
// block barrier instead of two; it fits three CTAs per SM only with shorter windows (kWinShort).
template <class IQ, int NC, bool DB = false>
struct alignas(128) Smem {
    static constexpr int kWin = DB ? kWinShort : kWinMax;
    static constexpr int kCB = DB ? 2 : 1;
    IQ raw[kStages][kRows][kWin];
    float4 coefA[NC >= 1 ? kCB : 1][NC >= 1 ? kRows : 1][NC >= 1 ? kWin : 1];
    float4 coefB[NC == 2 ? kCB : 1][NC == 2 ? kRows : 1][NC == 2 ? kWin : 1];
    RowMeta rowc[NC >= 1 ? kCB : 1][NC >= 1 ? kRows : 1];  // metadata of the rows whose coefficients are built
    // The fields of rowc that the packed row pass reads for every row, (ex2, d0sq, d0, base): one
    // 16-byte warp-uniform load (2 shared-memory wavefronts) instead of five 4-byte loads of the
    // 56-byte RowMeta (5 wavefronts), about 5 % of the kernel's wavefronts on the benchmark frame.
    float4 rowk[NC >= 1 ? kCB : 1][NC >= 1 ? kRows : 1];
    RowMeta row[kStages][kRows];
    StageMeta stage[kStages];
    RowMeta next_row[kSlots][kRows];    // precomputed metadata of upcoming stages (ring)
    StageMeta next_stage[kSlots];
    int next_bytes[kSlots][kRows];
    uint64_t full[kStages];
    // Abort flag per stage parity: set by a thread whose bounded wait for stage j gave up, before
    // stage j's barrier, and read by every thread after it. A thread one stage ahead writes the
    // other slot, so all threads leave the stage loop at the same stage.
    int abort[2];
    int tx_reach_bits;
    int part_last;  // stream-K: the pair counter's value before this part's arrival
};

// The double-buffered form runs three CTAs per SM: 228 KiB of shared memory per SM, 1 KiB of it
// reserved per CTA.
static_assert(3 * (sizeof(Smem<float2, 2, true>) + 1024) <= 228 * 1024, "three double-buffered CTAs per SM");

// Coefficient arrays staged per row: cubic always 2; linear 1 where the packed row pass runs
// (HERCULES without apodization), else 0 (the taps are read from the raw windows).
template <int SEQ, bool CUBIC, bool APO>
constexpr int coef_arrays() { return CUBIC ? 2 : (SEQ == HERCULES && !APO ? 1 : 0); }

struct Tile {
    double cx, cy, cz;  // tile centre (FP64)
    float radius;       // bound on |voxel - centre| over the tile
    float tx_reach;     // bound on |transmit-path offset| over the tile, in samples
};

// Stage k = (transmit t, row chunk, sub-signal g), with g fastest.
struct StageId {
    int t, g, c0, nq;
};
// Receive channels per stage (cutb_options.das_rows_per_stage): at most kRows, the rows the
// stage buffers hold; a stage of fewer rows leaves the rest of its buffer unused.
__host__ __device__ __forceinline__ int stage_rows(const DasArgs& a)
{
    return a.rows_per_stage > 0 && a.rows_per_stage < kRows ? a.rows_per_stage : kRows;
}

__device__ __forceinline__ StageId stage_id(const DasArgs& a, int k, int nchunks)
{
    StageId s;
    s.g = k % a.G;
    const int chunk = (k / a.G) % nchunks;
    s.t = k / (a.G * nchunks);
    const int rows = stage_rows(a);
    s.c0 = chunk * rows;
    s.nq = min(rows, a.C - s.c0);
    return s;
}

// Stage-uniform geometry, computed by every thread from the stage index.
template <int SEQ>
__device__ __forceinline__ StageMeta stage_meta(const DasArgs& a, const StageId& id, const Tile& tile)
{
    constexpr bool HERC = SEQ == HERCULES;
    StageMeta s{};
    s.t = id.t;
    s.g = id.g;
    s.c0 = id.c0;
    s.nq = id.nq;
    bool negate = false;
    if (a.G > 1) {
        int bit = id.g;
        if (HERC && a.encoding == WALSH && (id.t & 1)) bit = a.G - 1 - id.g;
        negate = (a.readi_row >> bit) & 1ull;
    }
    s.sign = negate ? -1.f : 1.f;
    s.uni_apo = 1.f;
    if constexpr (Seq<SEQ>::kTpw) {
        // plane wave at angle foci[t][2] (radians): delay lat sin(a) + z cos(a), lat = y (y-z plane) or x
        double sn, cs;
        sincos((double)a.angles[id.t], &sn, &cs);
        s.s_t = (float)sn;
        s.c_t = (float)cs;
        return s;
    }
    if constexpr (Seq<SEQ>::kUf) {
        // transmit row 0 is the flash: used transmit t reads row t + 1, from element elems[t] -
        // elems[0] places after the first (the first used transmit is scaled by 1/sqrt(128))
        s.t = id.t + 1;
        const double fx = (double)(a.xmin_x + a.px * 0.5f);
        const double et = fx + (double)(a.elems[id.t] - a.elems[0]) * (double)a.px;
        const double txd0 = sqrt((tile.cx - et) * (tile.cx - et) + tile.cz * tile.cz);
        s.et = (float)et;
        s.tx_d0 = (float)txd0;
        s.tx_d0sq = (float)(txd0 * txd0);
        s.two_tx_d0 = (float)(2.0 * txd0);
        s.ey2 = (float)(-2.0 * (et - tile.cx));
        s.uni_apo = id.t == 0 ? 0.088388347648318f : 1.f;
        return s;
    }
    if (HERC) {
        const double j = a.G > 1 ? (a.encoding == WALSH ? (double)(id.t * a.G + id.g) : (double)(id.g * a.T + id.t))
                                 : (double)id.t;
        const double yj = (double)a.xmin_y + j * (double)a.py;
        s.yj = (float)yj;
        s.ey2 = (float)(-2.0 * (yj - tile.cy));
        if (a.use_apo && a.apo_type == RX_TO_SIN) s.uni_apo = sin_apo(s.yj, a.xmax_y, a.to_power);
    } else {
        const double et = (double)a.xmin_x + (double)(id.g * a.T + id.t) * (double)a.px;
        const double txd0 = sqrt((tile.cx - et) * (tile.cx - et) + tile.cz * tile.cz);
        s.et = (float)et;
        s.tx_d0 = (float)txd0;
        s.tx_d0sq = (float)(txd0 * txd0);
        s.two_tx_d0 = (float)(2.0 * txd0);
        s.ey2 = (float)(-2.0 * (et - tile.cx));
        if (a.use_apo && (a.apo_type == TX_TO_SIN || a.apo_type == BOTH_TO_SIN))
            s.uni_apo = sin_apo(s.et, a.xmax_x, a.to_power);
    }
    return s;
}

// Window bounds and metadata of row q of stage `id` into batch slot `slot` (one thread per
// row; all threads of the CTA share the work of a batch of stages).
template <int SEQ, class IQ, int NC, bool DB>
__device__ void compute_row(Smem<IQ, NC, DB>& sm, int slot, const StageId& id, int q, const DasArgs& a,
                            const Tile& tile)
{
    constexpr bool HERC = SEQ == HERCULES;
    constexpr int SA = 16 / sizeof(IQ);  // samples per 16-byte unit
    if (q == 0) sm.next_stage[slot] = stage_meta<SEQ>(a, id, tile);
    int bytes = 0;
    RowMeta m{};
    if (q < id.nq) {
        const int c = id.c0 + q;
        // receive element: xdc_mins.x + c pitch (HERCULES, FORCES), + pitch / 2 (TPW, UFORCES)
        const double xc = (double)a.xmin_x + (Seq<SEQ>::kTpw || Seq<SEQ>::kUf ? 0.5 * (double)a.px : 0.0) +
                          (double)c * (double)a.px;
        double d0, base;
        if constexpr (Seq<SEQ>::kTpw) {
            const double ex = xc - tile.cx;
            d0 = sqrt(ex * ex + tile.cz * tile.cz);  // the receive path lies in the x-z plane
            double sn, cs;
            sincos((double)a.angles[id.t], &sn, &cs);
            const double lat = SEQ == kTpwYz ? tile.cy : tile.cx;
            base = (d0 + lat * sn + tile.cz * cs) * (double)a.spm + (double)a.delay;
            m.ex2 = (float)(-2.0 * ex);
        } else if constexpr (Seq<SEQ>::kUf) {
            const double fx = (double)(a.xmin_x + a.px * 0.5f);
            const double et = fx + (double)(a.elems[id.t] - a.elems[0]) * (double)a.px;
            const double txd0 = sqrt((tile.cx - et) * (tile.cx - et) + tile.cz * tile.cz);
            const double ex = xc - tile.cx;
            d0 = sqrt(ex * ex + tile.cz * tile.cz);
            base = (txd0 + d0) * (double)a.spm + (double)a.delay;
            m.ex2 = (float)(-2.0 * ex);
        } else if (HERC) {
            const double j = a.G > 1 ? (a.encoding == WALSH ? (double)(id.t * a.G + id.g) : (double)(id.g * a.T + id.t))
                                     : (double)id.t;
            const double yj = (double)a.xmin_y + j * (double)a.py;
            const double ex = xc - tile.cx, ey = yj - tile.cy, ez = -tile.cz;
            d0 = sqrt(ex * ex + ey * ey + ez * ez);
            // idx = (tx + d + fz) * spm + delay; tx(voxel) = tx(centre) + per-voxel offset.
            double txc = tile.cz;
            if (a.focus == 4) {
                const double dz = tile.cz - (double)a.fz;
                txc = copysign(sqrt(tile.cy * tile.cy + dz * dz), dz) + (double)a.fz;
            }
            base = (txc + d0 + (double)a.fz) * (double)a.spm + (double)a.delay;
            m.ex2 = (float)(-2.0 * ex);
        } else {
            const double et = (double)a.xmin_x + (double)(id.g * a.T + id.t) * (double)a.px;
            const double txd0 = sqrt((tile.cx - et) * (tile.cx - et) + tile.cz * tile.cz);
            const double ex = xc - tile.cx;
            d0 = sqrt(ex * ex + tile.cz * tile.cz);
            base = (txd0 + d0) * (double)a.spm + (double)a.delay;
            m.ex2 = (float)(-2.0 * ex);
        }
        // Every voxel lies within `radius` of the centre and a path length is 1-Lipschitz, so
        // the receive part moves the index by at most radius * spm and the transmit part by at
        // most tile.tx_reach samples.
        const double reach = (double)tile.radius * (double)a.spm + (double)tile.tx_reach + 1.0;
        const double smax = (double)a.S - 2.0;
        // the row clamp: [1, S - 2]; UFORCES [0, S - 2] (its tap below sample 0 reads zero)
        constexpr int kClampLo = Seq<SEQ>::kUf ? 0 : 1;
        const int i_lo = (int)floor(fmin(fmax(base - reach, (double)kClampLo), smax));
        const int i_hi = (int)floor(fmin(fmax(base + reach, (double)kClampLo), smax));
        int lo = max(0, i_lo - 2);
        const int hi = min(a.S, i_hi + 3);          // sample S is a zero tap
        lo -= lo % SA;                               // 16-byte aligned start
        const int len = hi - lo + 1;
        m.d0 = (float)d0;
        m.d0sq = (float)(d0 * d0);
        m.two_d0 = (float)(2.0 * d0);
        m.rx_apo = 1.f;
        if (a.use_apo && (a.apo_type == RX_TO_SIN || (!HERC && a.apo_type == BOTH_TO_SIN)))
            m.rx_apo = sin_apo((float)xc, a.xmax_x, a.to_power);
        m.lo = lo;
        m.xc = (float)xc;
        if constexpr (Seq<SEQ>::kTpw) {  // exp(i 2 pi fc/fs lo), the phase reduced exactly
            double sn, cs, ph = a.fc_fs * (double)lo;
            sincospi(2.0 * (ph - floor(ph)), &sn, &cs);
            m.rot_c = (float)cs;
            m.rot_s = (float)sn;
        }
        m.base = (float)(base - (double)lo);
        m.loclamp = (float)(kClampLo - lo);
        m.hiclamp = (float)(a.S - 2 - lo);
        m.len = 0;
        // UFORCES stages a row only when no index can come below 1, so the window never needs the
        // zero tap below sample 0; such rows read the global row with guarded taps instead.
        if (len + SA <= Smem<IQ, NC, DB>::kWin && (!Seq<SEQ>::kUf || base - reach >= 1.0)) {
            m.len = len;
            m.loclamp = fmaxf(m.loclamp, 1.f);
            m.hiclamp = fminf(m.hiclamp, (float)(len - 3));
            const int end = min(hi, a.S - 1);       // last real sample copied
            int count = end - lo + 1;
            count += (SA - count % SA) % SA;        // whole 16-byte units; stays inside the row
            bytes = count * (int)sizeof(IQ);
            // Every index lies in [base - reach, base + reach] (reach carries one sample of slack
            // over the FP32 rounding); inside [1, S - 3] neither the row clamp [1, S - 2] nor the
            // window bounds [1, len - 3] can bind, since lo <= floor(base - reach) - 2 and the
            // window ends at floor(base + reach) + 3 <= S.
            m.unclamped = (base - reach >= 1.0 && base + reach <= (double)a.S - 3.0) ? 1 : 0;
        }
    }
    sm.next_row[slot][q] = m;
    sm.next_bytes[slot][q] = bytes;
}

// Metadata of stages first .. first+kBatch-1 (all threads; a barrier must follow).
template <int SEQ, class IQ, int NC, bool DB>
__device__ __forceinline__ void compute_batch(Smem<IQ, NC, DB>& sm, int first, int nstages, int nchunks,
                                              const DasArgs& a, const Tile& tile)
{
    for (int i = threadIdx.x; i < kBatch * kRows; i += kThreads) {
        const int k = first + i / kRows;
        if (k < nstages) compute_row<SEQ>(sm, (k % kSlots), stage_id(a, k, nchunks), i % kRows, a, tile);
    }
}

// Issue stage k into buffer b from its precomputed metadata: lane q of one warp per row.
template <class IQ, int NC, bool DB>
__device__ __forceinline__ void issue_row(Smem<IQ, NC, DB>& sm, int b, int k, int q, const DasArgs& a,
                                          const IQ* __restrict__ iq)
{
    const int slot = k % kSlots;
    const StageMeta& st = sm.next_stage[slot];
    const RowMeta m = sm.next_row[slot][q];
    const unsigned bytes = (unsigned)sm.next_bytes[slot][q];
    if (q == 0) sm.stage[b] = st;
    sm.row[b][q] = m;
    // Test hook (cutb_debug_das_skip_stage): the stage is never issued, so its barrier phase never
    // completes and the bounded wait for it gives up.
    if (a.debug_skip && k == a.debug_skip - 1) return;
    if (bytes && m.lo + m.len - 1 == a.S) sm.raw[b][q][a.S - m.lo] = IQ{};  // zero tap past the row end
    // Order earlier generic-proxy accesses of this buffer before the async-proxy writes.
    fence_proxy_async();
    mbar_arrive_expect_tx(&sm.full[b], bytes);
    if (bytes) bulk_load(&sm.raw[b][q][0], iq + ((size_t)st.t * a.C + st.c0 + q) * a.S + m.lo, bytes, &sm.full[b]);
}

// Distance correction d - d0 from d^2 - d0^2 = delta: one approximate reciprocal square root
// and a Newton step on (d0 + e)^2 = d0^2 + delta, exact to FP32 rounding of the small terms.
__device__ __forceinline__ float path_offset(float delta, float d0, float d0sq, float two_d0)
{
    const float D = d0sq + delta;
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(D));
    const float e0 = fmaf(D, r, -d0);
    const float res = fmaf(e0, e0 + two_d0, -delta);
    return fmaf(-0.5f * r, res, e0);
}

// Interpolation coefficients of every staged interval of stage buffer b (all threads). The
// (row, interval) pairs are dealt out over the whole CTA: a staged row has at most `wint`
// intervals (i = 1 .. len - 3), and item e is interval 1 + e mod wint of row e / wint, so every
// thread builds about nq * wint / kThreads of them. A per-row loop over i left the threads past
// the window length idle (a 60-sample window keeps two of four warps busy) while the others
// built, and the idle warps then waited at the stage barrier.
//
// Threads first .. first + count - 1 share the items (all threads, or the ones that are not
// computing window metadata in this stage).
//
// rot_tab (TPW): the polynomial of interval i is multiplied by exp(i 2 pi fc/fs (lo + i)), the IQ
// rotation at its left end, from the row's exp(i 2 pi fc/fs lo) and rot_tab[i] = exp(i 2 pi fc/fs i);
// a voxel then only rotates by exp(i 2 pi fc/fs t) for its offset t in [0, 1).
__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

template <class IQ, int NC, bool DB>
__device__ __forceinline__ void build_coefficients(Smem<IQ, NC, DB>& sm, int b, int nq, int cb, int wint,
                                                   float rwint, int first, int count, const float2* rot_tab = nullptr)
{
    if (threadIdx.x < nq) {
        const RowMeta m = sm.row[b][threadIdx.x];
        sm.rowc[cb][threadIdx.x] = m;
        sm.rowk[cb][threadIdx.x] = make_float4(m.ex2, m.d0sq, m.d0, m.base);
    }
    const int n = nq * wint;
    if ((int)threadIdx.x < first) return;
#pragma unroll 1
    for (int e = (int)threadIdx.x - first; e < n; e += count) {
        // e / wint: (e + 1/2) / wint is at least 1 / (2 wint) from an integer, far above the
        // rounding of the product (e < 2^11).
        const int q = (int)(((float)e + 0.5f) * rwint);
        const int i = 1 + e - q * wint;
        if (i > sm.row[b][q].len - 3) continue;
        const IQ* p = &sm.raw[b][q][0];
        if constexpr (NC == 1) {
            // linear: value(t) = p0 + t (p1 - p0), the operations of the scalar staged pass
            const float2 p0 = to_f2(p[i]), p1 = to_f2(p[i + 1]);
            sm.coefA[cb][q][i] = make_float4(p0.x, p0.y, p1.x - p0.x, p1.y - p0.y);
        } else {
            const float2 pm1 = to_f2(p[i - 1]), p0 = to_f2(p[i]), p1 = to_f2(p[i + 1]), p2 = to_f2(p[i + 2]);
            float4 A, B;
            A.x = p0.x;
            A.y = p0.y;
            A.z = 0.5f * (p1.x - pm1.x);
            A.w = 0.5f * (p1.y - pm1.y);
            B.x = fmaf(-0.5f, p2.x, fmaf(2.f, p1.x, fmaf(-2.5f, p0.x, pm1.x)));
            B.y = fmaf(-0.5f, p2.y, fmaf(2.f, p1.y, fmaf(-2.5f, p0.y, pm1.y)));
            B.z = fmaf(0.5f, p2.x - pm1.x, 1.5f * (p0.x - p1.x));
            B.w = fmaf(0.5f, p2.y - pm1.y, 1.5f * (p0.y - p1.y));
            if (rot_tab) {
                const RowMeta& m = sm.row[b][q];
                const float2 r = cmulf(make_float2(m.rot_c, m.rot_s), rot_tab[i]);
                const float2 a0 = cmulf(make_float2(A.x, A.y), r), a1 = cmulf(make_float2(A.z, A.w), r);
                const float2 b0 = cmulf(make_float2(B.x, B.y), r), b1 = cmulf(make_float2(B.z, B.w), r);
                A = make_float4(a0.x, a0.y, a1.x, a1.y);
                B = make_float4(b0.x, b0.y, b1.x, b1.y);
            }
            sm.coefA[cb][q][i] = A;
            sm.coefB[cb][q][i] = B;
        }
    }
}

// Accumulates one row into the thread's voxels. STAGED: from shared memory (coefficients
// for cubic, raw taps for linear); otherwise from the global row with guarded taps.
template <int SEQ, bool CUBIC, bool CF, bool APO, bool STAGED, class IQ, int NCS, bool DB>
__device__ __forceinline__ void row_pass(const DasArgs& a, const Smem<IQ, NCS, DB>& sm, const RowMeta* rows, int b,
                                         int qi, const IQ* grow, const StageMeta& st, float dxe, const float (&sq)[kVpt],
                                         const float (&txs)[kVpt], const float (&vzv)[kVpt], float vx, float a2,
                                         float2 (&total)[kVpt], float (&inc)[kVpt], const float2* rot_tab = nullptr)
{
    using Q = Seq<SEQ>;
    constexpr bool HERC = SEQ == HERCULES;
    constexpr float kMagic = 8388608.f;  // 2^23: adding it with round-down leaves floor(x) in the mantissa
    const RowMeta& m = rows[qi];
    const float exdx = m.ex2 * dxe;
    const float base = m.base, d0 = m.d0, d0sq = m.d0sq, two_d0 = m.two_d0;
    const float loc = m.loclamp, hic = m.hiclamp;
    const float xc = m.xc;
    // TPW: 2 pi fc/fs, for the rotation within an interval
    const float phi = Q::kTpw ? (float)(6.283185307179586 * a.fc_fs) : 0.f;
#pragma unroll
    for (int v = 0; v < kVpt; ++v) {
        const float corr = path_offset(exdx + sq[v], d0, d0sq, two_d0);
        float w = st.sign;
        if (APO) {
            float apo;
            const float rx = xc - vx;
            if constexpr (Q::kTpw || Q::kUf) {
                // receive Hann window; the windowed value enters both sums (beamformer_kernels.cu:93-172,
                // 490-550). TPW skips windows below 0.1; UFORCES scales the first transmit by 1/sqrt(128).
                // vzv holds fn_rx / (2 depth) here: one multiply instead of a division per voxel and row
                const float c = __cosf(kPi * fminf(fabsf(rx) * vzv[v], 0.5f));
                apo = c * c;
                if (Q::kTpw && apo < 0.1f) continue;
                apo *= st.uni_apo;
            } else if (HERC) {
                apo = a.apo_type == RX_TO_SIN ? m.rx_apo * st.uni_apo
                                              : hann_apo(sqrtf(fmaf(rx, rx, a2)), vzv[v], a.fn_rx);
                if (!(apo > 0.1f)) continue;
            } else {
                const float ra = (a.apo_type == RX_TO_SIN || a.apo_type == BOTH_TO_SIN)
                                     ? m.rx_apo
                                     : hann_apo(fabsf(rx), vzv[v], a.fn_rx);
                if (!(ra > 0.f)) continue;
                const float ta = (a.apo_type == TX_TO_SIN || a.apo_type == BOTH_TO_SIN)
                                     ? st.uni_apo
                                     : hann_apo(fabsf(vx - st.et), vzv[v], a.fn_tx);
                apo = ra * ta;
            }
            w *= apo;
        }
        float idx = fmaf(corr, a.spm, base + txs[v]);
        idx = fminf(fmaxf(idx, loc), hic);
        float2 val;
        if constexpr (STAGED) {
            const float f = __fadd_rd(idx, kMagic);
            const int i = __float_as_int(f) - __float_as_int(kMagic);
            const float t = idx - (f - kMagic);
            if constexpr (CUBIC) {
                static_assert(!DB, "the scalar staged pass reads the single coefficient buffer");
                const float4 A = sm.coefA[0][qi][i], B = sm.coefB[0][qi][i];
                val.x = fmaf(fmaf(fmaf(B.z, t, B.x), t, A.z), t, A.x);
                val.y = fmaf(fmaf(fmaf(B.w, t, B.y), t, A.w), t, A.y);
            } else {
                const IQ* p = &sm.raw[b][qi][i];
                const float2 p0 = to_f2(p[0]), p1 = to_f2(p[1]);
                val = make_float2(fmaf(p1.x - p0.x, t, p0.x), fmaf(p1.y - p0.y, t, p0.y));
                // the linear taps are not pre-rotated: rotate to the interval's left end first
                if constexpr (Q::kTpw) val = cmulf(val, cmulf(make_float2(m.rot_c, m.rot_s), rot_tab[i]));
            }
            if constexpr (Q::kTpw) {  // the rest of the rotation, exp(i 2 pi fc/fs t), t in [0, 1)
                float sn, cs;
                __sincosf(phi * t, &sn, &cs);
                val = cmulf(val, make_float2(cs, sn));
            }
        } else {
            val = interp_global<CUBIC>(grow + m.lo, idx, -m.lo, a.S - m.lo);
            if constexpr (Q::kTpw) {  // exp(i 2 pi fc/fs (lo + idx)), the phase reduced in FP64
                double sn, cs, ph = a.fc_fs * ((double)m.lo + (double)idx);
                sincospi(2.0 * (ph - floor(ph)), &sn, &cs);
                val = cmulf(val, make_float2((float)cs, (float)sn));
            }
        }
        if constexpr (Q::kTpw || Q::kUf) {  // the windowed value enters the incoherent sum
            val.x *= w;
            val.y *= w;
            total[v].x += val.x;
            total[v].y += val.y;
            if (CF) inc[v] = fmaf(val.x, val.x, fmaf(val.y, val.y, inc[v]));
        } else {
            total[v].x = fmaf(w, val.x, total[v].x);
            total[v].y = fmaf(w, val.y, total[v].y);
            if (CF) inc[v] = fmaf(val.x, val.x, fmaf(val.y, val.y, inc[v]));
        }
    }
}

// ---- packed FP32x2 arithmetic (Blackwell add/sub/mul/fma.f32x2) ---------------------------
typedef unsigned long long f2x;
__device__ __forceinline__ f2x pk(float a, float b)
{
    f2x r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk(f2x v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c)
{
    f2x d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2x add2(f2x a, f2x b)
{
    f2x d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2x add2_rm(f2x a, f2x b)
{
    f2x d;
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2x sub2(f2x a, f2x b)
{
    f2x d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2x mul2(f2x a, f2x b)
{
    f2x d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ float rsqrt_approx(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// row_pass for HERCULES, cubic, staged rows, no apodization, on packed FP32x2 instructions:
// the delay arithmetic of voxel pairs (2p, 2p + 1) runs element-wise in one instruction each,
// and every voxel's complex Horner evaluation and accumulation in (re, im) pairs. Element by
// element the operations are those of row_pass: -(exdx + sq) negates the rounded sum exactly,
// so d0^2 - (-delta) = d0^2 + delta. Only the coherence energy is kept as (re^2, im^2) partial
// sums, added at the end.
template <bool CF, bool CLAMP, class IQ, int NC, bool DB>
__device__ __forceinline__ void row_pass_packed(const Smem<IQ, NC, DB>& sm, int cb, const RowMeta* rows, int qi, float dxe,
                                                float spm, f2x ww, const f2x (&sq2)[kVpt / 2],
                                                const f2x (&txs2)[kVpt / 2], f2x (&tot2)[kVpt], f2x (&inc2)[kVpt])
{
    constexpr float kMagic = 8388608.f;
    const float4 k = sm.rowk[cb][qi];  // (ex2, d0sq, d0, base) of rows[qi]
    const float exdx = k.x * dxe;
    const f2x nexdx2 = pk(-exdx, -exdx);
    const f2x d0sq2 = pk(k.y, k.y), nd02 = pk(-k.z, -k.z), mtwo2 = pk(-2.f, -2.f);
    const f2x base2 = pk(k.w, k.w), spm2 = pk(spm, spm), mhalf2 = pk(-0.5f, -0.5f);
    const f2x magic2 = pk(kMagic, kMagic);
    float loc = 0.f, hic = 0.f;
    if constexpr (CLAMP) loc = rows[qi].loclamp, hic = rows[qi].hiclamp;
    const float4* cA = sm.coefA[cb][qi];
    const float4* cB = sm.coefB[NC == 2 ? cb : 0][NC == 2 ? qi : 0];
#pragma unroll
    for (int p = 0; p < kVpt / 2; ++p) {
        const f2x nd = sub2(nexdx2, sq2[p]);  // -delta
        const f2x D = sub2(d0sq2, nd);        // d0^2 + delta
        float D0, D1;
        upk(D, D0, D1);
        const f2x r = pk(rsqrt_approx(D0), rsqrt_approx(D1));
        const f2x e0 = fma2(D, r, nd02);
        // e0 + 2 d0 as fma(-2, -d0, e0): the product is exact, so this is the sum with the row's two_d0
        const f2x res = fma2(e0, fma2(mtwo2, nd02, e0), nd);
        const f2x corr = fma2(mul2(mhalf2, r), res, e0);
        f2x ic = fma2(corr, spm2, add2(base2, txs2[p]));
        if constexpr (CLAMP) {
            float x0, x1;
            upk(ic, x0, x1);
            x0 = fminf(fmaxf(x0, loc), hic);
            x1 = fminf(fmaxf(x1, loc), hic);
            ic = pk(x0, x1);
        }
        const f2x f = add2_rm(ic, magic2);
        float f0, f1;
        upk(f, f0, f1);
        const int i0 = __float_as_int(f0) - __float_as_int(kMagic);
        const int i1 = __float_as_int(f1) - __float_as_int(kMagic);
        float t0, t1;
        upk(sub2(ic, sub2(f, magic2)), t0, t1);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = h ? i1 : i0;
            const f2x tt = h ? pk(t1, t1) : pk(t0, t0);
            f2x v;
            if constexpr (NC == 2) {
                const float4 A = cA[i], B = cB[i];
                v = fma2(fma2(fma2(pk(B.z, B.w), tt, pk(B.x, B.y)), tt, pk(A.z, A.w)), tt, pk(A.x, A.y));
            } else {
                const float4 A = cA[i];
                v = fma2(pk(A.z, A.w), tt, pk(A.x, A.y));
            }
            tot2[2 * p + h] = fma2(ww, v, tot2[2 * p + h]);
            if (CF) inc2[2 * p + h] = fma2(v, v, inc2[2 * p + h]);
        }
    }
}

// row_pass for TPW and UFORCES, cubic, staged rows, on packed FP32x2 instructions: the delay chain
// of voxel pairs as in row_pass_packed (the receive path of the scalar pass, element by element),
// the Horner evaluation and the accumulation in (re, im) pairs. The receive Hann window and the
// rotation exp(i 2 pi fc/fs t) stay scalar (special-function unit). A window below 0.1 (TPW)
// gives the voxel weight 0 instead of skipping it, which adds +-0 to its sums.
template <int SEQ, bool CF, bool CLAMP, class IQ, int NC, bool DB>
__device__ __forceinline__ void row_pass_packed_tu(const Smem<IQ, NC, DB>& sm, int cb, const RowMeta* rows, int qi,
                                                   float dxe, float spm, float vx, float phi, float sign,
                                                   float uni_apo, const f2x (&sq2)[kVpt / 2],
                                                   const f2x (&tsh2)[kVpt / 2], const float (&vzv)[kVpt],
                                                   f2x (&tot2)[kVpt], f2x (&inc2)[kVpt])
{
    static_assert(NC == 2, "cubic coefficients");
    constexpr float kMagic = 8388608.f;
    const float4 k = sm.rowk[cb][qi];  // (ex2, d0sq, d0, base) of rows[qi]
    const float exdx = k.x * dxe;
    const f2x nexdx2 = pk(-exdx, -exdx);
    const f2x d0sq2 = pk(k.y, k.y), nd02 = pk(-k.z, -k.z), td02 = pk(2.f * k.z, 2.f * k.z);
    const f2x base2 = pk(k.w, k.w), spm2 = pk(spm, spm), mhalf2 = pk(-0.5f, -0.5f);
    const f2x magic2 = pk(kMagic, kMagic);
    float loc = 0.f, hic = 0.f;
    if constexpr (CLAMP) loc = rows[qi].loclamp, hic = rows[qi].hiclamp;
    const float rxa = fabsf(rows[qi].xc - vx);
    const float4* cA = sm.coefA[cb][qi];
    const float4* cB = sm.coefB[cb][qi];
#pragma unroll
    for (int p = 0; p < kVpt / 2; ++p) {
        const f2x nd = sub2(nexdx2, sq2[p]);  // -delta
        const f2x D = sub2(d0sq2, nd);        // d0^2 + delta
        float D0, D1;
        upk(D, D0, D1);
        const f2x r = pk(rsqrt_approx(D0), rsqrt_approx(D1));
        const f2x e0 = fma2(D, r, nd02);
        const f2x res = fma2(e0, add2(e0, td02), nd);
        const f2x corr = fma2(mul2(mhalf2, r), res, e0);
        f2x ic = fma2(corr, spm2, add2(base2, tsh2[p]));
        if constexpr (CLAMP) {
            float x0, x1;
            upk(ic, x0, x1);
            x0 = fminf(fmaxf(x0, loc), hic);
            x1 = fminf(fmaxf(x1, loc), hic);
            ic = pk(x0, x1);
        }
        const f2x f = add2_rm(ic, magic2);
        float f0, f1;
        upk(f, f0, f1);
        const int i0 = __float_as_int(f0) - __float_as_int(kMagic);
        const int i1 = __float_as_int(f1) - __float_as_int(kMagic);
        float t0, t1;
        upk(sub2(ic, sub2(f, magic2)), t0, t1);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int v = 2 * p + h;
            const int i = h ? i1 : i0;
            const float t = h ? t1 : t0;
            // receive Hann window (vzv = fn_rx / (2 depth)), as the scalar pass
            const float c = __cosf(kPi * fminf(rxa * vzv[v], 0.5f));
            float apo = c * c;
            if (Seq<SEQ>::kTpw && apo < 0.1f) apo = 0.f;
            const float w = sign * (apo * uni_apo);
            const float4 A = cA[i], B = cB[i];
            const f2x tt = pk(t, t);
            f2x val = fma2(fma2(fma2(pk(B.z, B.w), tt, pk(B.x, B.y)), tt, pk(A.z, A.w)), tt, pk(A.x, A.y));
            if constexpr (Seq<SEQ>::kTpw) {  // the rest of the rotation, exp(i 2 pi fc/fs t), t in [0, 1)
                float sn, cs, vr, vi;
                __sincosf(phi * t, &sn, &cs);
                upk(val, vr, vi);
                const float2 rot = cmulf(make_float2(vr, vi), make_float2(cs, sn));
                val = pk(rot.x, rot.y);
            }
            const f2x vw = mul2(val, pk(w, w));
            tot2[v] = add2(tot2[v], vw);
            if (CF) inc2[v] = fma2(vw, vw, inc2[v]);
        }
    }
}

// Thread layout. HERCULES: lanes are 4 (x) x 8 (y) neighbours, whose delays differ by less
// than a sample or two, so their shared-memory reads fall in distinct banks or broadcast;
// warps and the kVpt registers of a thread run along z. FORCES (no y): lanes along x.
template <int SEQ, bool SHORT>
struct Layout {
    // HERCULES: lanes cover 4 (x) x 8 (y) voxels, each thread kVpt consecutive depths; the
    // four warps stack along z (4 x 8 x 32), or, for SHORT tiles, two along x and two along z
    // (8 x 8 x 16) -- the short tile halves the depth span, and with it the staged window,
    // when the z step is coarse. FORCES: lanes along x (32 x 1 x 32).
    static constexpr bool kShort = Seq<SEQ>::k3d && SHORT;
    static constexpr int TX = Seq<SEQ>::k3d ? (kShort ? 8 : 4) : 32;
    static constexpr int TY = Seq<SEQ>::k3d ? 8 : 1;
    static constexpr int TZ = (kShort ? 2 : kWarps) * kVpt;
};

// Parts of a tile under the stream-K decomposition (das_stream_kernel): the whole stage range, or
// the first or the last part of a tile whose stages two consecutive CTAs share.
// kPartSplit: part `pair` of `nparts` equal stage slices of tile `tile_id` (das_split_kernel).
constexpr int kPartFull = 0, kPartHead = 1, kPartTail = 2, kPartSplit = 3;
constexpr int kTileVoxels = kThreads * kVpt;
static_assert(kTileVoxels == (int)kStreamTileVoxels, "stream-K scratch holds one record per voxel of a tile");

// Stages of one tile: transmits x channel groups x READI sub-signals. UFORCES sums T - 1 transmits
// (row 0 is the flash; used transmit t reads row t + 1).
__host__ __device__ __forceinline__ int tile_stages(const DasArgs& a)
{
    return (a.seq == UFORCES ? a.T - 1 : a.T) * div_up(a.C, stage_rows(a)) * a.G;
}

// One tile (bx, by, bz) of the volume, stages k_lo .. k_hi - 1. Called by the grid
// kernel (a in parameter space) and by the persistent batch kernel (a in its parameter table).
template <int SEQ, bool CUBIC, bool CF, bool APO, class IQ, bool SHORT, bool DB = false>
__device__ __forceinline__ void das_tile(const IQ* __restrict__ iq, float2* __restrict__ vol, const DasArgs& a,
                                         Smem<IQ, coef_arrays<SEQ, CUBIC, APO>(), DB>& sm, int bx, int by, int bz,
                                         int k_lo, int k_hi, int part = kPartFull, int pair = 0, int nparts = 1,
                                         int tile_id = 0)
{
    constexpr int NC = coef_arrays<SEQ, CUBIC, APO>();
    static_assert(!DB || NC > 0, "two coefficient buffers need coefficients");
    using Q = Seq<SEQ>;
    constexpr bool HERC = SEQ == HERCULES;
    constexpr bool Y3 = Q::k3d;  // the tile spans y
    static_assert(!(Q::kTpw || Q::kUf) || (APO && CF), "TPW and UFORCES always window and weight");
    using L = Layout<SEQ, SHORT>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    // ---- tile, voxels, offsets from the tile centre -----------------------------------------
    const int tx0 = bx * L::TX, ty0 = by * L::TY, tz0 = bz * L::TZ;
    const float ix_c = tx0 + 0.5f * (L::TX - 1), iy_c = ty0 + 0.5f * (L::TY - 1), iz_c = tz0 + 0.5f * (L::TZ - 1);
    Tile tile;
    tile.cx = (double)a.vmin_x + (double)ix_c * (double)a.res_x;
    tile.cy = Y3 ? (double)a.vmin_y + (double)iy_c * (double)a.res_y : 0.0;
    tile.cz = (double)a.vmin_z + (double)iz_c * (double)a.res_z;
    {
        const double hx = 0.5 * (L::TX - 1) * fabs((double)a.res_x);
        const double hy = Y3 ? 0.5 * (L::TY - 1) * fabs((double)a.res_y) : 0.0;
        const double hz = 0.5 * (L::TZ - 1) * fabs((double)a.res_z);
        tile.radius = (float)(sqrt(hx * hx + hy * hy + hz * hz) * (1.0 + 1e-6) + 1e-9);
    }
    const int x_idx = tx0 + (Y3 ? (L::kShort ? 4 * (warp & 1) : 0) + (lane & 3) : lane);
    const int y_idx = Y3 ? ty0 + (lane >> 2) : 0;
    const int z_first = tz0 + (L::kShort ? (warp >> 1) : warp) * kVpt;
    // Offsets in voxel units are exact in FP32; scaled by the step they carry one rounding.
    const float dxe = ((float)x_idx - ix_c) * a.res_x;
    const float dye = Y3 ? ((float)y_idx - iy_c) * a.res_y : 0.f;
    const float vx = fmaf((float)x_idx, a.res_x, a.vmin_x);
    const float vy = fmaf((float)y_idx, a.res_y, a.vmin_y);
    float dz[kVpt], vzv[kVpt], txs[kVpt];
#pragma unroll
    for (int v = 0; v < kVpt; ++v) {
        dz[v] = ((float)(z_first + v) - iz_c) * a.res_z;
        vzv[v] = fmaf((float)(z_first + v), a.res_z, a.vmin_z);
        // TPW / UFORCES: only the receive Hann window reads the depth, as fn_rx / (2 depth)
        if constexpr (Seq<SEQ>::kTpw || Seq<SEQ>::kUf) vzv[v] = a.fn_rx * 0.5f / vzv[v];
        txs[v] = 0.f;
        if (HERC) {
            // Transmit path of this voxel relative to the centre's (FP64), in samples.
            double tx_rel = (double)dz[v];
            if (a.focus == 4) {
                const double vyd = tile.cy + (double)dye, dzf = tile.cz + (double)dz[v] - (double)a.fz;
                const double dzc = tile.cz - (double)a.fz;
                tx_rel = copysign(sqrt(vyd * vyd + dzf * dzf), dzf) - copysign(sqrt(tile.cy * tile.cy + dzc * dzc), dzc);
            }
            txs[v] = (float)(tx_rel * (double)a.spm);
        }
    }
    // Largest transmit offset over the tile (a focused transmit path jumps across the focal
    // depth, so it is measured rather than bounded). FORCES: the transmit path is 1-Lipschitz.
    if (threadIdx.x == 0) {
        sm.tx_reach_bits = 0;
        sm.abort[0] = sm.abort[1] = 0;
        for (int b = 0; b < kStages; ++b) mbar_init(&sm.full[b], kRows);
        fence_mbar_init();
    }
    __syncthreads();
    if (HERC) {
        float mx = 0.f;
#pragma unroll
        for (int v = 0; v < kVpt; ++v) mx = fmaxf(mx, fabsf(txs[v]));
        atomicMax(&sm.tx_reach_bits, __float_as_int(mx * 1.0001f + 1e-3f));
    }
    __syncthreads();
    tile.tx_reach = HERC ? __int_as_float(sm.tx_reach_bits) : tile.radius * a.spm;

    // Intervals per staged row, at most: compute_row's window spans i_lo - 2 - (SA - 1) ..
    // i_hi + 3 with i_hi - i_lo <= floor(2 reach) + 1 (reach is uniform over the tile), so
    // len - 3 <= floor(2 reach) + 3 + SA; a staged row also has len <= kWin - SA.
    constexpr int SA = 16 / sizeof(IQ);
    const int wint = min((int)floor(2.0 * ((double)tile.radius * (double)a.spm + (double)tile.tx_reach + 1.0)) + 3 + SA,
                         Smem<IQ, NC, DB>::kWin - 3);
    const float rwint = __frcp_rn((float)wint);

    // |delta|^2 and the z part of -2 (e - centre).delta, per voxel (only HERCULES receive paths
    // have a y component).
    const float two_cz = (float)(2.0 * tile.cz);
    const float dyr = HERC ? dye : 0.f;
    float qz[kVpt];
#pragma unroll
    for (int v = 0; v < kVpt; ++v) qz[v] = fmaf(two_cz, dz[v], fmaf(dxe, dxe, fmaf(dyr, dyr, dz[v] * dz[v])));

    // TPW: exp(i 2 pi fc/fs i) for the window indices, formed in FP64 once per tile.
    const float2* rot_tab = nullptr;
    if constexpr (Q::kTpw) {
        __shared__ float2 tpw_rot[Smem<IQ, NC, DB>::kWin];
        for (int i = threadIdx.x; i < Smem<IQ, NC, DB>::kWin; i += kThreads) {
            double sn, cs, ph = a.fc_fs * (double)i;
            sincospi(2.0 * (ph - floor(ph)), &sn, &cs);
            tpw_rot[i] = make_float2((float)cs, (float)sn);
        }
        rot_tab = tpw_rot;  // first read after the barrier that follows the first metadata batch
    }

    // HERCULES without apodization accumulates on packed FP32x2 (row_pass_packed), from cubic or
    // linear coefficients.
    constexpr bool PACKED = HERC && !APO;
    static_assert(!PACKED || NC > 0, "the packed pass reads coefficients");
    // TPW and UFORCES with cubic interpolation accumulate staged rows on packed FP32x2 as well
    // (row_pass_packed_tu); rows read from global memory take the scalar pass.
    constexpr bool PACKED_TU = (Q::kTpw || Q::kUf) && CUBIC && !DB;
    constexpr bool ANY_PACKED = PACKED || PACKED_TU;
    float2 total[kVpt];
    float inc[kVpt];
    f2x tot2[ANY_PACKED ? kVpt : 1], inc2[ANY_PACKED ? kVpt : 1], txs2[PACKED ? kVpt / 2 : 1];
#pragma unroll
    for (int v = 0; v < kVpt; ++v) {
        total[v] = make_float2(0.f, 0.f);
        inc[v] = 0.f;
        if constexpr (ANY_PACKED) {
            tot2[v] = 0ull;
            inc2[v] = 0ull;
        }
        if constexpr (PACKED) {
            if (v % 2 == 0) txs2[v / 2] = pk(txs[v], txs[v + 1]);
        }
    }

    const int nchunks = div_up(a.C, stage_rows(a));
    const int k_begin = k_lo, nstages = k_hi;
    // Window metadata (FP64) is computed for kBatch stages at a time by all threads; a stage's
    // bulk copies are then issued by lanes 0..kRows-1 of warp 0, one row per lane.
    static_assert(kRows <= 32 && kStages <= kBatch, "issue layout");
    compute_batch<SEQ>(sm, k_begin, nstages, nchunks, a, tile);
    __syncthreads();
    if (warp == 0 && lane < kRows)
        for (int j = 0; j < kStages && k_begin + j < nstages; ++j) issue_row(sm, j, k_begin + j, lane, a, iq);

    const long long wait_limit = a.wait_limit > 0 ? a.wait_limit : kWaitLimitCycles;
    int j_abort = -1;  // local stage at which the loop gave up
    for (int k = k_begin; k < nstages; ++k) {
        const int j = k - k_begin;  // local stage number: buffer and barrier phase
        const int b = j % kStages;
        if (!mbar_wait_bounded(&sm.full[b], (unsigned)(j / kStages) & 1u, wait_limit)) {
            sm.abort[j & 1] = 1;
            atomicOr(a.status, 1);
        }
        const StageMeta st = sm.stage[b];
        const int next = k + kStages;  // stage that refills buffer b
        // Every kBatch stages the first kBatch * kRows threads compute the next batch of window
        // metadata, one row each, and the other threads build this stage's coefficients alone,
        // so that both halves of the CTA reach the stage barrier together.
        constexpr int kMeta = kBatch * kRows;
        static_assert(kMeta < kThreads, "metadata rows leave threads for the coefficients");
        const bool batch = next < nstages && (next - k_begin) % kBatch == 0;
        if (batch) compute_batch<SEQ>(sm, next, nstages, nchunks, a, tile);
        int all_staged = 1;
        // DB: stage j builds into coefficient buffer j % 2, last read by stage j - 2's rows, which
        // every warp finished before the barrier below in stage j - 1; so the end-of-stage
        // barrier is not needed. A warp can then be one stage ahead of another, and touches
        // only that stage's buffers: coefficients j + 1 (other parity), raw stage and mbarrier
        // (j + 1) % kStages, metadata ring slots of stages j + kStages + 1 onwards.
        const int cb = DB ? (j & 1) : 0;
        if constexpr (NC > 0) {
            if (batch) build_coefficients(sm, b, st.nq, cb, wint, rwint, kMeta, kThreads - kMeta, rot_tab);
            else build_coefficients(sm, b, st.nq, cb, wint, rwint, 0, kThreads, rot_tab);
            all_staged = __syncthreads_and(threadIdx.x >= st.nq || sm.row[b][threadIdx.x].len > 0);
            if (DB && sm.abort[j & 1]) {
                j_abort = j;
                break;
            }
            // The raw buffer is free once transformed: refill it while this stage computes.
            if (warp == 0 && lane < kRows && next < nstages && !sm.abort[j & 1]) issue_row(sm, b, next, lane, a, iq);
        }
        const RowMeta* rows = NC > 0 ? sm.rowc[cb] : sm.row[b];
        if (NC == 0)
            for (int q = 0; q < st.nq; ++q) all_staged &= rows[q].len > 0;
        // Per-stage, per-voxel part of d^2 - d0^2 (receive path) and the FORCES transmit offset.
        float sq[kVpt], tsh[kVpt];
        float a2 = 0.f;
        if (APO && HERC) a2 = (st.yj - vy) * (st.yj - vy);
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            if (HERC) {
                sq[v] = fmaf(st.ey2, dye, qz[v]);
                tsh[v] = txs[v];
            } else if (Q::kTpw) {  // plane wave: the lateral (y or x) and depth offsets, exact lines
                sq[v] = qz[v];
                tsh[v] = fmaf(SEQ == kTpwYz ? dye : dxe, st.s_t, dz[v] * st.c_t) * a.spm;
            } else {
                sq[v] = qz[v];
                tsh[v] = path_offset(fmaf(st.ey2, dxe, qz[v]), st.tx_d0, st.tx_d0sq, st.two_tx_d0) * a.spm;
            }
        }
        const IQ* grow0 = iq + ((size_t)st.t * a.C + st.c0) * a.S;
        if constexpr (PACKED) {
            f2x sq2[kVpt / 2];
#pragma unroll
            for (int p = 0; p < kVpt / 2; ++p) sq2[p] = pk(sq[2 * p], sq[2 * p + 1]);
            const f2x ww = pk(st.sign, st.sign);
            // Stages whose rows can never reach the clamp run a clamp-free row pass. The branch is
            // taken per stage, not per row, so the unrolled row loop stays one straight-line block
            // in which the rows' independent delay chains interleave (a per-row branch measured 9%
            // slower; the full unroll of an 8-row stage 3% faster than unrolling by 2).
            // every row of the stage unclamped: lane q reads row q's flag, one load per warp
            const unsigned need = (1u << st.nq) - 1u;
            const bool row_unclamped = lane < st.nq && rows[lane].unclamped != 0;
            const bool unclamped = all_staged && (__ballot_sync(0xffffffffu, row_unclamped) & need) == need;
            if (unclamped && st.nq == kRows) {
#pragma unroll
                for (int qi = 0; qi < kRows; ++qi)
                    row_pass_packed<CF, false>(sm, cb, rows, qi, dxe, a.spm, ww, sq2, txs2, tot2, inc2);
            } else if (unclamped) {
#pragma unroll 4
                for (int qi = 0; qi < st.nq; ++qi)
                    row_pass_packed<CF, false>(sm, cb, rows, qi, dxe, a.spm, ww, sq2, txs2, tot2, inc2);
            } else if (all_staged) {
#pragma unroll 4
                for (int qi = 0; qi < st.nq; ++qi)
                    row_pass_packed<CF, true>(sm, cb, rows, qi, dxe, a.spm, ww, sq2, txs2, tot2, inc2);
            } else {
                for (int qi = 0; qi < st.nq; ++qi) {
                    if (rows[qi].len > 0)
                        row_pass_packed<CF, true>(sm, cb, rows, qi, dxe, a.spm, ww, sq2, txs2, tot2, inc2);
                    else
                        row_pass<SEQ, CUBIC, CF, APO, false>(a, sm, rows, b, qi, grow0 + (size_t)qi * a.S, st, dxe, sq,
                                                             tsh, vzv, vx, a2, total, inc);
                }
            }
        } else if constexpr (PACKED_TU) {
            f2x sq2[kVpt / 2], tsh2[kVpt / 2];
#pragma unroll
            for (int p = 0; p < kVpt / 2; ++p) {
                sq2[p] = pk(sq[2 * p], sq[2 * p + 1]);
                tsh2[p] = pk(tsh[2 * p], tsh[2 * p + 1]);
            }
            const float phi = Q::kTpw ? (float)(6.283185307179586 * a.fc_fs) : 0.f;  // 2 pi fc/fs
            const unsigned need = (1u << st.nq) - 1u;
            const bool row_unclamped = lane < st.nq && rows[lane].unclamped != 0;
            const bool unclamped = all_staged && (__ballot_sync(0xffffffffu, row_unclamped) & need) == need;
            if (unclamped) {
#pragma unroll 2
                for (int qi = 0; qi < st.nq; ++qi)
                    row_pass_packed_tu<SEQ, CF, false>(sm, cb, rows, qi, dxe, a.spm, vx, phi, st.sign, st.uni_apo, sq2,
                                                       tsh2, vzv, tot2, inc2);
            } else if (all_staged) {
#pragma unroll 2
                for (int qi = 0; qi < st.nq; ++qi)
                    row_pass_packed_tu<SEQ, CF, true>(sm, cb, rows, qi, dxe, a.spm, vx, phi, st.sign, st.uni_apo, sq2,
                                                      tsh2, vzv, tot2, inc2);
            } else {
                for (int qi = 0; qi < st.nq; ++qi) {
                    if (rows[qi].len > 0)
                        row_pass_packed_tu<SEQ, CF, true>(sm, cb, rows, qi, dxe, a.spm, vx, phi, st.sign, st.uni_apo,
                                                          sq2, tsh2, vzv, tot2, inc2);
                    else
                        row_pass<SEQ, CUBIC, CF, APO, false>(a, sm, rows, b, qi, grow0 + (size_t)qi * a.S, st, dxe, sq,
                                                             tsh, vzv, vx, a2, total, inc, rot_tab);
                }
            }
        } else if (all_staged) {
#pragma unroll 2
            for (int qi = 0; qi < st.nq; ++qi)
                row_pass<SEQ, CUBIC, CF, APO, true>(a, sm, rows, b, qi, grow0, st, dxe, sq, tsh, vzv, vx, a2, total,
                                                    inc, rot_tab);
        } else {
            for (int qi = 0; qi < st.nq; ++qi) {
                if (rows[qi].len > 0)
                    row_pass<SEQ, CUBIC, CF, APO, true>(a, sm, rows, b, qi, grow0, st, dxe, sq, tsh, vzv, vx, a2, total,
                                                        inc, rot_tab);
                else
                    row_pass<SEQ, CUBIC, CF, APO, false>(a, sm, rows, b, qi, grow0 + (size_t)qi * a.S, st, dxe, sq, tsh,
                                                         vzv, vx, a2, total, inc, rot_tab);
            }
        }
        if constexpr (!DB) {
            __syncthreads();
            if (sm.abort[j & 1]) {
                j_abort = j;
                break;
            }
        }
        if (NC == 0 && warp == 0 && lane < kRows && next < nstages) issue_row(sm, b, next, lane, a, iq);
    }
    if (j_abort >= 0) {
        // Stages j_abort + 1 .. j_abort + kStages - 1 were issued before the loop gave up (the
        // refill of stage j_abort's buffer was not); let their copies land before the CTA's shared
        // memory is released. Stage j_abort itself is the one whose wait ran out.
        for (int m = j_abort + 1; m < j_abort + kStages && k_begin + m < nstages; ++m)
            mbar_wait_bounded(&sm.full[m % kStages], (unsigned)(m / kStages) & 1u, wait_limit);
        return;
    }

    if constexpr (ANY_PACKED) {
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            float tx, ty, ix, iy;
            upk(tot2[v], tx, ty);
            upk(inc2[v], ix, iy);
            total[v].x += tx;
            total[v].y += ty;
            inc[v] += ix + iy;
        }
    }
    if (part == kPartSplit) {
        // Split: nparts CTAs summed equal stage slices of this tile. Each writes its sums to its own
        // record and counts its arrival; the last to arrive adds all records in slice order (its own
        // read back too), so the result does not depend on the arrival order. Nothing waits.
        float4* rec = a.sk_partials + (size_t)tile_id * nparts * kTileVoxels;
#pragma unroll
        for (int v = 0; v < kVpt; ++v)
            rec[(size_t)pair * kTileVoxels + threadIdx.x * kVpt + v] = make_float4(total[v].x, total[v].y, inc[v], 0.f);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) sm.part_last = atomicAdd(a.sk_counters + tile_id, 1);
        __syncthreads();
        if (sm.part_last != nparts - 1) return;  // a later slice finishes the tile
        __threadfence();
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            total[v] = make_float2(0.f, 0.f);
            inc[v] = 0.f;
        }
        for (int p = 0; p < nparts; ++p) {
#pragma unroll
            for (int v = 0; v < kVpt; ++v) {
                const float4 o = __ldcg(rec + (size_t)p * kTileVoxels + threadIdx.x * kVpt + v);
                total[v].x += o.x;
                total[v].y += o.y;
                inc[v] += o.z;
            }
        }
        if (threadIdx.x == 0) a.sk_counters[tile_id] = 0;  // ready for the next launch
    } else if (part != kPartFull) {
        // Stream-K: two consecutive CTAs summed the two parts of this tile's stages. Each writes its
        // sums to its own slot of the pair's scratch, then counts its arrival; the second to arrive
        // adds the other part's sums and finishes the tile. Addition of the two parts commutes, so
        // the result does not depend on which part arrives last. Nothing waits for the other part.
        float4* mine = a.sk_partials + ((size_t)pair * 2 + (part == kPartTail ? 1 : 0)) * kTileVoxels;
        const float4* other = a.sk_partials + ((size_t)pair * 2 + (part == kPartTail ? 0 : 1)) * kTileVoxels;
#pragma unroll
        for (int v = 0; v < kVpt; ++v) mine[threadIdx.x * kVpt + v] = make_float4(total[v].x, total[v].y, inc[v], 0.f);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) sm.part_last = atomicAdd(a.sk_counters + pair, 1);
        __syncthreads();
        if (sm.part_last == 0) return;  // the other part finishes the tile
        __threadfence();
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            const float4 o = __ldcg(other + threadIdx.x * kVpt + v);
            total[v].x += o.x;
            total[v].y += o.y;
            inc[v] += o.z;
        }
        if (threadIdx.x == 0) a.sk_counters[pair] = 0;  // ready for the next launch
    }
    if (x_idx >= a.X || y_idx >= a.Y) return;
#pragma unroll
    for (int v = 0; v < kVpt; ++v) {
        const int z = z_first + v;
        if (z >= a.Z) continue;
        float2 out = total[v];
        if (CF) {
            float cf = powf((out.x * out.x + out.y * out.y) / inc[v], a.cf_power);
            if (isnan(cf)) cf = 0.f;
            out.x *= cf;
            out.y *= cf;
        }
        if (a.splits > 1) {  // partial sums over a slice of the stages (no coherence factor)
            float2* o = vol + ((size_t)(z - a.z_out0) * a.Y + y_idx) * a.X + x_idx;
            atomicAdd(&o->x, out.x);
            atomicAdd(&o->y, out.y);
        } else if (Y3) {
            vol[((size_t)(z - a.z_out0) * a.Y + y_idx) * a.X + x_idx] = out;
        } else {  // y-invariant: one value for every y
            for (int y = 0; y < a.Y; ++y) vol[((size_t)(z - a.z_out0) * a.Y + y) * a.X + x_idx] = out;
        }
    }
}

// Whole grid: blockIdx.xyz is the tile. Tile list: blockIdx.x indexes a.tiles and blockIdx.y
// is the slice of the stages (transmits x channel groups) this CTA sums.
template <int SEQ, bool CUBIC, bool CF, bool APO, class IQ, bool SHORT, bool DB>
__global__ void __launch_bounds__(kThreads, 3)
das_kernel(const IQ* __restrict__ iq, float2* __restrict__ vol, DasArgs a)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<Smem<IQ, coef_arrays<SEQ, CUBIC, APO>(), DB>*>(smem_raw);
    using L = Layout<SEQ, SHORT>;
    int bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z + a.z_tile0;
    const int nst = tile_stages(a);
    int k_lo = 0, k_hi = nst;
    if (a.tiles) {
        const int nx = div_up(a.X, L::TX), ny = div_up(a.Y, L::TY);
        const int id = a.tiles[blockIdx.x];
        bx = id % nx;
        by = (id / nx) % ny;
        bz = id / (nx * ny);
        if (a.splits > 1) {  // this CTA's slice blockIdx.y of a.splits
            k_lo = (int)((long long)nst * blockIdx.y / a.splits);
            k_hi = (int)((long long)nst * (blockIdx.y + 1) / a.splits);
        }
    }
    das_tile<SEQ, CUBIC, CF, APO, IQ, SHORT, DB>(iq, vol, a, sm, bx, by, bz, k_lo, k_hi);
}

// Stream-K form of the grid kernel for volumes of more than one wave of tiles whose count is not
// a whole number of waves (gridDim.x CTAs = SMs x resident CTAs, <= tiles). The first waves run as
// in the grid kernel, CTA c taking tiles c, c + G, ... whole, so that the CTAs of a wave work on
// neighbouring tiles in step and share their windows in L2. The last wave and the partial one after
// it (R tiles, G <= R < 2G) are split into G equal contiguous ranges of tiles x stages, so that no
// CTA idles at the end. A range spans at least one tile, so a tile has at most two parts; the first
// part of a tile that CTA c cuts lies in c and the last in c + 1 (pair c), and the second to finish
// adds both (the part protocol of das_tile, through a.sk_partials / a.sk_counters).
template <int SEQ, bool CUBIC, bool CF, bool APO, class IQ, bool SHORT, bool DB>
__global__ void __launch_bounds__(kThreads, 3)
das_stream_kernel(const IQ* __restrict__ iq, float2* __restrict__ vol, DasArgs a)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<Smem<IQ, coef_arrays<SEQ, CUBIC, APO>(), DB>*>(smem_raw);
    using L = Layout<SEQ, SHORT>;
    const int nx = div_up(a.X, L::TX), ny = Seq<SEQ>::k3d ? div_up(a.Y, L::TY) : 1;
    const long long nst = tile_stages(a);
    const long long ntiles = (long long)nx * ny * div_up(a.Z, L::TZ);
    const long long G = gridDim.x;
    const long long whole = (ntiles / G - 1) * G;  // tiles of the data-parallel waves
    const long long work = (ntiles - whole) * nst;
    const long long s1 = work * (blockIdx.x + 1) / G;
    long long dp = blockIdx.x, s = work * blockIdx.x / G;
    // One loop with one call of the (large, inlined) tile body for both phases: two call sites
    // doubled the code and measured ~40 % slower.
    for (;;) {
        long long tile;
        int k0 = 0, k1 = (int)nst, part = kPartFull, pair = 0;
        if (dp < whole) {
            tile = dp;
            dp += G;
        } else if (s < s1) {
            const long long t = s / nst;
            tile = whole + t;
            k0 = (int)(s - t * nst);
            k1 = (int)min(nst, s1 - t * nst);
            part = k0 > 0 ? kPartTail : (k1 < nst ? kPartHead : kPartFull);
            pair = part == kPartTail ? (int)blockIdx.x - 1 : (int)blockIdx.x;
            s = t * nst + k1;
        } else {
            break;
        }
        das_tile<SEQ, CUBIC, CF, APO, IQ, SHORT, DB>(iq, vol, a, sm, (int)(tile % nx), (int)((tile / nx) % ny),
                                                     (int)(tile / ((long long)nx * ny)), k0, k1, part, pair);
        __syncthreads();
        if (sm.abort[0] | sm.abort[1]) return;
        if (threadIdx.x == 0)
            for (int b = 0; b < kStages; ++b) mbar_inval(&sm.full[b]);
        __syncthreads();
    }
}

// Split form: CTA (blockIdx.x, blockIdx.y) sums stage slice blockIdx.y of gridDim.y of tile
// tile_base + blockIdx.x (id order: z-major, then y, then x), and the last slice to finish a tile
// adds all slices (the kPartSplit protocol of das_tile; records and counters indexed by blockIdx.x
// in a.sk_partials / a.sk_counters). With one slice it is the grid kernel over a range of tile ids.
// Used for volumes of fewer tiles than half a wave, and for the partial last wave of larger ones.
template <int SEQ, bool CUBIC, bool CF, bool APO, class IQ, bool SHORT, bool DB>
__global__ void __launch_bounds__(kThreads, 3)
das_split_kernel(const IQ* __restrict__ iq, float2* __restrict__ vol, DasArgs a, int tile_base)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<Smem<IQ, coef_arrays<SEQ, CUBIC, APO>(), DB>*>(smem_raw);
    using L = Layout<SEQ, SHORT>;
    const int nx = div_up(a.X, L::TX), ny = Seq<SEQ>::k3d ? div_up(a.Y, L::TY) : 1;
    const int tile = tile_base + (int)blockIdx.x, P = gridDim.y, p = blockIdx.y;
    const long long nst = tile_stages(a);
    das_tile<SEQ, CUBIC, CF, APO, IQ, SHORT, DB>(iq, vol, a, sm, tile % nx, (tile / nx) % ny, tile / (nx * ny),
                                                 (int)(nst * p / P), (int)(nst * (p + 1) / P),
                                                 P > 1 ? kPartSplit : kPartFull, p, P, (int)blockIdx.x);
}

// Persistent delay-and-sum over the tiles of many frames: CTAs take (frame, tile) work items,
// heaviest first, from a device counter until the list is exhausted. Frame arguments sit in the
// kernel's parameter table (uniform per CTA, read through the constant cache).
template <int SEQ, bool CUBIC, bool CF, bool APO, class IQ, bool SHORT>
__global__ void __launch_bounds__(kThreads, 3)
das_batch_kernel(const DasBatchParams P, const int2* __restrict__ items, int nitems, int* __restrict__ counter)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<Smem<IQ, coef_arrays<SEQ, CUBIC, APO>()>*>(smem_raw);
    using L = Layout<SEQ, SHORT>;
    __shared__ int item_s;
    for (;;) {
        if (threadIdx.x == 0) item_s = atomicAdd(counter, 1);
        __syncthreads();
        const int it = item_s;
        if (it >= nitems) break;
        const int2 w = items[it];
        const DasFrame& f = P.f[w.x];
        const int nx = div_up(f.a.X, L::TX), ny = div_up(f.a.Y, L::TY);
        das_tile<SEQ, CUBIC, CF, APO, IQ, SHORT>((const IQ*)f.iq, f.vol, f.a, sm, w.y % nx, (w.y / nx) % ny,
                                                 w.y / (nx * ny), 0, tile_stages(f.a));
        __syncthreads();
        if (sm.abort[0] | sm.abort[1]) break;
        if (threadIdx.x == 0)
            for (int b = 0; b < kStages; ++b) mbar_inval(&sm.full[b]);
        __syncthreads();
    }
}

// CTAs of `kern` that one wave holds on the current device (SMs x resident CTAs), cached per
// device in `cache` (0: not yet known).
template <class Kernel>
bool wave_size(Kernel kern, size_t smem, std::atomic<int> (&cache)[64], int* wave)
{
    int dev = 0;
    CUTB_CUDA_OK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && (*wave = cache[dev].load(std::memory_order_relaxed)) > 0) return true;
    int sms = 0, per_sm = 0;
    CUTB_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CUTB_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
    *wave = sms * per_sm;
    if (dev >= 0 && dev < 64) cache[dev].store(*wave, std::memory_order_relaxed);
    return true;
}

// Set by prepare_das: launch_das_k only sets the kernel attributes and caches the wave size.
thread_local bool g_prepare_only = false;

template <int SEQ, bool CUBIC, bool CF, bool APO, class IQ, bool SHORT, bool DB>
bool launch_das_k(const DasArgs& a, const void* iq, void* volume, cudaStream_t st)
{
    using L = Layout<SEQ, SHORT>;
    // FORCES does not depend on y: one y-slice of tiles, each written to every y.
    dim3 grid(div_up(a.X, L::TX), Seq<SEQ>::k3d ? div_up(a.Y, L::TY) : 1,
              a.z_tiles > 0 ? a.z_tiles : div_up(a.Z, L::TZ));  // a z-slab: tiles z_tile0 .. + z_tiles - 1
    if (a.tiles) grid = dim3(a.ntiles, a.splits > 1 ? a.splits : 1, 1);
    CUTB_REQUIRE(grid.y <= 65535 && grid.z <= 65535, CUTB_ERR_UNSUPPORTED, "Output grid too large.");
    auto kern = das_kernel<SEQ, CUBIC, CF, APO, IQ, SHORT, DB>;
    const size_t smem = sizeof(Smem<IQ, coef_arrays<SEQ, CUBIC, APO>(), DB>);
    if (!a.tiles && a.z_tiles == 0 && a.sk_partials && a.sk_counters && a.schedule != 2 && a.schedule != 1) {
        // Split every tile of a small volume (fewer tiles than half a wave), or the tiles of a
        // partial last wave of a large one, over P CTAs of at least kBatch stages each, so that the
        // GPU stays full. Not HERCULES, whose small frames the batched kernel runs whole.
        auto pkern = das_split_kernel<SEQ, CUBIC, CF, APO, IQ, SHORT, DB>;
        static std::atomic<uint64_t> sp_smem_set{0};
        static std::atomic<int> sp_wave[64];
        if (!set_smem_limit(pkern, smem, sp_smem_set)) return false;
        int wave = 0;
        if (!wave_size(pkern, smem, sp_wave, &wave)) return false;
        if (g_prepare_only) return true;
        const long long tiles = (long long)grid.x * grid.y * grid.z;
        // HERCULES keeps one CTA per tile: splitting its partial last wave measured no faster
        // (83.19 vs 83.15 ms on 4096 tiles over 444 CTAs).
        const long long tail = SEQ == HERCULES ? 0 : (tiles > wave ? tiles % wave : tiles);
        const long long P = tail > 0 ? std::min<long long>(std::min<long long>(wave / tail, tile_stages(a) / kBatch),
                                                           2LL * a.sk_capacity / tail)
                                     : 0;
        if (tail > 0 && 2 * tail <= wave && P >= 2 && tail <= a.sk_capacity) {
            const long long whole = tiles - tail;
            if (whole > 0) {
                pkern<<<dim3((unsigned)whole, 1), kThreads, smem, st>>>((const IQ*)iq, (float2*)volume, a, 0);
                CUTB_CUDA_OK(cudaGetLastError());
            }
            CUTB_CUDA_OK(cudaMemsetAsync(a.sk_counters, 0, sizeof(int) * (size_t)tail, st));
            pkern<<<dim3((unsigned)tail, (unsigned)P), kThreads, smem, st>>>((const IQ*)iq, (float2*)volume, a,
                                                                             (int)whole);
            CUTB_CUDA_OK(cudaGetLastError());
            return true;
        }
    }
    if (!a.tiles && a.z_tiles == 0 && a.sk_partials && a.sk_counters) {
        // More than one wave of tiles that is not a whole number of waves: the stream-K form
        // spreads the last, partly empty wave's work over every CTA.
        auto skern = das_stream_kernel<SEQ, CUBIC, CF, APO, IQ, SHORT, DB>;
        static std::atomic<uint64_t> sk_smem_set{0};
        static std::atomic<int> sk_wave[64];
        if (!set_smem_limit(skern, smem, sk_smem_set)) return false;
        int wave = 0;
        if (!wave_size(skern, smem, sk_wave, &wave)) return false;
        const long long tiles = (long long)grid.x * grid.y * grid.z;
        if (g_prepare_only) return true;
        if (a.schedule == 2 && wave > 1 && tiles > wave && wave - 1 <= a.sk_capacity) {
            CUTB_CUDA_OK(cudaMemsetAsync(a.sk_counters, 0, sizeof(int) * (size_t)wave, st));
            skern<<<wave, kThreads, smem, st>>>((const IQ*)iq, (float2*)volume, a);
            CUTB_CUDA_OK(cudaGetLastError());
            return true;
        }
    }
    static std::atomic<uint64_t> smem_set{0};
    if (!set_smem_limit(kern, smem, smem_set)) return false;
    if (g_prepare_only) return true;
    kern<<<grid, kThreads, smem, st>>>((const IQ*)iq, (float2*)volume, a);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

// True when the short tile's staged window (the bound of prefer_short_tile for its half
// extents) fits the double-buffered form's kWinShort-sample buffers. Rows whose window still
// does not fit are read from global memory, so this only selects the faster form.
bool short_windows_fit(const DasArgs& a)
{
    using L = Layout<HERCULES, true>;
    const double hx = 0.5 * (L::TX - 1) * std::fabs((double)a.res_x), hy = 0.5 * (L::TY - 1) * std::fabs((double)a.res_y);
    const double hz = 0.5 * (L::TZ - 1) * std::fabs((double)a.res_z);
    const double reach = std::sqrt(hx * hx + hy * hy + hz * hz) * (double)a.spm;
    return 4.0 * reach + 8.0 <= (double)(kWinShort - 8);
}

template <int SEQ, bool CUBIC, bool CF, bool APO, class IQ, bool SHORT>
bool launch_das_t(const DasArgs& a, const void* iq, void* volume, cudaStream_t st)
{
    // HERCULES, short tile, coefficients: one barrier per stage when the windows are short.
    if constexpr (SEQ == HERCULES && SHORT && coef_arrays<SEQ, CUBIC, APO>() > 0 && !APO)
        if (short_windows_fit(a)) return launch_das_k<SEQ, CUBIC, CF, APO, IQ, SHORT, true>(a, iq, volume, st);
    return launch_das_k<SEQ, CUBIC, CF, APO, IQ, SHORT, false>(a, iq, volume, st);
}

// True when the 8 x 8 x 16 HERCULES tile is used. It is the default for volumes at least 8
// voxels wide: its staged windows are about half as long, so building the coefficients of a
// stage costs less per voxel (measured on 128 x 128 x 256, 128 x 128 x 4096 rows: 90.8 ms vs
// 93.3 ms for 4 x 8 x 32; the tuner picks it for most frames of the batched stream). Narrower
// volumes keep the 4 x 8 x 32 tile, unless its staged window (twice the largest index move
// over the tile, receive and transmit path each 1-Lipschitz, plus the interpolation taps)
// would not fit the stage buffers.
bool prefer_short_tile(const DasArgs& a)
{
    if (a.X >= 8) return true;
    const double hx = 1.5 * std::fabs((double)a.res_x), hy = 3.5 * std::fabs((double)a.res_y);
    const double hz = 15.5 * std::fabs((double)a.res_z);
    const double reach = std::sqrt(hx * hx + hy * hy + hz * hz) * (double)a.spm;
    return 4.0 * reach + 8.0 > (double)(kWinMax - 8);
}

// TPW and UFORCES: always windowed, always weighted by the coherence factor.
template <int SEQ, class IQ, bool SHORT>
bool launch_das_seq(const DasArgs& a, const void* iq, void* volume, cudaStream_t st)
{
    if (a.cubic) return launch_das_k<SEQ, true, true, true, IQ, SHORT, false>(a, iq, volume, st);
    return launch_das_k<SEQ, false, true, true, IQ, SHORT, false>(a, iq, volume, st);
}

template <int SEQ, class IQ, bool SHORT>
bool launch_das_s(const DasArgs& a, const void* iq, void* volume, cudaStream_t st)
{
#define CUTB_DAS_CASE(CUBIC, CF, APO)                                                   \
    if ((bool)a.cubic == CUBIC && (bool)a.apply_cf == CF && (bool)a.use_apo == APO) \
        return launch_das_t<SEQ, CUBIC, CF, APO, IQ, SHORT>(a, iq, volume, st);
    CUTB_DAS_CASE(true, true, false)
    CUTB_DAS_CASE(true, false, false)
    CUTB_DAS_CASE(false, true, false)
    CUTB_DAS_CASE(false, false, false)
    CUTB_DAS_CASE(true, true, true)
    CUTB_DAS_CASE(true, false, true)
    CUTB_DAS_CASE(false, true, true)
    CUTB_DAS_CASE(false, false, true)
#undef CUTB_DAS_CASE
    return false;
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
    CUTB_REQUIRE(a.seq == HERCULES || a.seq == FORCES || a.seq == RCA_TPW || a.seq == UFORCES, CUTB_ERR_UNSUPPORTED,
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
    CUTB_REQUIRE(std::isfinite(a.res_x) && std::isfinite(a.res_z) && std::isfinite(a.vmin_x) &&
                     std::isfinite(a.vmin_y) && std::isfinite(a.vmin_z),
                 CUTB_ERR_INVALID_ARGUMENT, "Output grid coordinates must be finite.");
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

    a.fc_over_fs = bp.center_frequency / bp.sampling_frequency;
    a.fc_fs = (double)bp.center_frequency / (double)bp.sampling_frequency;
    if (a.seq == RCA_TPW || a.seq == UFORCES) {
        // beamformer.cu:161-189, 416-468: no READI; TPW needs a plane focus, UFORCES the
        // sparse-element table (and, for a defined transmit path, a focus in the x-z plane).
        a.G = 1;
        a.readi_row = 0;
        a.apply_cf = 1;
        a.use_apo = 1;
        CUTB_REQUIRE(a.T <= MAX_ACQ_COUNT, CUTB_ERR_UNSUPPORTED, "At most %d transmits for this sequence.",
                     MAX_ACQ_COUNT);
        if (a.seq == RCA_TPW) {
            CUTB_REQUIRE(a.focus == 1 || a.focus == 2, CUTB_ERR_UNSUPPORTED,
                         "TPW beamforming requires a plane focus.");
        } else {
            CUTB_REQUIRE(bp.sparse_elements[0] != -1, CUTB_ERR_INVALID_ARGUMENT,
                         "Beamformer: UFORCES requires sparse elements to be defined.");
            CUTB_REQUIRE(a.focus == 3, CUTB_ERR_UNSUPPORTED,
                         "UFORCES needs a focused transmit in the x-z plane (same row/column orientation).");
            CUTB_REQUIRE(a.T >= 2, CUTB_ERR_INVALID_ARGUMENT, "UFORCES needs a flash plus at least one transmit.");
        }
        return true;
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

// Sequences whose voxels differ in y within a tile: HERCULES, and tilted plane waves in a y-z plane.
static bool das_3d(const DasArgs& a) { return a.seq == HERCULES || (a.seq == RCA_TPW && a.focus == 2); }
static bool use_short_tile(const DasArgs& a)
{
    return das_3d(a) && (a.tile == 2 || (a.tile == 0 && prefer_short_tile(a)));
}

// True when the staged windows of a TPW / UFORCES tile fit the stage buffers: the receive and the
// transmit path each move the index by at most the tile radius times spm, and a window spans twice
// that plus the interpolation taps. On coarse grids (wide tiles) the rows would be read from global
// memory instead, where the one-thread-per-voxel kernel is faster.
static bool seq_windows_fit(const DasArgs& a)
{
    double hx, hy = 0.0, hz;
    if (das_3d(a)) {
        const bool sh = use_short_tile(a);
        hx = 0.5 * ((sh ? Layout<kTpwYz, true>::TX : Layout<kTpwYz, false>::TX) - 1) * std::fabs((double)a.res_x);
        hy = 0.5 * (Layout<kTpwYz, false>::TY - 1) * std::fabs((double)a.res_y);
        hz = 0.5 * ((sh ? Layout<kTpwYz, true>::TZ : Layout<kTpwYz, false>::TZ) - 1) * std::fabs((double)a.res_z);
    } else {
        hx = 0.5 * (Layout<UFORCES, false>::TX - 1) * std::fabs((double)a.res_x);
        hz = 0.5 * (Layout<UFORCES, false>::TZ - 1) * std::fabs((double)a.res_z);
    }
    const double reach = std::sqrt(hx * hx + hy * hy + hz * hz) * (double)a.spm;
    return 4.0 * reach + 8.0 <= (double)(kWinMax - 8);
}

// TPW and UFORCES on the one-thread-per-voxel kernel (das_direct.cu) instead of the staged engine:
// on request (tile 3), or by default when the staged windows would not fit.
static bool das_direct(const DasArgs& a)
{
    return (a.seq == RCA_TPW || a.seq == UFORCES) && (a.tile == 3 || (a.tile == 0 && !seq_windows_fit(a)));
}

bool das_staged(const DasArgs& a)
{
    return (a.seq == HERCULES || a.seq == FORCES || a.seq == RCA_TPW || a.seq == UFORCES) && !das_direct(a);
}

bool das_uses_short_tile(const DasArgs& a) { return use_short_tile(a); }

namespace {
// grid > 0: launch with that many persistent CTAs; grid == 0: only prepare the kernel (shared
// memory attribute) and return its resident CTAs per SM in *per_sm.
template <bool CUBIC, bool CF, bool APO, class IQ, bool SHORT>
bool launch_batch_t(const DasBatchParams* P, const int2* items, int nitems, int* counter, int grid, int* per_sm,
                    cudaStream_t st)
{
    auto kern = das_batch_kernel<HERCULES, CUBIC, CF, APO, IQ, SHORT>;
    const size_t smem = sizeof(Smem<IQ, coef_arrays<HERCULES, CUBIC, APO>()>);
    if (grid <= 0) {
        CUTB_CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CUTB_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, kThreads, smem));
        return true;
    }
    kern<<<grid, kThreads, smem, st>>>(*P, items, nitems, counter);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

template <class IQ, bool SHORT>
bool launch_batch_s(const DasBatchParams* P, const int2* items, int nitems, int* counter, const DasArgs& a, int grid,
                    int* per_sm, cudaStream_t st)
{
#define CUTB_BATCH_CASE(CUBIC, CF, APO)                                                 \
    if ((bool)a.cubic == CUBIC && (bool)a.apply_cf == CF && (bool)a.use_apo == APO) \
        return launch_batch_t<CUBIC, CF, APO, IQ, SHORT>(P, items, nitems, counter, grid, per_sm, st);
    CUTB_BATCH_CASE(true, true, false)
    CUTB_BATCH_CASE(true, false, false)
    CUTB_BATCH_CASE(false, true, false)
    CUTB_BATCH_CASE(false, false, false)
    CUTB_BATCH_CASE(true, true, true)
    CUTB_BATCH_CASE(true, false, true)
    CUTB_BATCH_CASE(false, true, true)
    CUTB_BATCH_CASE(false, false, true)
#undef CUTB_BATCH_CASE
    return false;
}
}  // namespace

bool launch_das_batch(const DasBatchParams* P, const int2* items, int nitems, int* counter, const DasArgs& like,
                      bool iq_bf16, bool short_tile, int grid, int* per_sm, cudaStream_t st)
{
    CUTB_REQUIRE(like.seq == HERCULES, CUTB_ERR_UNSUPPORTED, "Batched delay-and-sum supports HERCULES frames.");
    CUTB_REQUIRE(grid <= 0 || (nitems > 0 && items && counter && P), CUTB_ERR_INVALID_ARGUMENT, "Empty batch.");
    CUTB_REQUIRE(grid > 0 || per_sm, CUTB_ERR_INVALID_ARGUMENT, "Missing occupancy output.");
    if (short_tile)
        return iq_bf16 ? launch_batch_s<__nv_bfloat162, true>(P, items, nitems, counter, like, grid, per_sm, st)
                       : launch_batch_s<float2, true>(P, items, nitems, counter, like, grid, per_sm, st);
    return iq_bf16 ? launch_batch_s<__nv_bfloat162, false>(P, items, nitems, counter, like, grid, per_sm, st)
                   : launch_batch_s<float2, false>(P, items, nitems, counter, like, grid, per_sm, st);
}

void das_grid_tiles(const DasArgs& a, int counts[3])
{
    int shape[3];
    das_tile_shape(a, shape);
    for (int i = 0; i < 3; ++i) counts[i] = div_up(i == 0 ? a.X : i == 1 ? a.Y : a.Z, shape[i]);
    if (!das_3d(a)) counts[1] = 1;  // y-invariant: one slice of tiles
}

void das_tile_shape(const DasArgs& a, int shape[3])
{
    if (das_direct(a)) {  // one thread per voxel: no tiles
        shape[0] = shape[1] = shape[2] = 1;
        return;
    }
    const bool sh = use_short_tile(a);
    shape[0] = das_3d(a) ? (sh ? Layout<HERCULES, true>::TX : Layout<HERCULES, false>::TX) : Layout<FORCES, false>::TX;
    shape[1] = das_3d(a) ? 8 : 1;
    shape[2] = sh ? Layout<HERCULES, true>::TZ : Layout<HERCULES, false>::TZ;
}

bool prepare_das(const DasArgs& a, bool iq_bf16)
{
    // sample counts the delay-and-sum rejects are reported at launch
    if (!das_staged(a) || a.S % 4 != 0) return true;
    g_prepare_only = true;
    const bool ok = launch_das(a, nullptr, iq_bf16, nullptr, nullptr, nullptr);
    g_prepare_only = false;
    return ok;
}

bool launch_das(const DasArgs& a, const void* iq, bool iq_bf16, void* volume, cudaStream_t st, int* launches)
{
    CUTB_REQUIRE(a.status != nullptr, CUTB_ERR_NOT_INITIALIZED, "Delay-and-sum status word not allocated.");
    CUTB_REQUIRE((uintptr_t)iq % 16 == 0, CUTB_ERR_INVALID_ARGUMENT,
                 "The analytic-signal buffer must be 16-byte aligned.");
    CUTB_REQUIRE(a.S % 4 == 0, CUTB_ERR_UNSUPPORTED,
                 "Delay-and-sum needs a sample count that is a multiple of 4 (got %d).", a.S);
    bool ok;
    if (a.seq == RCA_TPW || a.seq == UFORCES) {
        CUTB_REQUIRE(!a.tiles, CUTB_ERR_UNSUPPORTED, "Tile lists need HERCULES.");
        if (das_direct(a)) {
            if (g_prepare_only) return true;
            ok = launch_das_direct(a, iq, iq_bf16, volume, st);
        } else if (a.seq == UFORCES) {
            ok = iq_bf16 ? launch_das_seq<UFORCES, __nv_bfloat162, false>(a, iq, volume, st)
                         : launch_das_seq<UFORCES, float2, false>(a, iq, volume, st);
        } else if (a.focus != 2) {  // plane waves in the x-z plane: y-invariant
            ok = iq_bf16 ? launch_das_seq<RCA_TPW, __nv_bfloat162, false>(a, iq, volume, st)
                         : launch_das_seq<RCA_TPW, float2, false>(a, iq, volume, st);
        } else if (use_short_tile(a)) {
            ok = iq_bf16 ? launch_das_seq<kTpwYz, __nv_bfloat162, true>(a, iq, volume, st)
                         : launch_das_seq<kTpwYz, float2, true>(a, iq, volume, st);
        } else {
            ok = iq_bf16 ? launch_das_seq<kTpwYz, __nv_bfloat162, false>(a, iq, volume, st)
                         : launch_das_seq<kTpwYz, float2, false>(a, iq, volume, st);
        }
        if (ok && launches && !g_prepare_only) ++*launches;
        return ok;
    }
    CUTB_REQUIRE(!a.tiles || (a.ntiles > 0 && a.ntiles <= (1 << 24)), CUTB_ERR_INVALID_ARGUMENT, "Bad tile list.");
    CUTB_REQUIRE(a.splits <= 1 || (a.tiles && !a.apply_cf && a.seq == HERCULES), CUTB_ERR_UNSUPPORTED,
                 "Split delay-and-sum needs a tile list, HERCULES and no coherence factor.");
    if (use_short_tile(a))
        ok = iq_bf16 ? launch_das_s<HERCULES, __nv_bfloat162, true>(a, iq, volume, st)
                     : launch_das_s<HERCULES, float2, true>(a, iq, volume, st);
    else if (a.seq == HERCULES)
        ok = iq_bf16 ? launch_das_s<HERCULES, __nv_bfloat162, false>(a, iq, volume, st)
                     : launch_das_s<HERCULES, float2, false>(a, iq, volume, st);
    else
        ok = iq_bf16 ? launch_das_s<FORCES, __nv_bfloat162, false>(a, iq, volume, st)
                     : launch_das_s<FORCES, float2, false>(a, iq, volume, st);
    if (ok && launches) ++*launches;
    return ok;
}

}  // namespace cutb
