/*
 * ORACLE — CPU restatement of the upstream toolkit's RF -> volume path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: tests/, the smoke()
 * entry point and the bench's cpu_baseline leg may load it; the product library
 * never links, loads or calls it, and has no CPU fallback.
 *
 * Everything below restates the upstream formulas in FP64 (double) arithmetic,
 * except orc_convert_decode_i16, which reproduces the upstream FP32 result bit
 * for bit (the sums are exact integers, see there). Each function cites the
 * upstream file:line it follows (paths relative to the upstream repository
 * root, cuda_toolkit/src/...).
 *
 * Pinning: the upstream repository ships no tests, golden vectors or known-answer tests. This
 * restatement is pinned by (1) closed-form known answers (H*H^T = N*I, decode(H^T x) == x, the
 * analytic signal of pure cosines, the focus of a point scatterer, linearity) and (2) the golden
 * fixtures under tests/golden/, produced by upstream's own code: its sources compiled unmodified
 * for the CPU (oracle/Makefile.ref, CUDA/cuBLAS/cuFFT emulated by oracle/ref_shim/) and driven
 * through its entry points by tests/golden/make_golden.py.
 *
 * Threads: std::thread over rows / voxels; nthreads <= 0 uses every host core.
 */
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "../include/cuda_beamformer_parameters.h"

using cd = std::complex<double>;

namespace {

int resolve_threads(int n)
{
    if (n > 0) return n;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

template <class F>
void parallel_for(size_t count, int nthreads, F&& fn)
{
    nthreads = resolve_threads(nthreads);
    if (count == 0) return;
    if (nthreads == 1 || count < 2) { fn(size_t(0), count); return; }
    size_t chunk = (count + nthreads - 1) / nthreads;
    std::vector<std::thread> pool;
    for (int i = 0; i < nthreads; ++i) {
        size_t b = i * chunk, e = std::min(count, b + chunk);
        if (b >= e) break;
        pool.emplace_back([&, b, e] { fn(b, e); });
    }
    for (auto& t : pool) t.join();
}

bool is_pow2(unsigned n) { return n && !(n & (n - 1)); }

/*
 * Base Hadamard matrices of order 12 and 20 built from the quadratic-residue
 * character chi_q (chi(0) = 0, +1 on residues, -1 on non-residues), bordered by a
 * first row and column of +1:
 *   order 12 (q = 11): core[i][j] = -1 on the diagonal, chi(i - j) elsewhere;
 *   order 20 (q = 19): core[i][j] = -chi(i + j) (back-circulant), -1 where i + j = 0 mod q,
 * with i, j counted from 0 inside the core. These are the exact base tables that the
 * upstream decoder embeds (hadamard_decoder.cpp:8-45); the golden fixture
 * tests/golden/encoding_matrices.npz checks every supported order against the
 * upstream generator itself.
 */
std::vector<int> qr_base(unsigned order)
{
    unsigned q = order - 1;
    std::vector<int> chi(q, -1);
    chi[0] = 0;
    for (unsigned x = 1; x < q; ++x) chi[(x * x) % q] = 1;
    std::vector<int> h(order * order, 1);
    for (unsigned i = 1; i < order; ++i)
        for (unsigned j = 1; j < order; ++j) {
            unsigned a = i - 1, b = j - 1;
            int v;
            if (order == 12) v = (a == b) ? -1 : chi[(a + q - b) % q];
            else { unsigned k = (a + b) % q; v = k == 0 ? -1 : -chi[k]; }
            h[i * order + j] = v;
        }
    return h;
}

} // namespace

extern "C" {

/*
 * Encoding matrix of order n, row-major +-1 (hadamard_decoder.cpp:110-189, 191-222).
 * Sylvester doubling [[H, H], [H, -H]] from a base of order 1 (n = 2^k), 12 (n = 12*2^k)
 * or 20 (n = 20*2^k). ordering == 2 (WALSH) reorders the rows by their number of sign
 * changes. Returns 0, or -1 for an unsupported order.
 */
int orc_encoding_matrix(unsigned n, int ordering, signed char* out)
{
    if (n == 0 || n > 1024) return -1;
    unsigned base;
    std::vector<int> b;
    if (is_pow2(n)) { base = 1; b = {1}; }
    else if (n % 12 == 0 && is_pow2(n / 12)) { base = 12; b = qr_base(12); }
    else if (n % 20 == 0 && is_pow2(n / 20)) { base = 20; b = qr_base(20); }
    else return -1;
    std::vector<int> h((size_t)n * n, 0);
    for (unsigned i = 0; i < base; ++i)
        for (unsigned j = 0; j < base; ++j) h[(size_t)i * n + j] = b[i * base + j];
    for (unsigned len = base; len < n; len *= 2)
        for (unsigned r = 0; r < len; ++r)
            for (unsigned c = 0; c < len; ++c) {
                int v = h[(size_t)r * n + c];
                h[(size_t)r * n + c + len] = v;
                h[(size_t)(r + len) * n + c] = v;
                h[(size_t)(r + len) * n + c + len] = -v;
            }
    std::vector<unsigned> order(n);
    std::iota(order.begin(), order.end(), 0u);
    if (ordering == 2) {
        std::vector<unsigned> flips(n, 0);
        for (unsigned r = 0; r < n; ++r)
            for (unsigned c = 0; c + 1 < n; ++c)
                flips[r] += h[(size_t)r * n + c] * h[(size_t)r * n + c + 1] < 0;
        /* std::sort with upstream's comparator (hadamard_decoder.cpp:209-211): ties between rows
         * of equal sign-change count (possible with the 12/20 bases) are ordered as upstream's
         * sort orders them with the same C++ standard library. */
        std::sort(order.begin(), order.end(), [&](unsigned a, unsigned bb) { return flips[a] < flips[bb]; });
    }
    for (unsigned r = 0; r < n; ++r)
        for (unsigned c = 0; c < n; ++c) out[(size_t)r * n + c] = (signed char)h[(size_t)order[r] * n + c];
    return 0;
}

/*
 * Convert + channel reorder + decode of int16 raw data, reproducing the upstream
 * FP32 result exactly (data_conversion_kernels.cuh:25-41, hadamard_decoder.cpp:49-78).
 * raw: [R1][R0] int16, element (t, s) of raw channel m at m*R0 + t*S + s.
 * out: [T][C][S] float, out[t'][c][s] = fl32(fl32(1/T) * sum_t H[t'][t] * raw(map[c], t, s)).
 * The sum of at most 512 int16 products is an integer below 2^24, so FP32 accumulation
 * upstream is exact in any order; here it is accumulated in int64 and rounded once.
 * encoding 0 (NONE): out = raw reordered, no scaling.
 */
int orc_convert_decode_i16(const int16_t* raw, unsigned R0, unsigned R1, unsigned S, unsigned C, unsigned T,
                           const int16_t* map, int encoding, float* out, int nthreads)
{
    if ((size_t)T * S > R0) return -1;
    for (unsigned c = 0; c < C; ++c)
        if (map[c] < 0 || (unsigned)map[c] >= R1) return -1;
    std::vector<signed char> H;
    if (encoding != 0) {
        H.resize((size_t)T * T);
        if (orc_encoding_matrix(T, encoding, H.data()) != 0) return -1;
    }
    const float alpha = 1.0f / (float)T;
    parallel_for((size_t)C, nthreads, [&](size_t c0, size_t c1) {
        std::vector<int64_t> col(T);
        for (size_t c = c0; c < c1; ++c) {
            const int16_t* src = raw + (size_t)map[c] * R0;
            for (unsigned s = 0; s < S; ++s) {
                for (unsigned t = 0; t < T; ++t) col[t] = src[(size_t)t * S + s];
                for (unsigned tp = 0; tp < T; ++tp) {
                    float v;
                    if (encoding == 0) {
                        v = (float)col[tp];
                    } else {
                        int64_t acc = 0;
                        const signed char* hr = H.data() + (size_t)tp * T;
                        for (unsigned t = 0; t < T; ++t) acc += hr[t] * col[t];
                        v = alpha * (float)acc;
                    }
                    out[((size_t)tp * C + c) * S + s] = v;
                }
            }
        }
    });
    return 0;
}

/*
 * Same stage in FP64 for any input type (data_type 1 = int16, 2 = float32):
 * out[t'][c][s] = (1/T) * sum_t H[t'][t] * raw(map[c], t, s) in double.
 */
int orc_convert_decode_f64(const void* raw, int data_type, unsigned R0, unsigned R1, unsigned S, unsigned C,
                           unsigned T, const int16_t* map, int encoding, double* out, int nthreads)
{
    if ((size_t)T * S > R0 || (data_type != 1 && data_type != 2)) return -1;
    for (unsigned c = 0; c < C; ++c)
        if (map[c] < 0 || (unsigned)map[c] >= R1) return -1;
    std::vector<signed char> H;
    if (encoding != 0) {
        H.resize((size_t)T * T);
        if (orc_encoding_matrix(T, encoding, H.data()) != 0) return -1;
    }
    parallel_for((size_t)C, nthreads, [&](size_t c0, size_t c1) {
        std::vector<double> col(T);
        for (size_t c = c0; c < c1; ++c) {
            size_t base = (size_t)map[c] * R0;
            for (unsigned s = 0; s < S; ++s) {
                for (unsigned t = 0; t < T; ++t) {
                    size_t k = base + (size_t)t * S + s;
                    col[t] = data_type == 1 ? (double)((const int16_t*)raw)[k] : (double)((const float*)raw)[k];
                }
                for (unsigned tp = 0; tp < T; ++tp) {
                    double v;
                    if (encoding == 0) v = col[tp];
                    else {
                        double acc = 0;
                        const signed char* hr = H.data() + (size_t)tp * T;
                        for (unsigned t = 0; t < T; ++t) acc += hr[t] * col[t];
                        v = acc / T;
                    }
                    out[((size_t)tp * C + c) * S + s] = v;
                }
            }
        }
    });
    return 0;
}

} // extern "C"

namespace {

/* In-place FP64 DFT of length n (iterative radix-2 for powers of two, direct sum otherwise). */
void dft(std::vector<cd>& a, int sign)
{
    size_t n = a.size();
    if (n <= 1) return;
    if (!is_pow2((unsigned)n)) {
        std::vector<cd> r(n);
        for (size_t k = 0; k < n; ++k) {
            cd acc = 0;
            for (size_t j = 0; j < n; ++j) {
                double ang = sign * 2.0 * M_PI * (double)((k * j) % n) / (double)n;
                acc += a[j] * cd(std::cos(ang), std::sin(ang));
            }
            r[k] = acc;
        }
        a.swap(r);
        return;
    }
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    /* w[k] = exp(sign 2 pi i k / n); stage `len` uses w[k * n / len] (the same angles, from one table) */
    std::vector<cd> w(n / 2);
    for (size_t k = 0; k < n / 2; ++k) {
        double ang = sign * 2.0 * M_PI * (double)k / (double)n;
        w[k] = cd(std::cos(ang), std::sin(ang));
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        size_t half = len / 2, step = n / len;
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < half; ++k) {
                cd u = a[i + k], v = a[i + k + half] * w[k * step];
                a[i + k] = u + v;
                a[i + k + half] = u - v;
            }
    }
}

} // namespace

extern "C" {

/*
 * Match-filtered analytic signal of each row (hilbert_handler.cu:55-78, 132-155;
 * hilbert_kernels.cuh:17-40). For a row x of length N:
 *   X = DFT(x); Y[k] = X[k] * w_k * F[k] for 0 <= k <= N/2 (integer division), Y[k] = 0 above,
 *   w_0 = 0.75/N, w_k = 1.5/N otherwise (the Nyquist bin keeps 1.5/N),
 *   F = DFT_N of the zero-padded taps (F = 1 when ntaps == 0): circular convolution, no reversal;
 *   iq = sum_k Y[k] exp(+2*pi*i*k*n/N)  (unnormalised inverse).
 * in: rows x N real (double); out: rows x N complex (interleaved re, im).
 */
int orc_hilbert(const double* in, size_t rows, unsigned N, const float* taps, unsigned ntaps, double* out,
                int nthreads)
{
    if (N == 0 || ntaps > N) return -1;
    std::vector<cd> F(N, cd(1.0, 0.0));
    if (ntaps) {
        std::fill(F.begin(), F.end(), cd(0, 0));
        for (unsigned i = 0; i < ntaps; ++i) F[i] = (double)taps[i];
        dft(F, -1);
    }
    const unsigned half = N / 2;
    parallel_for(rows, nthreads, [&](size_t r0, size_t r1) {
        std::vector<cd> a(N);
        for (size_t r = r0; r < r1; ++r) {
            for (unsigned n = 0; n < N; ++n) a[n] = in[r * N + n];
            dft(a, -1);
            for (unsigned k = 0; k < N; ++k) {
                if (k > half) { a[k] = 0; continue; }
                double w = (k == 0 ? 0.75 : 1.5) / (double)N;
                a[k] *= w * F[k];
            }
            dft(a, +1);
            for (unsigned n = 0; n < N; ++n) {
                out[(r * N + n) * 2] = a[n].real();
                out[(r * N + n) * 2 + 1] = a[n].imag();
            }
        }
    });
    return 0;
}

} // extern "C"

namespace {

/* Geometry derived from the parameter block (beamformer.cu:17-98), in double. */
struct Geometry {
    unsigned S, C, T, G;          /* samples, channels, transmits, READI groups (>= 1) */
    unsigned X, Y, Z;
    double spm;                   /* samples per metre = fs / c */
    double px, py;                /* element pitch */
    double xmin_x, xmin_y;        /* centre of the first element: -half_aperture + pitch/2 */
    double xmax_x, xmax_y;
    double delay;                 /* (int)(time_offset * fs) */
    double vmin[3], res[3];
    double fz, fy;                /* focal point (fz = 0 for plane waves) */
    int focus;                    /* 2 = YZ_PLANE, 4 = YZ_FOCUS, 1 XZ_PLANE, 3 XZ_FOCUS, 0 none */
    double fn_rx, fn_tx, cf_power, to_power;
    int apo_type, seq, encoding, interpolate;
    uint64_t readi_row;           /* bit g set: sub-signal g is negated */
};

int derive(const CudaBeamformerParameters& bp, Geometry& g)
{
    g.S = bp.dec_data_dim[0];
    g.C = bp.dec_data_dim[1];
    g.T = bp.dec_data_dim[2];
    g.X = bp.output_points[0];
    g.Y = bp.output_points[1];
    g.Z = bp.output_points[2];
    if (!g.S || !g.C || !g.T || !g.X || !g.Y || !g.Z) return -1;
    /* The constants are FP32 values upstream (BeamformerConstants, beamformer_constants.cuh:32-72,
     * filled by beamformer.cu:17-98 in float arithmetic); they are formed the same way here and
     * only the per-voxel arithmetic below runs in double. */
    const float spm = bp.sampling_frequency / bp.speed_of_sound;
    const float hpx = bp.xdc_element_pitch[0] * 0.5f, hpy = bp.xdc_element_pitch[1] * 0.5f;
    g.spm = spm;
    g.px = bp.xdc_element_pitch[0];
    g.py = bp.xdc_element_pitch[1];
    g.xmin_x = (float)(-bp.xdc_transform[12] + hpx);
    g.xmin_y = (float)(-bp.xdc_transform[13] + hpy);
    g.xmax_x = (float)(bp.xdc_transform[12] - hpx);
    g.xmax_y = (float)(bp.xdc_transform[13] - hpy);
    g.delay = (double)(int)(bp.time_offset * bp.sampling_frequency);
    for (int a = 0; a < 3; ++a) g.vmin[a] = bp.output_min_coordinate[a];
    /* Lateral step is used for both x and y (beamformer.cu:42-49); a single point has step 0. */
    const float rx = g.X > 1 ? (bp.output_max_coordinate[0] - bp.output_min_coordinate[0]) / (float)(g.X - 1) : 0.f;
    const float rz = g.Z > 1 ? (bp.output_max_coordinate[2] - bp.output_min_coordinate[2]) / (float)(g.Z - 1) : 0.f;
    g.res[0] = rx;
    g.res[1] = rx;
    g.res[2] = rz;
    g.fy = bp.foci[1];
    g.fz = bp.foci[2];
    g.seq = bp.das_shader_id;
    if (bp.tx_orientation == ORIENT_NONE) g.focus = 0;
    else if (std::isinf(bp.foci[2]) || bp.das_shader_id == RCA_TPW) {
        g.fz = 0.0;
        g.focus = bp.tx_orientation == bp.rx_orientation ? 1 : 2;
    } else {
        g.focus = bp.tx_orientation == bp.rx_orientation ? 3 : 4;
    }
    g.fn_rx = bp.fn_rx;
    g.fn_tx = bp.fn_tx;
    g.cf_power = std::min(std::max((double)bp.coherency_weighting, 0.0), 1.0);
    g.to_power = bp.to_power;
    g.apo_type = bp.apo_type;
    g.encoding = bp.decode;
    g.interpolate = bp.interpolate ? 1 : 0;
    g.G = (unsigned)(uint8_t)bp.readi_group_count;
    if (g.G == 0) g.G = 1;
    g.readi_row = 0;
    if (g.G > 1) {
        if (g.encoding == 0) return -1;
        if (g.G > 64) return -1;
        std::vector<signed char> h((size_t)g.G * g.G);
        if (orc_encoding_matrix(g.G, g.encoding, h.data()) != 0) return -1;
        unsigned id = (unsigned)(uint8_t)bp.readi_group_id;
        if (id >= g.G) return -1;
        for (unsigned k = 0; k < g.G; ++k)
            if (h[(size_t)id * g.G + k] < 0) g.readi_row |= (uint64_t)1 << k;
    }
    return 0;
}

/* Receive f-number Hann window (beamformer_utils.cuh:142-154). */
double hann_apo(double lateral, double depth, double fnum)
{
    double a = fnum * (lateral / depth) / 2.0;
    a = std::fmin(a, 0.5);  /* fminf semantics upstream: a NaN argument yields 0.5 */
    double c = std::cos(M_PI * a);
    return c * c;
}

/* Sine apodization raised to an integer power (templated_beamformer.cuh:86-99). */
double sin_apo(double loc, double centre, double power)
{
    double a = M_PI * loc / centre;
    a = std::min(std::max(a, -M_PI), M_PI);
    a = std::sin(a);
    double r = 1.0;
    for (unsigned i = 0; (double)i < power; ++i) r *= a;
    return r;
}

/* Row read with index clamped to [1, S-2], then cubic Catmull-Rom (beamformer_utils.cuh:99-125)
 * or linear (:127-140). Taps past the row end read as 0; their weight is 0 at the clamp. */
cd sample_row(const double* row, unsigned S, double idx, int cubic)
{
    idx = std::min(std::max(idx, 1.0), (double)S - 2.0);
    long i = (long)std::floor(idx);
    double t = idx - (double)i;
    auto P = [&](long k) -> cd { return (k >= 0 && k < (long)S) ? cd(row[2 * k], row[2 * k + 1]) : cd(0, 0); };
    if (!cubic) return P(i) + t * (P(i + 1) - P(i));
    cd pm1 = P(i - 1), p0 = P(i), p1 = P(i + 1), p2 = P(i + 2);
    cd m0 = 0.5 * (p1 - pm1), m1 = 0.5 * (p2 - p0);
    double t2 = t * t, t3 = t2 * t;
    double h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + t, h01 = -2 * t3 + 3 * t2, h11 = t3 - t2;
    return h00 * p0 + h01 * p1 + h10 * m0 + h11 * m1;
}

double coherence(cd total, double incoherent, double power)
{
    double cf = std::norm(total) / incoherent;
    cf = std::pow(cf, power);
    return std::isnan(cf) ? 0.0 : cf;
}

/* HERCULES voxel (templated_beamformer.cuh:102-216). CF is applied when its exponent is > 0. */
cd hercules_voxel(const Geometry& g, const double* iq, double vx, double vy, double vz)
{
    double tx_d;
    if (g.focus == 2) {
        tx_d = vz;              /* |(0, vy*sin 0, vz*cos 0)| signed by z, + fz (= 0) */
    } else {
        double ty = vy, tz = vz - g.fz;
        tx_d = std::copysign(std::sqrt(ty * ty + tz * tz), tz) + g.fz;
    }
    cd total = 0;
    double inc = 0;
    unsigned G = g.encoding ? g.G : 1;
    for (unsigned sg = 0; sg < G; ++sg)
        for (unsigned t = 0; t < g.T; ++t) {
            double j;
            if (g.G > 1 && g.encoding == 1) j = (double)sg * g.T + t;
            else if (g.G > 1 && g.encoding == 2) j = (double)t * g.G + sg;
            else j = t;
            double ry = g.xmin_y + j * g.py - vy;
            bool negate = false;
            if (g.G > 1) {
                unsigned bit = sg;
                if (g.encoding == 2 && (t & 1u)) bit = g.G - 1 - sg;
                negate = (g.readi_row >> bit) & 1u;
            }
            for (unsigned c = 0; c < g.C; ++c) {
                double rx = g.xmin_x + (double)c * g.px - vx;
                double apo;
                if (g.apo_type == RX_TO_SIN)
                    apo = sin_apo(rx + vx, g.xmax_x, g.to_power) * sin_apo(ry + vy, g.xmax_y, g.to_power);
                else
                    apo = hann_apo(std::sqrt(rx * rx + ry * ry), vz, g.fn_rx);
                if (!(apo > 0.1)) continue;
                double idx = (tx_d + std::sqrt(rx * rx + ry * ry + vz * vz) + g.fz) * g.spm + g.delay;
                const double* row = iq + ((size_t)t * g.C + c) * g.S * 2;
                cd v = sample_row(row, g.S, idx, g.interpolate);
                total += (negate ? -apo : apo) * v;
                inc += std::norm(v);
            }
        }
    if (g.cf_power > 0) total *= coherence(total, inc, g.cf_power);
    return total;
}

/* FORCES voxel (templated_beamformer.cuh:219-324); y is ignored, CF always applied. */
cd forces_voxel(const Geometry& g, const double* iq, double vx, double vz)
{
    cd total = 0;
    double inc = 0;
    for (unsigned c = 0; c < g.C; ++c) {
        double ec = g.xmin_x + (double)c * g.px;
        double rxx = ec - vx;
        double rx_dist = std::sqrt(rxx * rxx + vz * vz);
        double rx_apo;
        if (g.apo_type == RX_HANN || g.apo_type == TX_TO_SIN) rx_apo = hann_apo(std::fabs(rxx), vz, g.fn_rx);
        else rx_apo = sin_apo(ec, g.xmax_x, g.to_power);
        if (!(rx_apo > 0.0)) continue;
        for (unsigned sg = 0; sg < g.G; ++sg) {
            bool negate = g.G > 1 && ((g.readi_row >> sg) & 1u);
            for (unsigned t = 0; t < g.T; ++t) {
                double et = g.xmin_x + (double)(sg * g.T + t) * g.px;
                double txx = vx - et;
                double tx_apo;
                if (g.apo_type == BOTH_TO_SIN || g.apo_type == TX_TO_SIN) tx_apo = sin_apo(et, g.xmax_x, g.to_power);
                else tx_apo = hann_apo(std::fabs(txx), vz, g.fn_tx);
                double apo = rx_apo * tx_apo;
                double idx = (std::sqrt(txx * txx + vz * vz) + rx_dist) * g.spm + g.delay;
                const double* row = iq + ((size_t)t * g.C + c) * g.S * 2;
                cd v = sample_row(row, g.S, idx, g.interpolate);
                total += (negate ? -apo : apo) * v;
                inc += std::norm(v);
            }
        }
    }
    return total * coherence(total, inc, g.cf_power);
}

/* UFORCES voxel (beamformer_kernels.cu:93-172): the FORCES geometry with transmit elements from
 * the sparse-element table. Transmit row 0 is a discarded flash, so transmit t < T - 1 reads row
 * t + 1; the first used transmit is scaled by 1/sqrt(128); receive element c sits at
 * xdc_mins.x + pitch/2 + c*pitch and transmit t at xdc_mins.x + pitch/2 + (elem[t] - elem[0])*pitch
 * (the focal point of beamformer_kernels.cu:114 plus the element offsets); the index is clamped
 * to [0, S-2] (the tap below sample 0 reads as 0 here); only the receive Hann window applies and
 * the incoherent sum takes the windowed values; CF always applied. */
cd uforces_voxel(const Geometry& g, const double* iq, const short* elems, double vx, double vz)
{
    static const double kISqrt128 = (double)0.088388347648318f;
    cd total = 0;
    double inc = 0;
    const double fx = (double)(float)(g.xmin_x + (float)g.px / 2.f);
    for (unsigned t = 0; t + 1 < g.T; ++t) {
        const double txx = fx + (double)(elems[t] - elems[0]) * g.px - vx;
        const double tx = std::sqrt(txx * txx + vz * vz);
        for (unsigned c = 0; c < g.C; ++c) {
            const double rxx = g.xmin_x - vx + g.px / 2 + (double)c * g.px;
            const double rx = std::sqrt(rxx * rxx + vz * vz);
            double idx = (rx + tx) * g.spm + g.delay;
            idx = std::min(std::max(idx, 0.0), (double)g.S - 2.0);
            const double* row = iq + ((size_t)(t + 1) * g.C + c) * g.S * 2;
            cd v = sample_row(row, g.S, idx < 1.0 ? 1.0 : idx, g.interpolate);
            if (idx < 1.0) {  /* [0, 1): taps -1..2 around sample 0, the tap below 0 reads 0 */
                auto P = [&](long k) -> cd { return (k >= 0 && k < (long)g.S) ? cd(row[2 * k], row[2 * k + 1]) : cd(0, 0); };
                const double tt = idx;
                if (!g.interpolate) {
                    v = P(0) + tt * (P(1) - P(0));
                } else {
                    cd pm1 = 0, p0 = P(0), p1 = P(1), p2 = P(2);
                    cd m0 = 0.5 * (p1 - pm1), m1 = 0.5 * (p2 - p0);
                    double t2 = tt * tt, t3 = t2 * tt;
                    v = (2 * t3 - 3 * t2 + 1) * p0 + (-2 * t3 + 3 * t2) * p1 + (t3 - 2 * t2 + tt) * m0 + (t3 - t2) * m1;
                }
            }
            if (t == 0) v *= kISqrt128;
            v *= hann_apo(std::fabs(rxx), vz, g.fn_rx);
            total += v;
            inc += std::norm(v);
        }
    }
    return total * coherence(total, inc, g.cf_power);
}

/* Tilted-plane-wave voxel (beamformer_kernels.cu:490-550, angles from foci[t][2] as in
 * beamformer.cu:439-443): receive element c at xdc_mins.x + pitch/2 + c*pitch, distance in the
 * x-z plane; transmit path lat*sin(a) + z*cos(a) with lat = y for a YZ plane, x otherwise; the
 * receive Hann window skips values below 0.1; every sample is rotated by
 * exp(i 2 pi idx fc / fs) after the clamp to [1, S-2]; the incoherent sum takes the windowed
 * values; CF always applied. */
cd tpw_voxel(const Geometry& g, const double* iq, const float* angles, double fc_fs, double vx, double vy, double vz)
{
    cd total = 0;
    double inc = 0;
    const double lat = g.focus == 2 ? vy : vx;
    for (unsigned c = 0; c < g.C; ++c) {
        const double rxx = g.xmin_x - vx + g.px / 2 + (double)c * g.px;
        const double rx = std::sqrt(rxx * rxx + vz * vz);
        const double apo = hann_apo(std::fabs(rxx), vz, g.fn_rx);
        if (apo < 0.1) continue;
        for (unsigned t = 0; t < g.T; ++t) {
            const double a = angles[t];
            const double tx = lat * std::sin(a) + vz * std::cos(a);
            double idx = (rx + tx) * g.spm + g.delay;
            idx = std::min(std::max(idx, 1.0), (double)g.S - 2.0);
            const double* row = iq + ((size_t)t * g.C + c) * g.S * 2;
            cd v = sample_row(row, g.S, idx, g.interpolate);
            const double ph = 2.0 * M_PI * idx * fc_fs;
            v *= cd(std::cos(ph), std::sin(ph));
            v *= apo;
            total += v;
            inc += std::norm(v);
        }
    }
    return total * coherence(total, inc, g.cf_power);
}

} // namespace

extern "C" {

/*
 * Delay-and-sum of a complex [T][C][S] analytic signal into a complex [Z][Y][X] volume
 * (beamformer.cu:139-197 dispatch; HERCULES needs a YZ focus, FORCES any focus).
 * voxels: linear voxel indices (z*X*Y + y*X + x) to evaluate, or NULL for all of them;
 * out receives one complex value per evaluated voxel. Returns 0, or -1 if the
 * parameters are rejected (same rejections as the product library).
 */
int orc_das(const double* iq, const CudaBeamformerParameters* bp, const int64_t* voxels, size_t nvox, double* out,
            int nthreads)
{
    Geometry g;
    if (derive(*bp, g) != 0) return -1;
    std::vector<float> angles;
    std::vector<short> elems;
    if (g.seq == HERCULES) {
        if (g.focus != 2 && g.focus != 4) return -1;
        if (g.G > 32) return -1;
    } else if (g.seq == FORCES) {
        if (g.G > 1 && g.encoding != 1) return -1;
    } else if (g.seq == RCA_TPW) {
        if ((g.focus != 1 && g.focus != 2) || g.T > 256) return -1;
        for (unsigned t = 0; t < g.T; ++t) angles.push_back(bp->foci[t * 3 + 2]);
    } else if (g.seq == UFORCES) {
        if (g.focus != 3 || g.T < 2 || g.T > 256 || bp->sparse_elements[0] == -1) return -1;
        for (unsigned t = 0; t < g.T; ++t) elems.push_back(bp->sparse_elements[t]);
    } else {
        return -1;
    }
    const double fc_fs = (double)bp->center_frequency / (double)bp->sampling_frequency;
    size_t total = voxels ? nvox : (size_t)g.X * g.Y * g.Z;
    parallel_for(total, nthreads, [&](size_t b, size_t e) {
        for (size_t k = b; k < e; ++k) {
            size_t lin = voxels ? (size_t)voxels[k] : k;
            size_t x = lin % g.X, y = (lin / g.X) % g.Y, z = lin / ((size_t)g.X * g.Y);
            double vx = g.vmin[0] + (double)x * g.res[0];
            double vy = g.vmin[1] + (double)y * g.res[1];
            double vz = g.vmin[2] + (double)z * g.res[2];
            cd v = g.seq == HERCULES  ? hercules_voxel(g, iq, vx, vy, vz)
                   : g.seq == FORCES  ? forces_voxel(g, iq, vx, vz)
                   : g.seq == RCA_TPW ? tpw_voxel(g, iq, angles.data(), fc_fs, vx, vy, vz)
                                      : uforces_voxel(g, iq, elems.data(), vx, vz);
            out[2 * k] = v.real();
            out[2 * k + 1] = v.imag();
        }
    });
    return 0;
}

int orc_version(void) { return 1; }

} // extern "C"
