// Host driver for the shared-memory FFT building blocks (csrc/fft_core.cuh), compiled with g++.
// The passes of one transform run thread by thread (tau = 0 .. N/16 - 1), with every barrier of the
// device kernel becoming the end of a loop over the threads. For each length 2^4 .. 2^13 and a
// nonzero bank skew it checks that
//   * the paired transform (two inputs on the lanes of float2) equals, lane by lane and bit for bit,
//     the scalar transform of each input;
//   * both agree with an FP64 DFT to FP32 rounding (relative L2 below 1e-5).
// For 2^14 .. 2^17 it also runs the scalar transform with its exchange arrays split into slices of
// 2^14 elements, as the thread-block-cluster kernel holds them (one slice per CTA): the result must
// equal the single-array transform bit for bit and an FP64 radix-2 FFT to FP32 rounding.
// Prints one line per length and exits non-zero on the first failure.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "fft_core.cuh"

using namespace cutb::fft;

template <int LOGN, int SIGN, int P = 0>
void scalar_passes(std::vector<cplx[16]>& x, const cplx* tw, float* sre, float* sim,
                   const std::vector<BaseTwiddles<LOGN>>& wb)
{
    constexpr int NP = pass_count(LOGN);
    if constexpr (P < NP) {
        const uint32_t T = (uint32_t)x.size();
        for (uint32_t tau = 0; tau < T; ++tau) fft_pass<LOGN, P, SIGN>(x[tau], tau, tw, sre, sim, wb[tau]);
        if constexpr (P < NP - 1)
            for (uint32_t tau = 0; tau < T; ++tau) fft_gather<LOGN>(x[tau], tau, sre, sim);
        scalar_passes<LOGN, SIGN, P + 1>(x, tw, sre, sim, wb);
    }
}

template <int LOGN, int SIGN, int P = 0>
void paired_passes(std::vector<cplx2[16]>& x, const cplx* tw, float2* sre, float2* sim, uint32_t skew,
                   const std::vector<BaseTwiddles<LOGN>>& wb)
{
    constexpr int NP = pass_count(LOGN);
    if constexpr (P < NP) {
        const uint32_t T = (uint32_t)x.size();
        for (uint32_t tau = 0; tau < T; ++tau) fft_pass2<LOGN, P, SIGN>(x[tau], tau, tw, sre, sim, skew, wb[tau]);
        if constexpr (P < NP - 1)
            for (uint32_t tau = 0; tau < T; ++tau) fft_gather2<LOGN>(x[tau], tau, sre, sim, skew);
        paired_passes<LOGN, SIGN, P + 1>(x, tw, sre, sim, skew, wb);
    }
}

static bool same_bits(float a, float b) { return std::memcmp(&a, &b, sizeof(float)) == 0; }

// Exchange arrays in slices of 2^14 elements (slice pos >> 14, offset pos & (2^14 - 1)).
struct SlicedExchange {
    std::vector<float>* re;
    std::vector<float>* im;
    void store(uint32_t pos, cplx v) const
    {
        re[pos >> 14][pos & 16383u] = v.x;
        im[pos >> 14][pos & 16383u] = v.y;
    }
    cplx load(uint32_t pos) const { return {re[pos >> 14][pos & 16383u], im[pos >> 14][pos & 16383u]}; }
};

template <int LOGN, int SIGN, class EX, int P = 0>
void ex_passes(std::vector<cplx[16]>& x, const cplx* tw, const EX& ex, const std::vector<BaseTwiddles<LOGN>>& wb)
{
    constexpr int NP = pass_count(LOGN);
    if constexpr (P < NP) {
        const uint32_t T = (uint32_t)x.size();
        for (uint32_t tau = 0; tau < T; ++tau) fft_pass_ex<LOGN, P, SIGN>(x[tau], tau, tw, ex, wb[tau]);
        if constexpr (P < NP - 1)
            for (uint32_t tau = 0; tau < T; ++tau) fft_gather_ex<LOGN>(x[tau], tau, ex);
        ex_passes<LOGN, SIGN, EX, P + 1>(x, tw, ex, wb);
    }
}

// FP64 radix-2 FFT, sum_j a[j] exp(sign 2 pi i j k / n).
static void fft64(std::vector<std::complex<double>>& a, int sign)
{
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    const double two_pi = 6.283185307179586476925286766559;
    for (size_t len = 2; len <= n; len <<= 1)
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < len / 2; ++k) {
                const std::complex<double> w = std::polar(1.0, sign * two_pi * (double)k / (double)len);
                const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
}

template <int LOGN, int SIGN>
bool check_sliced(std::mt19937& rng)
{
    constexpr uint32_t N = 1u << LOGN, T = N / 16, R = N >> 14;
    const double two_pi = 6.283185307179586476925286766559;
    std::vector<cplx> tw(N);
    for (uint32_t m = 0; m < N; ++m) {
        const std::complex<double> w = std::polar(1.0, -two_pi * m / N);
        tw[m] = {(float)w.real(), (float)w.imag()};
    }
    std::vector<BaseTwiddles<LOGN>> wb(T);
    for (uint32_t tau = 0; tau < T; ++tau) load_base_twiddles<LOGN>(wb[tau], tau, tw.data());
    std::normal_distribution<float> g(0.f, 1.f);
    std::vector<cplx> a(N);
    for (auto& v : a) v = {g(rng), g(rng)};
    std::vector<cplx[16]> xs(T), xw(T);
    for (uint32_t tau = 0; tau < T; ++tau)
        for (int m = 0; m < 16; ++m) xs[tau][m] = xw[tau][m] = a[tau + m * T];
    std::vector<float> re(N), im(N);
    std::vector<std::vector<float>> sre(R, std::vector<float>(16384)), sim(R, std::vector<float>(16384));
    ex_passes<LOGN, SIGN>(xw, tw.data(), ShmemPair{re.data(), im.data()}, wb);
    ex_passes<LOGN, SIGN>(xs, tw.data(), SlicedExchange{sre.data(), sim.data()}, wb);
    std::vector<std::complex<double>> ref(N);
    for (uint32_t n = 0; n < N; ++n) ref[n] = {a[n].x, a[n].y};
    fft64(ref, SIGN);
    double num = 0, den = 0;
    for (uint32_t tau = 0; tau < T; ++tau)
        for (int m = 0; m < 16; ++m) {
            const cplx u = xs[tau][m], w = xw[tau][m];
            if (!same_bits(u.x, w.x) || !same_bits(u.y, w.y)) {
                std::printf("FAIL 2^%d: sliced exchange differs at n = %u\n", LOGN, tau + m * T);
                return false;
            }
            const std::complex<double> r = ref[tau + m * T];
            num += std::norm(std::complex<double>(u.x, u.y) - r);
            den += std::norm(r);
        }
    const double rel = std::sqrt(num / den);
    std::printf("2^%d sign %+d in %u slices: equals the single-array transform bit for bit, rel-L2 vs FP64 %.2e\n",
                LOGN, SIGN, R, rel);
    return rel < 1e-5;
}

template <int LOGN, int SIGN>
bool check(uint32_t skew, std::mt19937& rng)
{
    constexpr uint32_t N = 1u << LOGN, T = N / 16;
    const double two_pi = 6.283185307179586476925286766559;
    std::vector<cplx> tw(N);
    for (uint32_t m = 0; m < N; ++m) {
        const std::complex<double> w = std::polar(1.0, -two_pi * m / N);
        tw[m] = {(float)w.real(), (float)w.imag()};
    }
    std::vector<BaseTwiddles<LOGN>> wb(T);
    for (uint32_t tau = 0; tau < T; ++tau) load_base_twiddles<LOGN>(wb[tau], tau, tw.data());

    std::normal_distribution<float> g(0.f, 1.f);
    std::vector<cplx> a(N), b(N);
    for (uint32_t n = 0; n < N; ++n) a[n] = {g(rng), g(rng)}, b[n] = {g(rng), g(rng)};

    // element n = tau + m T sits in register m of thread tau before the first pass and after the last
    std::vector<cplx[16]> xa(T), xb(T);
    std::vector<cplx2[16]> xp(T);
    for (uint32_t tau = 0; tau < T; ++tau)
        for (int m = 0; m < 16; ++m) {
            const uint32_t n = tau + m * T;
            xa[tau][m] = a[n];
            xb[tau][m] = b[n];
            xp[tau][m] = {make_float2(a[n].x, b[n].x), make_float2(a[n].y, b[n].y)};
        }
    std::vector<float> sre(N), sim(N);
    std::vector<float2> pre(N), pim(N);
    scalar_passes<LOGN, SIGN>(xa, tw.data(), sre.data(), sim.data(), wb);
    scalar_passes<LOGN, SIGN>(xb, tw.data(), sre.data(), sim.data(), wb);
    paired_passes<LOGN, SIGN>(xp, tw.data(), pre.data(), pim.data(), skew, wb);

    double num = 0, den = 0;
    for (uint32_t tau = 0; tau < T; ++tau)
        for (int m = 0; m < 16; ++m) {
            const cplx2 p = xp[tau][m];
            const cplx sa = xa[tau][m], sb = xb[tau][m];
            if (!same_bits(p.re.x, sa.x) || !same_bits(p.im.x, sa.y) || !same_bits(p.re.y, sb.x) ||
                !same_bits(p.im.y, sb.y)) {
                std::printf("FAIL 2^%d sign %d skew %u: paired lane differs from scalar at n = %u\n", LOGN, SIGN,
                            skew, tau + m * T);
                return false;
            }
            // FP64 DFT of input a at bin k = n
            const uint32_t k = tau + m * T;
            std::complex<double> ref = 0;
            for (uint32_t n = 0; n < N; ++n)
                ref += std::complex<double>(a[n].x, a[n].y) * std::polar(1.0, SIGN * two_pi * ((uint64_t)k * n % N) / N);
            num += std::norm(std::complex<double>(sa.x, sa.y) - ref);
            den += std::norm(ref);
        }
    const double rel = std::sqrt(num / den);
    std::printf("2^%d sign %+d skew %u: paired == scalar bit for bit, rel-L2 vs FP64 %.2e\n", LOGN, SIGN, skew, rel);
    return rel < 1e-5;
}

template <int LOGN>
bool check_len(std::mt19937& rng)
{
    return check<LOGN, +1>(0, rng) && check<LOGN, -1>(0, rng) && check<LOGN, +1>(LOGN < 8 ? 6 : 0, rng);
}

int main()
{
    std::mt19937 rng(7);
    const bool ok = check_len<4>(rng) && check_len<5>(rng) && check_len<6>(rng) && check_len<7>(rng) &&
                    check_len<8>(rng) && check_len<9>(rng) && check_len<10>(rng) && check_len<11>(rng) &&
                    check_len<12>(rng) && check_len<13>(rng) && check_sliced<14, -1>(rng) &&
                    check_sliced<15, -1>(rng) && check_sliced<16, +1>(rng) && check_sliced<17, -1>(rng);
    return ok ? 0 : 1;
}
