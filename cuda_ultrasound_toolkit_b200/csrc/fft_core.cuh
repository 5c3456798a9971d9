// Shared-memory Stockham FFT building blocks for one power-of-two row of N points,
// held by N/16 threads with 16 complex values each.
//
// Invariant between passes: thread tau holds element n = tau + m*(N/16) in register
// x[m] (m = 0..15) before the first pass and after the last one, for every radix
// sequence. That lets a forward and an inverse transform run back to back with the
// spectrum staying in registers (spectral multiply in between), and makes the first
// global load and the last global store coalesced across threads.
//
// Pass with radix R after `ns` points have been combined: butterfly j in [0, N/R)
// reads elements j + r*N/R (r < R), twiddles them by w^(r*(j mod ns)) with
// w = exp(sign*2*pi*i/(ns*R)), runs an R-point DFT and writes element
// (j/ns)*ns*R + (j mod ns) + r*ns. Thread tau runs butterflies j = tau + u*N/16,
// u < 16/R, whose inputs are exactly its registers x[u + r*16/R].
//
// All functions are __host__ __device__ so a CPU test can drive the same arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace cutb {
namespace fft {

struct cplx {
    float x, y;
};

__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b)
{
    return {fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x)};
}
// Multiply by (sign * i): sign = -1 -> -i, +1 -> +i.
template <int SIGN>
__host__ __device__ __forceinline__ cplx mul_i(cplx a)
{
    if constexpr (SIGN < 0) return {a.y, -a.x};
    else return {-a.y, a.x};
}

// exp(SIGN * 2*pi*i * k / 16) for the fixed angles used inside the 8- and 16-point DFTs.
template <int SIGN>
__host__ __device__ __forceinline__ cplx w16(int k)
{
    constexpr float c1 = 0.92387953251128674f, s1 = 0.38268343236508978f, h = 0.70710678118654752f;
    float re, im;
    switch (k & 15) {
        case 0: re = 1.f; im = 0.f; break;
        case 1: re = c1; im = s1; break;
        case 2: re = h; im = h; break;
        case 3: re = s1; im = c1; break;
        case 4: re = 0.f; im = 1.f; break;
        case 5: re = -s1; im = c1; break;
        case 6: re = -h; im = h; break;
        case 7: re = -c1; im = s1; break;
        case 8: re = -1.f; im = 0.f; break;
        case 9: re = -c1; im = -s1; break;
        case 10: re = -h; im = -h; break;
        case 11: re = -s1; im = -c1; break;
        case 12: re = 0.f; im = -1.f; break;
        case 13: re = s1; im = -c1; break;
        case 14: re = h; im = -h; break;
        default: re = c1; im = -s1; break;
    }
    return {re, SIGN < 0 ? -im : im};
}

template <int SIGN>
__host__ __device__ __forceinline__ void dft2(cplx& a, cplx& b)
{
    cplx t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int SIGN>
__host__ __device__ __forceinline__ void dft4(cplx& a, cplx& b, cplx& c, cplx& d)
{
    cplx t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = mul_i<SIGN>(csub(b, d));
    a = cadd(t0, t2);
    c = csub(t0, t2);
    b = cadd(t1, t3);
    d = csub(t1, t3);
}

// In-place R-point DFT of v[0..R-1], natural input and output order.
template <int R, int SIGN>
__host__ __device__ __forceinline__ void dft(cplx (&v)[R])
{
    if constexpr (R == 2) {
        dft2<SIGN>(v[0], v[1]);
    } else if constexpr (R == 4) {
        dft4<SIGN>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        // Even/odd split: two 4-point DFTs, then the radix-2 combination with w8^k.
        cplx e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft4<SIGN>(e[0], e[1], e[2], e[3]);
        dft4<SIGN>(o[0], o[1], o[2], o[3]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            cplx t = k == 0 ? o[0] : cmul(o[k], w16<SIGN>(2 * k));
            v[k] = cadd(e[k], t);
            v[k + 4] = csub(e[k], t);
        }
    } else {
        static_assert(R == 16, "radix");
        // 16 = 4 x 4: DFT over n1 of v[4*n1 + n2], twiddle w16^(n2*k1), DFT over n2.
        cplx y[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            cplx a = v[n2], b = v[4 + n2], c = v[8 + n2], d = v[12 + n2];
            dft4<SIGN>(a, b, c, d);
            y[0][n2] = a; y[1][n2] = b; y[2][n2] = c; y[3][n2] = d;
        }
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1)
#pragma unroll
            for (int n2 = 1; n2 < 4; ++n2) y[k1][n2] = cmul(y[k1][n2], w16<SIGN>(n2 * k1));
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            dft4<SIGN>(y[k1][0], y[k1][1], y[k1][2], y[k1][3]);
            v[k1] = y[k1][0];
            v[k1 + 4] = y[k1][1];
            v[k1 + 8] = y[k1][2];
            v[k1 + 12] = y[k1][3];
        }
    }
}

// Radix of pass p for a transform of size N = 2^logn: radix-16 passes first, the
// remaining factor (2, 4 or 8) last.
__host__ __device__ constexpr int pass_count(int logn) { return logn / 4 + (logn % 4 ? 1 : 0); }
__host__ __device__ constexpr int pass_radix(int logn, int p) { return p < logn / 4 ? 16 : 1 << (logn % 4); }
__host__ __device__ constexpr int pass_ns_log(int logn, int p) { return 4 * p; }  // log2 of points combined before pass p

// Swizzled shared-memory index: the bank bits of i are XORed with S(b), b = i / 32,
// S(b) = (b mod 16) + 16 * bit3(b). A warp's 32 stores of one register in the first pass
// (i = 16 tau + r) and in the second (i = 256 (tau / 16) + tau mod 16 + 16 r) then hit 32
// different banks, and a gather of 32 consecutive elements stays a permutation of one row
// of banks.
__host__ __device__ __forceinline__ uint32_t spad(uint32_t i) { return i ^ (((i >> 5) & 15u) | ((i >> 4) & 16u)); }
__host__ __device__ constexpr uint32_t spad_size(uint32_t n) { return n; }

// Butterflies of pass p for thread tau, reading and writing registers x[]. For the last
// pass the results stay in registers (natural order); otherwise they are scattered to
// the shared arrays sre/sim at their output positions. tw = exp(-2*pi*i*m/N), m < N.
// Base twiddles of the radix-16 passes p > 0 of thread tau: wb[p] = {w^k, w^(4k)} with
// w = exp(-2*pi*i/(ns*16)), k = tau mod ns; the 15 twiddles of the pass are products of these.
template <int LOGN>
struct BaseTwiddles {
    cplx w[pass_count(LOGN) > 1 ? pass_count(LOGN) : 1][2];
};
template <int LOGN>
__host__ __device__ __forceinline__ void load_base_twiddles(BaseTwiddles<LOGN>& wb, uint32_t tau,
                                                            const cplx* __restrict__ tw)
{
#pragma unroll
    for (int p = 1; p < pass_count(LOGN); ++p) {
        if (pass_radix(LOGN, p) != 16) continue;
        const int sh = LOGN - pass_ns_log(LOGN, p) - 4;
        const uint32_t k = tau & ((1u << pass_ns_log(LOGN, p)) - 1);
        wb.w[p][0] = tw[k << sh];
        wb.w[p][1] = tw[(4 * k) << sh];
    }
}

// The exchange arrays of one transform: element `pos` (already swizzled) stored and loaded as
// (re, im). ShmemPair: two float arrays in this CTA's shared memory; a cluster form spreads them
// over the shared memory of several CTAs (hilbert.cu).
struct ShmemPair {
    float* re;
    float* im;
    __host__ __device__ __forceinline__ void store(uint32_t pos, cplx v) const
    {
        re[pos] = v.x;
        im[pos] = v.y;
    }
    __host__ __device__ __forceinline__ cplx load(uint32_t pos) const { return {re[pos], im[pos]}; }
};

template <int LOGN, int P, int SIGN, class EX>
__host__ __device__ __forceinline__ void fft_pass_ex(cplx (&x)[16], uint32_t tau, const cplx* __restrict__ tw,
                                                     const EX& ex, const BaseTwiddles<LOGN>& wb)
{
    constexpr int N = 1 << LOGN;
    constexpr int TPF = N / 16;
    constexpr int R = pass_radix(LOGN, P);
    constexpr int B = 16 / R;
    constexpr int NS_LOG = pass_ns_log(LOGN, P);
    constexpr int NS = 1 << NS_LOG;
    constexpr bool LAST = P == pass_count(LOGN) - 1;
    constexpr int TW_SHIFT = LOGN - NS_LOG - (R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1);  // log2(N/(ns*R))
#pragma unroll
    for (int u = 0; u < B; ++u) {
        const uint32_t j = tau + u * TPF;
        const uint32_t k = j & (NS - 1);
        cplx v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = x[u + r * B];
        if constexpr (P > 0 && R == 16) {
            // w^(r k), r = 1..15, from two table entries w^k and w^(4k): w^(4a + b) = w^(4a) w^b,
            // at most three rounded products deep.
            cplx p[16];
            p[1] = wb.w[P][0];
            p[4] = wb.w[P][1];
            if constexpr (SIGN > 0) p[1].y = -p[1].y, p[4].y = -p[4].y;
            p[2] = cmul(p[1], p[1]);
            p[3] = cmul(p[2], p[1]);
            p[8] = cmul(p[4], p[4]);
            p[12] = cmul(p[8], p[4]);
#pragma unroll
            for (int a4 = 4; a4 < 16; a4 += 4)
#pragma unroll
                for (int b = 1; b < 4; ++b) p[a4 + b] = cmul(p[a4], p[b]);
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], p[r]);
        } else if constexpr (P > 0) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                cplx w = tw[(r * k) << TW_SHIFT];
                if constexpr (SIGN > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        dft<R, SIGN>(v);
        if constexpr (LAST) {
#pragma unroll
            for (int r = 0; r < R; ++r) x[u + r * B] = v[r];
        } else {
            const uint32_t base = (j >> NS_LOG) * (NS * R) + k;
#pragma unroll
            for (int r = 0; r < R; ++r) ex.store(spad(base + r * NS), v[r]);
        }
    }
}

template <int LOGN, int P, int SIGN>
__host__ __device__ __forceinline__ void fft_pass(cplx (&x)[16], uint32_t tau, const cplx* __restrict__ tw,
                                                  float* sre, float* sim, const BaseTwiddles<LOGN>& wb)
{
    fft_pass_ex<LOGN, P, SIGN>(x, tau, tw, ShmemPair{sre, sim}, wb);
}

// Gather this thread's 16 elements (tau + m*N/16) back from the exchange arrays.
template <int LOGN, class EX>
__host__ __device__ __forceinline__ void fft_gather_ex(cplx (&x)[16], uint32_t tau, const EX& ex)
{
    constexpr int TPF = (1 << LOGN) / 16;
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = ex.load(spad(tau + m * TPF));
}

template <int LOGN>
__host__ __device__ __forceinline__ void fft_gather(cplx (&x)[16], uint32_t tau, const float* sre, const float* sim)
{
    fft_gather_ex<LOGN>(x, tau, ShmemPair{const_cast<float*>(sre), const_cast<float*>(sim)});
}

// ---- Two transforms at once on paired FP32 lanes ----------------------------------------------
// Element m of two transforms A and B of the same length and direction is held as
// re = (A.re, B.re), im = (A.im, B.im). Every function below applies the scalar one above lane by
// lane, with the same operations in the same order (so each lane's result is bit-identical to the
// scalar transform's), on Blackwell's paired FP32 instructions: one add, multiply or fused
// multiply-add for both lanes. Twiddles are the same for both lanes and are held broadcast.
struct cplx2 {
    float2 re, im;
};

__host__ __device__ __forceinline__ float2 add2(float2 a, float2 b)
{
#ifdef __CUDA_ARCH__
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}
// a - b as fma(b, -1, a): the same rounding as the subtraction (measured slightly faster than an
// add of the negated operand)
__host__ __device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
#ifdef __CUDA_ARCH__
    return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
#else
    return make_float2(a.x - b.x, a.y - b.y);
#endif
}
__host__ __device__ __forceinline__ float2 mul2(float2 a, float2 b)
{
#ifdef __CUDA_ARCH__
    return __fmul2_rn(a, b);
#else
    return make_float2(a.x * b.x, a.y * b.y);
#endif
}
__host__ __device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
#ifdef __CUDA_ARCH__
    return __ffma2_rn(a, b, c);
#else
    return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}

// A twiddle w broadcast to both lanes: (w.x, w.x), (w.y, w.y) and (-w.y, -w.y).
struct tw2 {
    float2 x, y, ny;
};
__host__ __device__ __forceinline__ tw2 make_tw2(cplx w)
{
    return {make_float2(w.x, w.x), make_float2(w.y, w.y), make_float2(-w.y, -w.y)};
}
// cmul(v, w) = {fma(v.x, w.x, -v.y w.y), fma(v.x, w.y, v.y w.x)} in both lanes.
__host__ __device__ __forceinline__ cplx2 cmul2(cplx2 v, tw2 w)
{
    return {fma2(v.re, w.x, mul2(v.im, w.ny)), fma2(v.re, w.y, mul2(v.im, w.x))};
}
__host__ __device__ __forceinline__ cplx2 cadd2(cplx2 a, cplx2 b) { return {add2(a.re, b.re), add2(a.im, b.im)}; }
__host__ __device__ __forceinline__ cplx2 csub2(cplx2 a, cplx2 b) { return {sub2(a.re, b.re), sub2(a.im, b.im)}; }

template <int SIGN>
__host__ __device__ __forceinline__ void dft4_2(cplx2& a, cplx2& b, cplx2& c, cplx2& d)
{
    // dft4 with t3 = mul_i<SIGN>(b - d) folded into the last two sums: for SIGN < 0,
    // t1 + t3 = (t1.re + u.im, t1.im - u.re) and t1 - t3 = (t1.re - u.im, t1.im + u.re), u = b - d.
    const cplx2 t0 = cadd2(a, c), t1 = csub2(a, c), t2 = cadd2(b, d), u = csub2(b, d);
    a = cadd2(t0, t2);
    c = csub2(t0, t2);
    if constexpr (SIGN < 0) {
        b = {add2(t1.re, u.im), sub2(t1.im, u.re)};
        d = {sub2(t1.re, u.im), add2(t1.im, u.re)};
    } else {
        b = {sub2(t1.re, u.im), add2(t1.im, u.re)};
        d = {add2(t1.re, u.im), sub2(t1.im, u.re)};
    }
}

template <int R, int SIGN>
__host__ __device__ __forceinline__ void dft_2(cplx2 (&v)[R])
{
    if constexpr (R == 2) {
        const cplx2 t = v[0];
        v[0] = cadd2(t, v[1]);
        v[1] = csub2(t, v[1]);
    } else if constexpr (R == 4) {
        dft4_2<SIGN>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        cplx2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft4_2<SIGN>(e[0], e[1], e[2], e[3]);
        dft4_2<SIGN>(o[0], o[1], o[2], o[3]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const cplx2 t = k == 0 ? o[0] : cmul2(o[k], make_tw2(w16<SIGN>(2 * k)));
            v[k] = cadd2(e[k], t);
            v[k + 4] = csub2(e[k], t);
        }
    } else {
        static_assert(R == 16, "radix");
        cplx2 y[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            cplx2 a = v[n2], b = v[4 + n2], c = v[8 + n2], d = v[12 + n2];
            dft4_2<SIGN>(a, b, c, d);
            y[0][n2] = a; y[1][n2] = b; y[2][n2] = c; y[3][n2] = d;
        }
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1)
#pragma unroll
            for (int n2 = 1; n2 < 4; ++n2) y[k1][n2] = cmul2(y[k1][n2], make_tw2(w16<SIGN>(n2 * k1)));
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            dft4_2<SIGN>(y[k1][0], y[k1][1], y[k1][2], y[k1][3]);
            v[k1] = y[k1][0];
            v[k1 + 4] = y[k1][1];
            v[k1 + 8] = y[k1][2];
            v[k1 + 12] = y[k1][3];
        }
    }
}

// Shared-memory index of the paired exchange (float2 arrays, 8 bytes per element): bits 0..3 of
// i are XORed with bits 4..7, and with `skew` = (row in block * N/16) mod 16 where several rows
// share a warp. Every store and gather pattern of the passes then gives the 16 lanes of each
// half-warp 16 different 8-byte bank pairs (checked on the CPU for N = 32 .. 8192).
__host__ __device__ __forceinline__ uint32_t spad2(uint32_t i, uint32_t skew) { return i ^ ((i >> 4) & 15u) ^ skew; }

// fft_pass on two transforms: the pass's twiddles are formed once and applied to both lanes.
template <int LOGN, int P, int SIGN>
__host__ __device__ __forceinline__ void fft_pass2(cplx2 (&x)[16], uint32_t tau, const cplx* __restrict__ tw,
                                                   float2* sre, float2* sim, uint32_t skew,
                                                   const BaseTwiddles<LOGN>& wb)
{
    constexpr int N = 1 << LOGN;
    constexpr int TPF = N / 16;
    constexpr int R = pass_radix(LOGN, P);
    constexpr int B = 16 / R;
    constexpr int NS_LOG = pass_ns_log(LOGN, P);
    constexpr int NS = 1 << NS_LOG;
    constexpr bool LAST = P == pass_count(LOGN) - 1;
    constexpr int TW_SHIFT = LOGN - NS_LOG - (R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1);
#pragma unroll
    for (int u = 0; u < B; ++u) {
        const uint32_t j = tau + u * TPF;
        const uint32_t k = j & (NS - 1);
        cplx2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = x[u + r * B];
        if constexpr (P > 0 && R == 16) {
            // Formed on scalar FP32, as in fft_pass, and broadcast where applied: a paired
            // instruction occupies both FP32 sub-pipes, so generating a broadcast twiddle on
            // paired lanes would cost three times the FP32 work (measured 0.309 -> 0.283 ms on
            // 16384 rows of 4096 samples).
            cplx p[16];
            p[1] = wb.w[P][0];
            p[4] = wb.w[P][1];
            if constexpr (SIGN > 0) p[1].y = -p[1].y, p[4].y = -p[4].y;
            p[2] = cmul(p[1], p[1]);
            p[3] = cmul(p[2], p[1]);
            p[8] = cmul(p[4], p[4]);
            p[12] = cmul(p[8], p[4]);
#pragma unroll
            for (int a4 = 4; a4 < 16; a4 += 4)
#pragma unroll
                for (int b = 1; b < 4; ++b) p[a4 + b] = cmul(p[a4], p[b]);
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul2(v[r], make_tw2(p[r]));
        } else if constexpr (P > 0) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                cplx w = tw[(r * k) << TW_SHIFT];
                if constexpr (SIGN > 0) w.y = -w.y;
                v[r] = cmul2(v[r], make_tw2(w));
            }
        }
        dft_2<R, SIGN>(v);
        if constexpr (LAST) {
#pragma unroll
            for (int r = 0; r < R; ++r) x[u + r * B] = v[r];
        } else {
            const uint32_t base = (j >> NS_LOG) * (NS * R) + k;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t pos = spad2(base + r * NS, skew);
                sre[pos] = v[r].re;
                sim[pos] = v[r].im;
            }
        }
    }
}

template <int LOGN>
__host__ __device__ __forceinline__ void fft_gather2(cplx2 (&x)[16], uint32_t tau, const float2* sre,
                                                     const float2* sim, uint32_t skew)
{
    constexpr int TPF = (1 << LOGN) / 16;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const uint32_t pos = spad2(tau + m * TPF, skew);
        x[m] = {sre[pos], sim[pos]};
    }
}

}  // namespace fft
}  // namespace cutb
