// Fused convert + channel reorder + transmit decode.
//
// Upstream this stage is three passes (cuda_toolkit/src/rf_processing/):
//   convert_to_f32        data_conversion/data_conversion_kernels.cuh:25-41
//                          out[t][c][s] = (float) raw[map[c]*R0 + t*S + s]
//   cublasSgemm decode     hadamard/hadamard_decoder.cpp:49-78
//                          dec[t'][c][s] = fl32(1/T) * sum_t H[t'][t] * out[t][c][s]
//   cudaMemcpy2D repack    rf_processor.cpp:143-146 (real -> .x of complex)
//
// Here it is one HBM pass: every element is read once and written once. The encoding
// matrix has Kronecker structure H = S_{T/B} (x) B (Sylvester doubling of a base of order
// B = 1, 12 or 20), so the T x T product is evaluated as a fast Walsh-Hadamard transform:
// T*log2(T) additions per column instead of T^2 multiply-adds. Integer input is
// accumulated in int32, which is exact, and scaled once by fl32(1/T); for T <= 512 every
// partial sum upstream is an integer below 2^24, so the result is bit-identical to the
// upstream FP32 GEMM whatever its summation order.
//
// Thread layout: a warp holds, for 32/L sample groups of V consecutive samples, the T
// transmits split as T = L * R: each lane keeps R transmits in registers (t = hi*R + r)
// and L lanes share a sample group. The R-point transform runs in registers, the L-point
// transform across lanes with __shfl_xor_sync. Loads are V-wide vectors along samples.
#include <type_traits>
#include <utility>

#include "common.cuh"
#include "stages.h"

namespace cutb {
namespace {

constexpr int kDecodeThreads = 256;

// Entry (i, j) of the order-12 / order-20 base matrix (see encoding.cpp:qr_base).
constexpr int base_sign(int order, int i, int j)
{
    if (order == 1 || i == 0 || j == 0) return 1;
    const int q = order - 1;
    const int a = i - 1, b = j - 1;
    auto chi = [q](int x) {
        x %= q;
        if (x == 0) return 0;
        for (int y = 1; y < q; ++y)
            if ((y * y) % q == x) return 1;
        return -1;
    };
    if (order == 12) return a == b ? -1 : chi(a + q - b);
    const int k = (a + b) % q;
    return k == 0 ? -1 : -chi(k);
}

template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>)
{
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f)
{
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// ---- vector loads (streaming: each raw element is read exactly once) -------------------
template <int V, class Acc>
__device__ __forceinline__ void load_vec(Acc (&d)[V], const int16_t* p, bool ok)
{
    if constexpr (V == 4) {
        int2 w = ok ? __ldcs(reinterpret_cast<const int2*>(p)) : make_int2(0, 0);
        d[0] = (int16_t)(w.x & 0xffff); d[1] = (int16_t)(w.x >> 16);
        d[2] = (int16_t)(w.y & 0xffff); d[3] = (int16_t)(w.y >> 16);
    } else if constexpr (V == 2) {
        int w = ok ? __ldcs(reinterpret_cast<const int*>(p)) : 0;
        d[0] = (int16_t)(w & 0xffff); d[1] = (int16_t)(w >> 16);
    } else {
        d[0] = ok ? (Acc)__ldcs(reinterpret_cast<const short*>(p)) : (Acc)0;
    }
}
template <int V, class Acc>
__device__ __forceinline__ void load_vec(Acc (&d)[V], const float* p, bool ok)
{
    if constexpr (V == 4) {
        float4 w = ok ? __ldcs(reinterpret_cast<const float4*>(p)) : make_float4(0, 0, 0, 0);
        d[0] = w.x; d[1] = w.y; d[2] = w.z; d[3] = w.w;
    } else if constexpr (V == 2) {
        float2 w = ok ? __ldcs(reinterpret_cast<const float2*>(p)) : make_float2(0, 0);
        d[0] = w.x; d[1] = w.y;
    } else {
        d[0] = ok ? __ldcs(p) : 0.f;
    }
}

// ---- vector stores: packed floats (OSTRIDE 1) or complex with zero imaginary part (2) ---
template <int V, int OSTRIDE>
__device__ __forceinline__ void store_vec(float* p, const float (&v)[V])
{
    if constexpr (OSTRIDE == 1) {
        if constexpr (V == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
        else if constexpr (V == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
        else *p = v[0];
    } else {
        if constexpr (V == 4) {
            reinterpret_cast<float4*>(p)[0] = make_float4(v[0], 0.f, v[1], 0.f);
            reinterpret_cast<float4*>(p)[1] = make_float4(v[2], 0.f, v[3], 0.f);
        } else if constexpr (V == 2) {
            *reinterpret_cast<float4*>(p) = make_float4(v[0], 0.f, v[1], 0.f);
        } else {
            *reinterpret_cast<float2*>(p) = make_float2(v[0], 0.f);
        }
    }
}

// In-register part of the transform: dense base matrix on each block of BASE transmits,
// then a Walsh-Hadamard butterfly over the R/BASE blocks.
template <int R, int BASE, int V, class Acc>
__device__ __forceinline__ void register_transform(Acc (&x)[R][V])
{
    constexpr int NB = R / BASE;
    if constexpr (BASE > 1) {
#pragma unroll
        for (int blk = 0; blk < NB; ++blk)
#pragma unroll
            for (int v = 0; v < V; ++v) {
                Acc in[BASE];
#pragma unroll
                for (int b = 0; b < BASE; ++b) in[b] = x[blk * BASE + b][v];
                static_for<BASE>([&](auto bo) {
                    Acc acc = 0;
                    static_for<BASE>([&](auto bi) {
                        constexpr int sgn = base_sign(BASE, decltype(bo)::value, decltype(bi)::value);
                        if constexpr (sgn > 0) acc += in[decltype(bi)::value];
                        else acc -= in[decltype(bi)::value];
                    });
                    x[blk * BASE + decltype(bo)::value][v] = acc;
                });
            }
    }
#pragma unroll
    for (int h = 1; h < NB; h <<= 1)
#pragma unroll
        for (int blk = 0; blk < NB; ++blk)
            if (!(blk & h))
#pragma unroll
                for (int b = 0; b < BASE; ++b)
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        const Acc p = x[blk * BASE + b][v], q = x[(blk + h) * BASE + b][v];
                        x[blk * BASE + b][v] = p + q;
                        x[(blk + h) * BASE + b][v] = p - q;
                    }
}

template <int R, int BASE, int V, class TIn, int OSTRIDE>
__global__ void __launch_bounds__(kDecodeThreads)
decode_kernel(const TIn* __restrict__ raw, float* __restrict__ out, DecodeArgs a)
{
    using Acc = std::conditional_t<std::is_same_v<TIn, int16_t>, int, float>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int hi = lane / a.G, grp = lane % a.G;
    const uint32_t c = blockIdx.y;
    const int64_t s = (int64_t)blockIdx.x * (kDecodeThreads / 32) * a.G * V + (int64_t)(warp * a.G + grp) * V;
    const bool active = s < (int64_t)a.S;
    const TIn* src = raw + (uint64_t)__ldg(&a.map[c]) * a.R0 + (active ? s : 0);

    Acc x[R][V];
#pragma unroll
    for (int r = 0; r < R; ++r) load_vec<V>(x[r], src + (uint64_t)(hi * R + r) * a.S, active);

    register_transform<R, BASE, V>(x);

    // Lane part of the Walsh-Hadamard transform: butterflies between lanes whose
    // transmit-block index `hi` differs in one bit.
    for (uint32_t m = 1; m < a.L; m <<= 1) {
        const bool upper = hi & m;
        const int delta = m * a.G;
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const Acc o = __shfl_xor_sync(0xffffffffu, x[r][v], delta);
                x[r][v] = upper ? o - x[r][v] : x[r][v] + o;
            }
    }
    if (!active) return;

#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t row = __ldg(&a.out_row[hi * R + r]);
        float v[V];
#pragma unroll
        for (int k = 0; k < V; ++k) v[k] = __fmul_rn(a.alpha, (float)x[r][k]);
        store_vec<V, OSTRIDE>(out + (((uint64_t)row * a.C + c) * a.S + s) * OSTRIDE, v);
    }
}

// decode == NONE: plain convert + reorder (data_conversion_kernels.cuh:25-41).
template <int V, class TIn, int OSTRIDE>
__global__ void __launch_bounds__(kDecodeThreads)
convert_kernel(const TIn* __restrict__ raw, float* __restrict__ out, DecodeArgs a)
{
    const int64_t s = ((int64_t)blockIdx.x * kDecodeThreads + threadIdx.x) * V;
    const uint32_t c = blockIdx.y, t = blockIdx.z;
    if (s >= (int64_t)a.S) return;
    float x[V];
    load_vec<V>(x, raw + (uint64_t)__ldg(&a.map[c]) * a.R0 + (uint64_t)t * a.S + s, true);
    store_vec<V, OSTRIDE>(out + (((uint64_t)t * a.C + c) * a.S + s) * OSTRIDE, x);
}

template <int R, int BASE, int V, class TIn, int OSTRIDE>
cudaError_t launch_decode_t(const void* raw, float* out, const DecodeArgs& a, cudaStream_t st)
{
    const uint32_t samples_per_block = (kDecodeThreads / 32) * a.G * V;
    dim3 grid(div_up(a.S, samples_per_block), a.C);
    decode_kernel<R, BASE, V, TIn, OSTRIDE><<<grid, kDecodeThreads, 0, st>>>((const TIn*)raw, out, a);
    return cudaGetLastError();
}

template <int R, int BASE, class TIn, int OSTRIDE>
cudaError_t launch_decode_v(const void* raw, float* out, const DecodeArgs& a, bool wide, cudaStream_t st)
{
    constexpr int VW = R <= 16 ? 4 : 2;
    return wide ? launch_decode_t<R, BASE, VW, TIn, OSTRIDE>(raw, out, a, st)
                : launch_decode_t<R, BASE, 1, TIn, OSTRIDE>(raw, out, a, st);
}

template <class TIn, int OSTRIDE>
cudaError_t launch_decode_rb(int R, int base, const void* raw, float* out, const DecodeArgs& a, bool wide,
                             cudaStream_t st)
{
#define CUTB_DECODE_CASE(RR, BB) \
    if (R == RR && base == BB) return launch_decode_v<RR, BB, TIn, OSTRIDE>(raw, out, a, wide, st);
    CUTB_DECODE_CASE(1, 1)
    CUTB_DECODE_CASE(2, 1)
    CUTB_DECODE_CASE(4, 1)
    CUTB_DECODE_CASE(8, 1)
    CUTB_DECODE_CASE(16, 1)
    CUTB_DECODE_CASE(32, 1)
    CUTB_DECODE_CASE(12, 12)
    CUTB_DECODE_CASE(24, 12)
    CUTB_DECODE_CASE(20, 20)
#undef CUTB_DECODE_CASE
    return cudaErrorInvalidValue;
}

template <class TIn, int OSTRIDE>
cudaError_t launch_convert(const void* raw, float* out, const DecodeArgs& a, bool wide, cudaStream_t st)
{
    if (wide) {
        dim3 grid(div_up(a.S, kDecodeThreads * 4u), a.C, a.T);
        convert_kernel<4, TIn, OSTRIDE><<<grid, kDecodeThreads, 0, st>>>((const TIn*)raw, out, a);
    } else {
        dim3 grid(div_up(a.S, (uint32_t)kDecodeThreads), a.C, a.T);
        convert_kernel<1, TIn, OSTRIDE><<<grid, kDecodeThreads, 0, st>>>((const TIn*)raw, out, a);
    }
    return cudaGetLastError();
}

}  // namespace

// Splits T = L * R (lanes x registers) for the kernel. R holds the base factor.
bool plan_decode_split(unsigned T, unsigned base, unsigned& R, unsigned& L)
{
    const unsigned p = T / base;  // power of two
    if (base == 1) {
        if (p <= 16) { R = p; L = 1; }
        else if (p <= 512) { R = 16; L = p / 16; }
        else { R = 32; L = p / 32; }
    } else {
        if (p <= 32) { R = base; L = p; }
        else { R = base * (p / 32); L = 32; }
    }
    return (R == 1 || R == 2 || R == 4 || R == 8 || R == 16 || R == 32 || (base == 12 && (R == 12 || R == 24)) ||
            (base == 20 && R == 20)) && L <= 32;
}

bool launch_decode(const DecodeSetup& d, const void* raw, int data_type, float* out, unsigned out_stride,
                   cudaStream_t st)
{
    DecodeArgs a = d.args;
    const size_t esize = data_type == TYPE_I16 ? 2 : 4;
    cudaError_t err;
    if (d.encoding == NONE) {
        const bool wide = (a.S % 4 == 0) && (a.R0 % 4 == 0) && ((uintptr_t)raw % (4 * esize) == 0) &&
                          ((uintptr_t)out % 16 == 0);
        if (data_type == TYPE_I16)
            err = out_stride == 1 ? launch_convert<int16_t, 1>(raw, out, a, wide, st)
                                  : launch_convert<int16_t, 2>(raw, out, a, wide, st);
        else
            err = out_stride == 1 ? launch_convert<float, 1>(raw, out, a, wide, st)
                                  : launch_convert<float, 2>(raw, out, a, wide, st);
    } else {
        const unsigned vw = d.R <= 16 ? 4 : 2;
        const bool wide = (a.S % vw == 0) && (a.R0 % vw == 0) && ((uintptr_t)raw % (vw * esize) == 0) &&
                          ((uintptr_t)out % 16 == 0);
        if (data_type == TYPE_I16)
            err = out_stride == 1 ? launch_decode_rb<int16_t, 1>(d.R, d.base, raw, out, a, wide, st)
                                  : launch_decode_rb<int16_t, 2>(d.R, d.base, raw, out, a, wide, st);
        else
            err = out_stride == 1 ? launch_decode_rb<float, 1>(d.R, d.base, raw, out, a, wide, st)
                                  : launch_decode_rb<float, 2>(d.R, d.base, raw, out, a, wide, st);
    }
    CUTB_CUDA_OK(err);
    return true;
}

}  // namespace cutb
