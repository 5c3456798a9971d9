// Match-filtered analytic signal, one shared-memory FFT kernel.
//
// Upstream (cuda_toolkit/src/rf_processing/rf_ffts/) runs, per frame: a cudaMemset of the
// output, a strided cuFFT R2C, a mask/scale/filter kernel (hilbert_kernels.cuh:17-40)
// and an in-place cuFFT C2C inverse (hilbert_handler.cu:132-155). Per row x of N samples:
//   Y[k] = DFT(x)[k] * w_k * F[k] for k <= N/2, 0 above; w_0 = 0.75/N, w_k = 1.5/N
//   (the Nyquist bin keeps 1.5/N); F = DFT_N(zero-padded taps), no time reversal
//   (hilbert_handler.cu:55-78); iq = unnormalised inverse DFT of Y.
//
// Here each CTA transforms two rows a, b at once in shared memory and writes the IQ of
// both exactly once. With G[k] = w_k F[k] (k <= N/2, else 0) split into its Hermitian
// parts Ge[k] = (G[k] + conj G[-k]) / 2 and Go[k] = (G[k] - conj G[-k]) / (2i), and
// Z = DFT(x_a + i x_b):
//   IDFT(Z Ge) = Re(iq_a) + i Re(iq_b),  IDFT(Z Go) = Im(iq_a) + i Im(iq_b),
// because x_a, x_b are real (their spectra are Hermitian) and so are Ge, Go. That is 1.5
// complex FFTs per row instead of 2, with no separation step. The two inverse transforms run
// together on paired FP32 lanes (lane 0: Z Ge, lane 1: Z Go; one instruction for both), so that
// element n of the paired result is (Re iq_a, Im iq_a), (Re iq_b, Im iq_b): the output samples
// themselves. Ge, Go and the twiddles are precomputed in FP64 on the host and stored as FP32
// tables. A thread reads two twiddles per radix-16 pass once, at the start (all transforms share
// them), and forms the pass's 15 twiddles as products of those: a per-butterfly table read per
// twiddle had kept the load/store unit saturated (0.73 ms -> 0.31 ms on 16384 rows of 4096
// samples); the paired inverse then took the kernel from 3 to 2 transforms' worth of
// instructions per row pair.
#include <atomic>
#include <cmath>
#include <complex>
#include <vector>

#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include "common.cuh"
#include "fft_core.cuh"
#include "stages.h"

namespace cutb {
namespace {

using fft::cplx;

template <int LOGN>
constexpr int hilbert_fft_per_block() { return (1 << LOGN) / 16 >= 128 ? 1 : 128 / ((1 << LOGN) / 16); }

template <int LOGN, int SIGN, int P = 0>
__device__ __forceinline__ void run_fft(cplx (&x)[16], uint32_t tau, const cplx* tw, float* sre, float* sim,
                                        const fft::BaseTwiddles<LOGN>& wb)
{
    constexpr int NP = fft::pass_count(LOGN);
    if constexpr (P < NP) {
        fft::fft_pass<LOGN, P, SIGN>(x, tau, tw, sre, sim, wb);
        if constexpr (P < NP - 1) {
            __syncthreads();
            fft::fft_gather<LOGN>(x, tau, sre, sim);
            __syncthreads();
        }
        run_fft<LOGN, SIGN, P + 1>(x, tau, tw, sre, sim, wb);
    }
}

// Two transforms at once on paired FP32 lanes (fft::fft_pass2), exchanging through float2 arrays.
template <int LOGN, int SIGN, int P = 0>
__device__ __forceinline__ void run_fft2(fft::cplx2 (&x)[16], uint32_t tau, const cplx* tw, float2* sre, float2* sim,
                                         uint32_t skew, const fft::BaseTwiddles<LOGN>& wb)
{
    constexpr int NP = fft::pass_count(LOGN);
    if constexpr (P < NP) {
        fft::fft_pass2<LOGN, P, SIGN>(x, tau, tw, sre, sim, skew, wb);
        if constexpr (P < NP - 1) {
            __syncthreads();
            fft::fft_gather2<LOGN>(x, tau, sre, sim, skew);
            __syncthreads();
        }
        run_fft2<LOGN, SIGN, P + 1>(x, tau, tw, sre, sim, skew, wb);
    }
}

// Writes output sample i (streaming: it is not read again by this kernel).
__device__ __forceinline__ void store_iq(float2* out, uint64_t i, float re, float im)
{
    __stcs(out + i, make_float2(re, im));
}
__device__ __forceinline__ void store_iq(__nv_bfloat162* out, uint64_t i, float re, float im)
{
    out[i] = __floats2bfloat162_rn(re, im);
}

template <int LOGN>
constexpr int hilbert_threads() { return hilbert_fft_per_block<LOGN>() * (1 << LOGN) / 16; }
template <int LOGN>
constexpr int hilbert_min_blocks() { return hilbert_threads<LOGN>() <= 256 ? 2 : 1; }
// At 2^14 points the pair form needs 256 KiB of shared memory (the paired exchange buffers),
// above the 227 KiB a CTA may have; one row per CTA needs half of that.
template <int LOGN>
constexpr bool hilbert_single_row() { return LOGN >= 14; }
template <int LOGN>
constexpr size_t hilbert_smem_bytes()
{
    constexpr size_t N = size_t(1) << LOGN;
    return hilbert_fft_per_block<LOGN>() *
           (hilbert_single_row<LOGN>() ? 2 * fft::spad_size(N) * sizeof(float) : 2 * N * sizeof(float2));
}
static_assert(hilbert_smem_bytes<14>() <= 227 * 1024 && hilbert_smem_bytes<13>() <= 227 * 1024, "shared memory");

// PAD: rows of a.n samples (any length) transformed at the power-of-two length N >= 2 a.n - 1 with
// zeros appended; the spectral tables then hold the weight of the equivalent length-N circular
// convolution (build_hilbert_tables), and only the first a.n outputs are stored.
template <int LOGN, class OutT, bool PAD>
__global__ void __launch_bounds__(hilbert_threads<LOGN>(), hilbert_min_blocks<LOGN>())
hilbert_kernel(const float* __restrict__ in, OutT* __restrict__ out, HilbertArgs a)
{
    constexpr uint32_t N = 1u << LOGN;
    constexpr uint32_t TPF = N / 16;
    constexpr uint32_t FPB = hilbert_fft_per_block<LOGN>();
    constexpr uint32_t PN = fft::spad_size(N);
    constexpr bool SINGLE = hilbert_single_row<LOGN>();
    extern __shared__ float smem[];

    const uint32_t L = PAD ? a.n : N;  // samples per row in memory
    const uint32_t grp = threadIdx.x / TPF, tau = threadIdx.x % TPF;
    const uint64_t pair = (uint64_t)blockIdx.x * FPB + grp;
    const uint64_t ra = SINGLE ? (uint64_t)blockIdx.x : 2 * pair, rb = ra + 1;
    const bool has_a = ra < a.rows, has_b = !SINGLE && rb < a.rows;
    // Exchange arrays of the scalar transforms: the start of this row's region (the paired inverse
    // reuses the whole region as two float2 arrays).
    float* sre = smem + grp * (SINGLE ? 2 * PN : 4 * N);
    float* sim = sre + PN;
    const cplx* tw = reinterpret_cast<const cplx*>(a.twiddle);

    fft::BaseTwiddles<LOGN> wb;
    fft::load_base_twiddles<LOGN>(wb, tau, tw);
    cplx z[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const uint64_t n = tau + m * TPF;
        const bool in_row = !PAD || n < L;
        z[m].x = has_a && in_row ? __ldcs(in + (ra * L + n) * a.in_stride) : 0.f;
        z[m].y = has_b && in_row ? __ldcs(in + (rb * L + n) * a.in_stride) : 0.f;
    }
    run_fft<LOGN, -1>(z, tau, tw, sre, sim, wb);  // z[m] = Z[tau + m*TPF]

    // Spectral weight per bin k: (Ge.re, Go.re, Ge.im, Go.im).
    const float4* wt = reinterpret_cast<const float4*>(a.weight);
    if constexpr (SINGLE) {
        // One real row: iq = IDFT(X G) with G = Ge + i Go.
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const uint32_t k = tau + m * TPF;
            const float4 w = __ldg(wt + k);
            z[m] = fft::cmul(z[m], cplx{w.x - w.w, w.z + w.y});
        }
        run_fft<LOGN, +1>(z, tau, tw, sre, sim, wb);
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const uint64_t n = tau + m * TPF;
            if (has_a && (!PAD || n < L)) store_iq(out, ra * L + n, z[m].x, z[m].y);
        }
    } else {
        // Lane 0: Z Ge, lane 1: Z Go, each cmul(z, weight) = {fma(z.x, w.x, -z.y w.y), fma(z.x, w.y, z.y w.x)};
        // the paired inverse then leaves (Re iq_a, Im iq_a) in .re and (Re iq_b, Im iq_b) in .im.
        fft::cplx2 y[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const uint32_t k = tau + m * TPF;
            const float4 w = __ldg(wt + k);
            const float2 zx = make_float2(z[m].x, z[m].x), zy = make_float2(z[m].y, z[m].y);
            y[m].re = fft::fma2(zx, make_float2(w.x, w.y), fft::mul2(zy, make_float2(-w.z, -w.w)));
            y[m].im = fft::fma2(zx, make_float2(w.z, w.w), fft::mul2(zy, make_float2(w.x, w.y)));
        }
        // The forward transform's last shared-memory reads ended at a barrier, so the paired
        // buffers (which overlay its arrays) are free.
        float2* s2re = reinterpret_cast<float2*>(smem) + grp * 2 * N;
        const uint32_t skew = (grp * TPF) & 15u;
        run_fft2<LOGN, +1>(y, tau, tw, s2re, s2re + N, skew, wb);
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const uint64_t n = tau + m * TPF;
            if (PAD && n >= L) continue;
            if (has_a) store_iq(out, ra * L + n, y[m].re.x, y[m].re.y);
            if (has_b) store_iq(out, rb * L + n, y[m].im.x, y[m].im.y);
        }
    }
}

template <int LOGN, class OutT, bool PAD>
bool launch_hilbert_t(const float* in, void* out, const HilbertArgs& a, cudaStream_t st)
{
    constexpr uint32_t FPB = hilbert_fft_per_block<LOGN>();
    constexpr size_t smem = hilbert_smem_bytes<LOGN>();
    auto kern = hilbert_kernel<LOGN, OutT, PAD>;
    static std::atomic<uint64_t> smem_set{0};
    if (!set_smem_limit(kern, smem, smem_set)) return false;
    const uint64_t units = hilbert_single_row<LOGN>() ? a.rows : (a.rows + 1) / 2;  // rows or row pairs
    const uint64_t blocks = div_up(units, (uint64_t)FPB);
    CUTB_REQUIRE(blocks <= 0x7fffffffull, CUTB_ERR_INVALID_ARGUMENT, "Too many rows for one launch.");
    kern<<<(unsigned)blocks, hilbert_threads<LOGN>(), smem, st>>>(in, (OutT*)out, a);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

// ---- Rows longer than one CTA holds: a thread-block cluster per row --------------------------
// A CTA's shared memory holds the exchange arrays of 2^14 points (2 x 64 KiB). A row of N = 2^15 ..
// 2^17 points is transformed by a cluster of R = N / 2^14 CTAs of 1024 threads: CTA r runs threads
// tau = 1024 r .. 1024 r + 1023 of the N/16-thread Stockham transform (the same passes as the
// one-CTA kernels) and holds positions r 2^14 .. (r + 1) 2^14 - 1 of the exchange arrays; the passes
// store to and gather from the owning CTA through distributed shared memory, and cluster barriers
// separate the phases. One real row per cluster: iq = IDFT(X G) with G = Ge + i Go.
namespace cg = cooperative_groups;
constexpr int kSliceLog = 14;                        // exchange positions per CTA: 2^14
constexpr uint32_t kSlice = 1u << kSliceLog;
constexpr int kClusterThreads = (int)(kSlice / 16);  // 1024

// The exchange arrays spread over the cluster: position pos lives in CTA pos >> 14 at offset
// pos & (2^14 - 1) of its `re` / `im` arrays (the swizzle of fft::spad keeps a position in its slice).
// Addresses stay 32-bit: this CTA's shared-memory address of the offset is mapped to the owning
// CTA's in the cluster window (mapa), and the access goes to that window directly.
__device__ __forceinline__ uint32_t cluster_address(uint32_t local, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}
struct ClusterExchange {
    uint32_t re;  // shared-memory addresses of this CTA's arrays (the same offsets in every CTA)
    uint32_t im;
    __device__ __forceinline__ void store(uint32_t pos, cplx v) const
    {
        const uint32_t rank = pos >> kSliceLog, off = (pos & (kSlice - 1)) * 4u;
        asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(cluster_address(re + off, rank)), "f"(v.x) : "memory");
        asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(cluster_address(im + off, rank)), "f"(v.y) : "memory");
    }
    __device__ __forceinline__ cplx load(uint32_t pos) const
    {
        const uint32_t rank = pos >> kSliceLog, off = (pos & (kSlice - 1)) * 4u;
        cplx v;
        asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v.x) : "r"(cluster_address(re + off, rank)) : "memory");
        asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v.y) : "r"(cluster_address(im + off, rank)) : "memory");
        return v;
    }
};

// The cluster kernel runs at 64 registers a thread: each pass loads its two base twiddles (w^k and
// w^(4k), read through the cache) just before it instead of holding every pass's for the kernel.
template <int LOGN, int SIGN, int P = 0>
__device__ __forceinline__ void run_fft_cluster(cplx (&x)[16], uint32_t tau, const cplx* tw, const ClusterExchange& ex)
{
    constexpr int NP = fft::pass_count(LOGN);
    if constexpr (P < NP) {
        fft::BaseTwiddles<LOGN> wb;
        if constexpr (P > 0 && fft::pass_radix(LOGN, P) == 16) {
            constexpr int sh = LOGN - fft::pass_ns_log(LOGN, P) - 4;
            const uint32_t k = tau & ((1u << fft::pass_ns_log(LOGN, P)) - 1);
            wb.w[P][0] = tw[k << sh];
            wb.w[P][1] = tw[(4 * k) << sh];
        }
        fft::fft_pass_ex<LOGN, P, SIGN>(x, tau, tw, ex, wb);
        if constexpr (P < NP - 1) {
            cg::this_cluster().sync();  // every store of the pass is visible cluster-wide
            fft::fft_gather_ex<LOGN>(x, tau, ex);
            cg::this_cluster().sync();  // every gather is done before the next pass stores
        }
        run_fft_cluster<LOGN, SIGN, P + 1>(x, tau, tw, ex);
    }
}

template <int LOGN, class OutT, bool PAD>
__global__ void __launch_bounds__(kClusterThreads, 1)
hilbert_cluster_kernel(const float* __restrict__ in, OutT* __restrict__ out, HilbertArgs a)
{
    constexpr uint32_t N = 1u << LOGN;
    constexpr uint32_t TPF = N / 16;
    constexpr uint32_t R = N >> kSliceLog;
    static_assert(R >= 2 && R <= 8, "clusters of 2 .. 8 CTAs");
    extern __shared__ float smem[];
    cg::cluster_group cl = cg::this_cluster();
    const uint32_t rank = cl.block_rank();
    const uint32_t tau = rank * kClusterThreads + threadIdx.x;
    const uint64_t row = blockIdx.x / R;
    const uint32_t L = PAD ? a.n : N;
    const bool has_row = row < a.rows;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(smem);
    const ClusterExchange ex{base, base + kSlice * 4u};
    const cplx* tw = reinterpret_cast<const cplx*>(a.twiddle);
    cplx z[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const uint64_t n = tau + m * TPF;
        z[m].x = has_row && (!PAD || n < L) ? __ldcs(in + (row * L + n) * a.in_stride) : 0.f;
        z[m].y = 0.f;
    }
    cl.sync();  // every CTA of the cluster runs before any shared memory of another is written
    run_fft_cluster<LOGN, -1>(z, tau, tw, ex);
    const float4* wt = reinterpret_cast<const float4*>(a.weight);
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const float4 w = __ldg(wt + tau + m * TPF);
        z[m] = fft::cmul(z[m], cplx{w.x - w.w, w.z + w.y});
    }
    run_fft_cluster<LOGN, +1>(z, tau, tw, ex);
    // The last shared-memory accesses ended at a cluster barrier, so no CTA leaves while another
    // still reads its arrays.
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const uint64_t n = tau + m * TPF;
        if (has_row && (!PAD || n < L)) store_iq(out, row * L + n, z[m].x, z[m].y);
    }
}

template <int LOGN, class OutT, bool PAD>
bool launch_hilbert_cluster(const float* in, void* out, const HilbertArgs& a, cudaStream_t st)
{
    constexpr unsigned R = 1u << (LOGN - kSliceLog);
    constexpr size_t smem = 2 * kSlice * sizeof(float);
    auto kern = hilbert_cluster_kernel<LOGN, OutT, PAD>;
    static std::atomic<uint64_t> smem_set{0};
    if (!set_smem_limit(kern, smem, smem_set)) return false;
    CUTB_REQUIRE(a.rows * R <= 0x7fffffffull, CUTB_ERR_INVALID_ARGUMENT, "Too many rows for one launch.");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(a.rows * R));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = R;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUTB_CUDA_OK(cudaLaunchKernelEx(&cfg, kern, in, (OutT*)out, a));
    return true;
}

template <class OutT, bool PAD>
bool launch_hilbert_o(const float* in, void* out, const HilbertArgs& a, cudaStream_t st)
{
    switch (a.log_n) {
        case 4: return launch_hilbert_t<4, OutT, PAD>(in, out, a, st);
        case 5: return launch_hilbert_t<5, OutT, PAD>(in, out, a, st);
        case 6: return launch_hilbert_t<6, OutT, PAD>(in, out, a, st);
        case 7: return launch_hilbert_t<7, OutT, PAD>(in, out, a, st);
        case 8: return launch_hilbert_t<8, OutT, PAD>(in, out, a, st);
        case 9: return launch_hilbert_t<9, OutT, PAD>(in, out, a, st);
        case 10: return launch_hilbert_t<10, OutT, PAD>(in, out, a, st);
        case 11: return launch_hilbert_t<11, OutT, PAD>(in, out, a, st);
        case 12: return launch_hilbert_t<12, OutT, PAD>(in, out, a, st);
        case 13: return launch_hilbert_t<13, OutT, PAD>(in, out, a, st);
        case 14: return launch_hilbert_t<14, OutT, PAD>(in, out, a, st);
        case 15: return launch_hilbert_cluster<15, OutT, PAD>(in, out, a, st);
        case 16: return launch_hilbert_cluster<16, OutT, PAD>(in, out, a, st);
        case 17: return launch_hilbert_cluster<17, OutT, PAD>(in, out, a, st);
        default: break;
    }
    set_error(CUTB_ERR_UNSUPPORTED, "Hilbert transform length 2^%u not supported.", a.log_n);
    return false;
}

using cd = std::complex<double>;

// In-place FP64 radix-2 FFT (power-of-two length), sum_j a[j] exp(sign 2 pi i j k / n); the
// twiddles come from exact index arithmetic.
void fft_fp64(std::vector<cd>& a, int sign)
{
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    const double two_pi = 6.283185307179586476925286766559;
    std::vector<cd> w(n / 2);
    for (size_t k = 0; k < n / 2; ++k) w[k] = std::polar(1.0, sign * two_pi * (double)k / (double)n);
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len / 2, step = n / len;
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < half; ++k) {
                const cd u = a[i + k], v = a[i + k + half] * w[k * step];
                a[i + k] = u + v;
                a[i + k + half] = u - v;
            }
    }
}

}  // namespace

unsigned hilbert_fft_length(unsigned n)
{
    if (n == 0) return 0;
    if (is_pow2(n) && n >= 16) return n <= kMaxHilbertLength ? n : 0;
    unsigned m = 16;
    while (m < 2 * (uint64_t)n - 1) m <<= 1;
    return m <= kMaxHilbertLength ? m : 0;
}

bool hilbert_supported_length(unsigned n) { return hilbert_fft_length(n) != 0; }

// Host tables, all computed in double and rounded once to float: twiddles exp(-2*pi*i*m/M) of the
// FFT length M = hilbert_fft_length(n) and the Hermitian parts of the spectral weight, interleaved
// per bin as (Ge.re, Go.re, Ge.im, Go.im) so that one 16-byte load gives both paired lanes.
//
// Power-of-two rows (M = n): the weight is G = w * F itself.
//
// Other lengths: upstream's cuFFT transforms at the row length n itself. The filter-and-mask step
// is a length-n circular convolution, iq[j] = sum_m x[m] g[(j - m) mod n], with the kernel
// g[j] = sum_k G[k] exp(+2 pi i k j / n) = (taps circularly convolved with mk)[j], where
// mk[j] = sum_{k <= n/2} w_k exp(2 pi i k j / n) has the closed form
//   mk[0] = (0.75 + 1.5 K) / n,  mk[j] = (0.75 + 1.5 e^{i pi j (K+1)/n} sin(pi j K / n) / sin(pi j / n)) / n
// (K = floor(n/2), a geometric series). The same convolution of the zero-padded row follows from a
// length-M circular convolution with h, h[j] = g[j] and h[M - j] = g[n - j] (the negative lags),
// which do not overlap when M >= 2n - 1; its spectral weight is DFT_M(h) / M (the kernel's inverse
// transform is unnormalised). Only outputs 0..n-1 are kept.
bool build_hilbert_tables(unsigned n, const float* taps, unsigned ntaps, std::vector<float>& twiddle,
                          std::vector<float>& weight)
{
    const unsigned M = hilbert_fft_length(n);
    CUTB_REQUIRE(M != 0, CUTB_ERR_UNSUPPORTED,
                 "Sample count %u not supported by the FFT (powers of two up to %u, other lengths up to %u).", n,
                 kMaxHilbertLength, kMaxHilbertLength / 2);
    CUTB_REQUIRE(ntaps <= n, CUTB_ERR_INVALID_ARGUMENT, "Match filter longer (%u) than the sample count (%u).", ntaps,
                 n);
    const double two_pi = 6.283185307179586476925286766559, pi = two_pi / 2;
    twiddle.resize(2 * (size_t)M);
    std::vector<cd> root(M);
    for (unsigned m = 0; m < M; ++m) {
        root[m] = std::polar(1.0, -two_pi * (double)m / (double)M);
        twiddle[2 * m] = (float)root[m].real();
        twiddle[2 * m + 1] = (float)root[m].imag();
    }
    std::vector<cd> g(M, cd(0, 0));
    if (M == n) {
        const unsigned half = n / 2;
        for (unsigned k = 0; k <= half; ++k) {
            cd f(1.0, 0.0);
            if (ntaps) {
                f = 0;
                for (unsigned t = 0; t < ntaps; ++t) f += (double)taps[t] * root[(uint64_t)k * t % n];
            }
            g[k] = ((k == 0 ? 0.75 : 1.5) / (double)n) * f;
        }
    } else {
        const uint64_t K = n / 2, two_n = 2 * (uint64_t)n;
        std::vector<cd> mk(n), gt(n, cd(0, 0));
        mk[0] = (0.75 + 1.5 * (double)K) / (double)n;
        for (uint64_t j = 1; j < n; ++j) {
            const double ratio = std::sin(pi * (double)(j * K % two_n) / n) / std::sin(pi * (double)j / n);
            mk[j] = (0.75 + 1.5 * std::polar(ratio, pi * (double)(j * (K + 1) % two_n) / n)) / (double)n;
        }
        if (ntaps == 0) gt = mk;
        for (unsigned t = 0; t < ntaps; ++t)
            for (unsigned j = 0; j < n; ++j) gt[j] += (double)taps[t] * mk[(j + n - t) % n];
        for (unsigned j = 0; j < n; ++j) g[j] = gt[j];
        for (unsigned j = 1; j < n; ++j) g[M - j] = gt[n - j];
        fft_fp64(g, -1);
        for (auto& v : g) v /= (double)M;
    }
    weight.resize(4 * (size_t)M);
    for (unsigned k = 0; k < M; ++k) {
        const cd gm = std::conj(g[(M - k) % M]);
        const cd e = 0.5 * (g[k] + gm);
        const cd o = (g[k] - gm) / cd(0.0, 2.0);
        weight[4 * (size_t)k] = (float)e.real();
        weight[4 * (size_t)k + 1] = (float)o.real();
        weight[4 * (size_t)k + 2] = (float)e.imag();
        weight[4 * (size_t)k + 3] = (float)o.imag();
    }
    return true;
}

bool launch_hilbert(const HilbertArgs& a, const float* in, void* out, bool bf16, cudaStream_t st)
{
    CUTB_REQUIRE(a.n >= 1 && hilbert_fft_length(a.n) == (1u << a.log_n), CUTB_ERR_INVALID_ARGUMENT,
                 "Hilbert rows of %u samples do not match the transform length 2^%u.", a.n, a.log_n);
    const bool pad = a.n != (1u << a.log_n);
    if (pad) return bf16 ? launch_hilbert_o<__nv_bfloat162, true>(in, out, a, st)
                         : launch_hilbert_o<float2, true>(in, out, a, st);
    return bf16 ? launch_hilbert_o<__nv_bfloat162, false>(in, out, a, st) : launch_hilbert_o<float2, false>(in, out, a, st);
}

}  // namespace cutb
