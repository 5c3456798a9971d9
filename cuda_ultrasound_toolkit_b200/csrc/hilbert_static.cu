// cutb_hilbert_static: the match-filtered analytic signal without any device allocation.
//
// Who needs it: applications that own the GPU's memory budget themselves, such as an
// acquisition loop that reserves every buffer it will use before scanning starts, or a
// plugin host that only lends the library its own buffers. They cannot let a library call
// cudaMalloc/cudaFree: those calls can stall on device-wide synchronisation in the middle of
// a frame, and they fail once the host has reserved the memory. cutb_hilbert needs a plan,
// and creating a plan allocates the twiddle and spectral-weight tables that the kernel reads.
// This entry point keeps those tables in a fixed file-scope device array instead, so every
// byte it touches is either the caller's input/output or that array.
//
// The array holds the tables of one transform of up to kStaticMaxSamples points (384 KiB): rows
// of up to 16384 samples when the count is a power of two, up to 8192 otherwise (those run as a
// zero-padded transform of at least twice the length). Every GPU that loads the library keeps the
// array until the process exits. Each call
// rewrites all the tables it needs, on the caller's stream, before the kernel reads them, so
// nothing in the array has to start at zero. All calls share the array: calls that overlap
// on the GPU (on different streams, or issued from several host threads) race on it and must
// be serialised by the caller.
#include <mutex>
#include <vector>

#include "common.cuh"
#include "stages.h"

namespace cutb {
namespace {

constexpr unsigned kStaticMaxSamples = 16384;
constexpr int kMaxDevices = 64;

// twiddle (kStaticMaxSamples complex values) | spectral weight (kStaticMaxSamples x 4 floats).
static __device__ __align__(256) float g_hilbert_tables[3 * 2 * kStaticMaxSamples];

std::mutex g_setup_mutex;
float* g_table_address[kMaxDevices] = {};

// Device address of the table array on the current device. In host code the name
// g_hilbert_tables is only a handle for the runtime, not an address the kernel may use; the
// address is looked up once per device, with that device current.
bool table_address(float** out)
{
    int dev = 0;
    CUTB_CUDA_OK(cudaGetDevice(&dev));
    CUTB_REQUIRE(dev >= 0 && dev < kMaxDevices, CUTB_ERR_UNSUPPORTED, "Device index %d too large.", dev);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_table_address[dev]) {
        void* p = nullptr;
        CUTB_CUDA_OK(cudaGetSymbolAddress(&p, g_hilbert_tables));
        g_table_address[dev] = static_cast<float*>(p);
    }
    *out = g_table_address[dev];
    return true;
}

}  // namespace
}  // namespace cutb

using namespace cutb;

extern "C" CUTB_API bool cutb_hilbert_static(const float* d_in, uint in_stride, void* d_iq, uint samples,
                                             size_t rows, const float* taps, uint ntaps, void* stream)
{
    CUTB_REQUIRE(d_in && d_iq, CUTB_ERR_INVALID_ARGUMENT, "cutb_hilbert_static: null device buffer.");
    CUTB_REQUIRE(in_stride == 1 || in_stride == 2, CUTB_ERR_INVALID_ARGUMENT, "Input stride must be 1 or 2.");
    CUTB_REQUIRE(rows > 0, CUTB_ERR_INVALID_ARGUMENT, "cutb_hilbert_static: no rows.");
    CUTB_REQUIRE(samples <= kStaticMaxSamples, CUTB_ERR_INVALID_ARGUMENT,
                 "cutb_hilbert_static: %u samples per row exceed the fixed table capacity of %u.", samples,
                 kStaticMaxSamples);
    CUTB_REQUIRE(hilbert_supported_length(samples), CUTB_ERR_UNSUPPORTED,
                 "Sample count %u not supported by the FFT (powers of two up to %u, other lengths up to %u).",
                 samples, kMaxHilbertLength, kMaxHilbertLength / 2);
    CUTB_REQUIRE(hilbert_fft_length(samples) <= kStaticMaxSamples, CUTB_ERR_INVALID_ARGUMENT,
                 "cutb_hilbert_static: %u samples per row need a transform of %u points, above the fixed table "
                 "capacity of %u.", samples, hilbert_fft_length(samples), kStaticMaxSamples);
    CUTB_REQUIRE(ntaps == 0 || taps, CUTB_ERR_INVALID_ARGUMENT, "Null match filter.");
    // The table upload copies from host vectors that are freed when the call returns, so a graph
    // captured from it would replay reads of freed memory: capture is refused.
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    CUTB_CUDA_OK(cudaStreamIsCapturing((cudaStream_t)stream, &capturing));
    CUTB_REQUIRE(capturing == cudaStreamCaptureStatusNone, CUTB_ERR_UNSUPPORTED,
                 "cutb_hilbert_static cannot be captured in a CUDA graph (its tables are uploaded from host "
                 "memory that the call frees).");
    std::vector<float> tw, weight;  // host memory only
    if (!build_hilbert_tables(samples, taps, ntaps, tw, weight)) return false;
    float* tables = nullptr;
    if (!table_address(&tables)) return false;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = tw.size();  // 2 floats per point of the FFT length (<= kStaticMaxSamples)
    CUTB_CUDA_OK(cudaMemcpyAsync(tables, tw.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
    CUTB_CUDA_OK(cudaMemcpyAsync(tables + n, weight.data(), 2 * n * sizeof(float), cudaMemcpyHostToDevice, st));
    HilbertArgs a{};
    a.rows = rows;
    a.n = samples;
    a.log_n = 0;
    while ((1u << a.log_n) < n / 2) ++a.log_n;
    a.in_stride = in_stride;
    a.twiddle = tables;
    a.weight = tables + n;
    return launch_hilbert(a, d_in, d_iq, false, st);
}
