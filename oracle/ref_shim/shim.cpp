/*
 * CPU emulation of the CUDA runtime, cuBLAS, cuFFT and GL-interop calls that the upstream
 * toolkit's RF -> volume sources make. TEST INFRASTRUCTURE ONLY: oracle/Makefile.ref links it
 * with the upstream sources, compiled unmodified for the host, into oracle/_ref/, so that
 * upstream's own code (entry points, RfProcessor, Beamformer, kernels) can be run on the CPU to
 * produce golden vectors. Nothing in the product library links or loads it.
 *
 * "Device" memory is host memory. Kernels run serially through cutb_ref_launch (refshim.h).
 * cuBLAS Sgemm is a plain column-major FP32 product; cuFFT transforms are computed in double
 * and rounded to float (upstream uses FP32 cuFFT, so intermediate results differ from a GPU
 * run by FP32 rounding only).
 */
#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cufft.h>

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

typedef unsigned int GLuint;

extern "C" {
uint3 threadIdx, blockIdx;
dim3 blockDim, gridDim;
int warpSize = 32;

void cutb_ref_set_index(uint3 thread, uint3 block, dim3 block_dim, dim3 grid_dim)
{
    threadIdx = thread;
    blockIdx = block;
    blockDim = block_dim;
    gridDim = grid_dim;
}

/* ---- runtime -------------------------------------------------------------------------------- */
cudaError_t cudaMalloc(void** p, size_t n)
{
    *p = std::calloc(n ? n : 1, 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaMallocPitch(void** p, size_t* pitch, size_t width, size_t height)
{
    *pitch = (width + 255) / 256 * 256;
    return cudaMalloc(p, *pitch * height);
}
cudaError_t cudaFree(void* p)
{
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind)
{
    std::memmove(d, s, n);
    return cudaSuccess;
}
cudaError_t cudaMemcpy2D(void* d, size_t dpitch, const void* s, size_t spitch, size_t width, size_t height,
                         cudaMemcpyKind)
{
    for (size_t r = 0; r < height; ++r)
        std::memmove((char*)d + r * dpitch, (const char*)s + r * spitch, width);
    return cudaSuccess;
}
cudaError_t cudaMemset(void* d, int v, size_t n)
{
    std::memset(d, v, n);
    return cudaSuccess;
}
cudaError_t cudaMemcpyToSymbol(const void* symbol, const void* src, size_t count, size_t offset, cudaMemcpyKind)
{
    std::memcpy((char*)symbol + offset, src, count);
    return cudaSuccess;
}
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaStreamDestroy(cudaStream_t) { return cudaSuccess; }
const char* cudaGetErrorName(cudaError_t) { return "cudaError(emulated)"; }
const char* cudaGetErrorString(cudaError_t) { return "emulated CUDA error"; }

/* ---- GL interop: buffer ids resolve to host buffers registered by the harness ------------- */
static std::map<GLuint, std::pair<void*, size_t>>& gl_buffers()
{
    static auto* m = new std::map<GLuint, std::pair<void*, size_t>>;  // outlives upstream's statics
    return *m;
}
void ref_register_buffer(GLuint id, void* ptr, size_t bytes) { gl_buffers()[id] = {ptr, bytes}; }

cudaError_t cudaGraphicsGLRegisterBuffer(cudaGraphicsResource_t* res, GLuint buffer, unsigned int)
{
    if (!gl_buffers().count(buffer)) return cudaErrorInvalidValue;
    *res = (cudaGraphicsResource_t)(uintptr_t)buffer;
    return cudaSuccess;
}
cudaError_t cudaGraphicsMapResources(int, cudaGraphicsResource_t*, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaGraphicsUnmapResources(int, cudaGraphicsResource_t*, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaGraphicsUnregisterResource(cudaGraphicsResource_t) { return cudaSuccess; }
cudaError_t cudaGraphicsResourceGetMappedPointer(void** p, size_t* n, cudaGraphicsResource_t res)
{
    auto it = gl_buffers().find((GLuint)(uintptr_t)res);
    if (it == gl_buffers().end()) return cudaErrorInvalidValue;
    *p = it->second.first;
    *n = it->second.second;
    return cudaSuccess;
}

/* ---- cuBLAS: column-major C = alpha op(A) op(B) + beta C, FP32 accumulation in k order --------- */
cublasStatus_t cublasCreate_v2(cublasHandle_t* h)
{
    *h = (cublasHandle_t)(uintptr_t)1;
    return CUBLAS_STATUS_SUCCESS;
}
cublasStatus_t cublasDestroy_v2(cublasHandle_t) { return CUBLAS_STATUS_SUCCESS; }
cublasStatus_t cublasSgemm_v2(cublasHandle_t, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                              const float* alpha, const float* A, int lda, const float* B, int ldb,
                              const float* beta, float* C, int ldc)
{
    if (ta != CUBLAS_OP_N || tb != CUBLAS_OP_N) return CUBLAS_STATUS_NOT_SUPPORTED;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            float acc = 0.f;
            for (int p = 0; p < k; ++p) acc += A[i + (size_t)p * lda] * B[p + (size_t)j * ldb];
            float prev = *beta == 0.f ? 0.f : *beta * C[i + (size_t)j * ldc];
            C[i + (size_t)j * ldc] = *alpha * acc + prev;
        }
    return CUBLAS_STATUS_SUCCESS;
}

/* ---- cuFFT ---------------------------------------------------------------------------------- */
struct Plan {
    int n, batch, type;
    int istride, idist, ostride, odist;
};
static std::map<cufftHandle, Plan>& plans()
{
    static auto* m = new std::map<cufftHandle, Plan>;  // outlives upstream's statics
    return *m;
}
static cufftHandle next_handle = 1;

cufftResult cufftPlanMany(cufftHandle* plan, int rank, int* n, int* inembed, int istride, int idist, int* onembed,
                          int ostride, int odist, cufftType type, int batch)
{
    if (rank != 1) return CUFFT_INVALID_VALUE;
    Plan p{n[0], batch, (int)type, istride, idist, ostride, odist};
    if (!inembed) {  // basic layout
        p.istride = 1;
        p.idist = type == CUFFT_C2R ? n[0] / 2 + 1 : n[0];
    }
    if (!onembed) {
        p.ostride = 1;
        p.odist = type == CUFFT_R2C ? n[0] / 2 + 1 : n[0];
    }
    *plan = next_handle++;
    plans()[*plan] = p;
    return CUFFT_SUCCESS;
}
cufftResult cufftPlan1d(cufftHandle* plan, int nx, cufftType type, int batch)
{
    return cufftPlanMany(plan, 1, &nx, nullptr, 1, 0, nullptr, 1, 0, type, batch);
}
cufftResult cufftDestroy(cufftHandle plan)
{
    plans().erase(plan);
    return CUFFT_SUCCESS;
}

static void dft(std::vector<std::complex<double>>& a, int sign)
{
    const size_t n = a.size();
    std::vector<std::complex<double>> r(n);
    for (size_t k = 0; k < n; ++k) {
        std::complex<double> acc = 0;
        for (size_t j = 0; j < n; ++j) {
            const double ang = sign * 2.0 * M_PI * (double)((k * j) % n) / (double)n;
            acc += a[j] * std::complex<double>(std::cos(ang), std::sin(ang));
        }
        r[k] = acc;
    }
    a.swap(r);
}
static void fft(std::vector<std::complex<double>>& a, int sign)
{
    const size_t n = a.size();
    if (n & (n - 1)) return dft(a, sign);
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1)
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < len / 2; ++k) {
                const double ang = sign * 2.0 * M_PI * (double)k / (double)len;
                const std::complex<double> w(std::cos(ang), std::sin(ang));
                const auto u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
}

cufftResult cufftExecR2C(cufftHandle plan, cufftReal* in, cufftComplex* out)
{
    const Plan& p = plans().at(plan);
    std::vector<std::complex<double>> a(p.n);
    for (int b = 0; b < p.batch; ++b) {
        for (int j = 0; j < p.n; ++j) a[j] = in[(size_t)b * p.idist + (size_t)j * p.istride];
        fft(a, -1);
        for (int k = 0; k <= p.n / 2; ++k) {
            cufftComplex& o = out[(size_t)b * p.odist + (size_t)k * p.ostride];
            o.x = (float)a[k].real();
            o.y = (float)a[k].imag();
        }
    }
    return CUFFT_SUCCESS;
}
cufftResult cufftExecC2C(cufftHandle plan, cufftComplex* in, cufftComplex* out, int direction)
{
    const Plan& p = plans().at(plan);
    std::vector<std::complex<double>> a(p.n);
    for (int b = 0; b < p.batch; ++b) {
        for (int j = 0; j < p.n; ++j) {
            const cufftComplex& v = in[(size_t)b * p.idist + (size_t)j * p.istride];
            a[j] = {v.x, v.y};
        }
        fft(a, direction == CUFFT_FORWARD ? -1 : +1);
        for (int k = 0; k < p.n; ++k) {
            cufftComplex& o = out[(size_t)b * p.odist + (size_t)k * p.ostride];
            o.x = (float)a[k].real();
            o.y = (float)a[k].imag();
        }
    }
    return CUFFT_SUCCESS;
}
}  // extern "C"
