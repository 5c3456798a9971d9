// FP32 FMA throughput probe. The delay-and-sum stage is bound by FP32 issue rate, for
// which no measured device peak is otherwise available; the benchmark reports its
// achieved FLOP/s against this probe (and against the nominal SM count x 128 lanes x 2
// x clock). Each thread runs 8 independent FMA chains so the pipeline never waits on a
// dependency.
#include "common.cuh"

namespace {

__global__ void __launch_bounds__(256) fma_probe(float* out, int iters, float a, float b)
{
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == 12345.678f) out[0] = s;  // keeps the chains live
}

}  // namespace

extern "C" CUTB_API bool cutb_calibrate_fp32(double* tflops, void* stream)
{
    CUTB_REQUIRE(tflops != nullptr, CUTB_ERR_INVALID_ARGUMENT, "Null output.");
    int dev = 0, sms = 0;
    CUTB_CUDA_OK(cudaGetDevice(&dev));
    CUTB_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t st = (cudaStream_t)stream;
    float* d_out = nullptr;
    CUTB_CUDA_OK(cudaMalloc(&d_out, sizeof(float)));
    const int blocks = sms * 8, threads = 256, iters = 1 << 15;
    cudaEvent_t e0, e1;
    CUTB_CUDA_OK(cudaEventCreate(&e0));
    CUTB_CUDA_OK(cudaEventCreate(&e1));
    fma_probe<<<blocks, threads, 0, st>>>(d_out, 1024, 0.999f, 1e-3f);  // warm up
    CUTB_CUDA_OK(cudaEventRecord(e0, st));
    fma_probe<<<blocks, threads, 0, st>>>(d_out, iters, 0.999f, 1e-3f);
    CUTB_CUDA_OK(cudaEventRecord(e1, st));
    CUTB_CUDA_OK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CUTB_CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    *tflops = 2.0 * 8.0 * (double)iters * blocks * threads / (ms * 1e-3) / 1e12;
    return true;
}
