/* Force-included before every upstream source when it is compiled for the CPU (test
 * infrastructure only, see oracle/Makefile.ref). Makes the CUDA headers declare mutable
 * thread-index variables, gives host definitions of the device intrinsics upstream's kernels
 * call, and provides the serial kernel launcher that replaces the <<<grid, block>>> syntax. */
#pragma once
#define __STORAGE__ extern
#include <cuda_runtime.h>
#include <device_launch_parameters.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cuComplex.h>
#include <cufft.h>
#include <cublas_v2.h>
#include <npp.h>
#include <cmath>
#include <cstring>
#include <cstdint>
#include <algorithm>

/* Upstream writes `__forceinline__ inline`, a duplicate specifier for a host compiler. The CUDA
 * headers above keep the real definition; upstream code sees an attribute that adds nothing. */
#undef __forceinline__
#define __forceinline__ __attribute__((unused))

inline void __syncthreads() {}
template <class T>
cudaError_t cudaMemcpyToSymbol(const T& symbol, const void* src, size_t count, size_t offset = 0,
                               cudaMemcpyKind kind = cudaMemcpyHostToDevice)
{
    return cudaMemcpyToSymbol((const void*)&symbol, src, count, offset, kind);
}

inline float __cosf(float x) { return std::cos(x); }
inline float __sinf(float x) { return std::sin(x); }
inline int __float2int_rd(float x) { return (int)std::floor(x); }
inline unsigned __float_as_uint(float x) { unsigned u; std::memcpy(&u, &x, 4); return u; }
inline float __uint_as_float(unsigned u) { float x; std::memcpy(&x, &u, 4); return x; }
inline int __float_as_int(float x) { int u; std::memcpy(&u, &x, 4); return u; }
inline float __int_as_float(int u) { float x; std::memcpy(&x, &u, 4); return x; }
using std::isnan;
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }

extern "C" void cutb_ref_set_index(uint3 thread, uint3 block, dim3 block_dim, dim3 grid_dim);

/* Runs kernel(args...) for every thread of the grid, one after another. */
template <class K, class... A>
void cutb_ref_launch(dim3 grid, dim3 block, K kernel, A... args)
{
    for (unsigned bz = 0; bz < grid.z; ++bz)
        for (unsigned by = 0; by < grid.y; ++by)
            for (unsigned bx = 0; bx < grid.x; ++bx)
                for (unsigned tz = 0; tz < block.z; ++tz)
                    for (unsigned ty = 0; ty < block.y; ++ty)
                        for (unsigned tx = 0; tx < block.x; ++tx) {
                            cutb_ref_set_index(make_uint3(tx, ty, tz), make_uint3(bx, by, bz), block, grid);
                            kernel(args...);
                        }
}
