// Shared host/device helpers of the B200 RF -> volume library: error state,
// logging, CUDA call checking and the tracked device allocator.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/cuda_toolkit_b200.h"

namespace cutb {

// Records `code` and a formatted message for the calling thread and, unless
// CUTB_LOG=0, prints the message to stderr (the upstream library reports every
// failure on stderr and returns false: cuda_toolkit/src/defs.h:125-178).
void set_error(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void log_info(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
int log_level();

// cudaMalloc wrapper honouring the allocation-failure test hook.
cudaError_t device_alloc(void** ptr, size_t bytes);
void device_free(void* ptr);

}  // namespace cutb

#define CUTB_CUDA_OK(call)                                                                      \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            ::cutb::set_error(CUTB_ERR_CUDA, "CUDA error %s (%d) '%s' at %s:%d", cudaGetErrorName(e_), \
                              (int)e_, cudaGetErrorString(e_), __FILE__, __LINE__);             \
            return false;                                                                       \
        }                                                                                       \
    } while (0)

#define CUTB_REQUIRE(cond, code, ...)                                                           \
    do {                                                                                        \
        if (!(cond)) {                                                                          \
            ::cutb::set_error((code), __VA_ARGS__);                                             \
            return false;                                                                       \
        }                                                                                       \
    } while (0)

namespace cutb {

// Ceil division.
template <class A, class B>
__host__ __device__ constexpr A div_up(A a, B b) { return (a + (A)b - 1) / (A)b; }

inline bool is_pow2(uint64_t n) { return n && !(n & (n - 1)); }

// Raises `kern`'s dynamic shared-memory limit to `bytes` on the current device. The attribute is
// held per device, so the caller's `done` mask records the devices (bit d: device d) already set:
// a single flag for the process would skip every device after the first. Devices past 63 set it
// on every call. Concurrent first calls only repeat the idempotent attribute call.
template <class Kernel>
bool set_smem_limit(Kernel kern, size_t bytes, std::atomic<uint64_t>& done)
{
    int dev = 0;
    CUTB_CUDA_OK(cudaGetDevice(&dev));
    const uint64_t bit = dev >= 0 && dev < 64 ? 1ull << dev : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return true;
    CUTB_CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done.fetch_or(bit, std::memory_order_release);
    return true;
}

}  // namespace cutb
