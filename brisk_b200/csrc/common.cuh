// Shared helpers for the B200 SDP Newton-step kernels (sm_100a only).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <atomic>
#include <cstdio>
#include <cmath>

#if !defined(__CUDA_ARCH__) || (__CUDA_ARCH__ >= 1000)
#else
#error "brisk_b200 is built for sm_100a only"
#endif

// Status codes returned through the C ABI (BGPU_OK, BGPU_ERR_*).
#include "../../include/bgpu.h"

#define BGPU_CHECK(call)                                                                   \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            fprintf(stderr, "brisk_b200: CUDA error %s at %s:%d: %s\n", cudaGetErrorName(e_), \
                    __FILE__, __LINE__, cudaGetErrorString(e_));                           \
            return BGPU_ERR_CUDA;                                                          \
        }                                                                                  \
    } while (0)

// Every kernel launch of the library is counted (bgpu_launch_count): the benchmark reports how
// many of its own kernels ran inside the timed region.
extern long long g_bgpu_launches;
#define BGPU_LAUNCH_CHECK()                 \
    do {                                    \
        __atomic_add_fetch(&g_bgpu_launches, 1, __ATOMIC_RELAXED); \
        BGPU_CHECK(cudaGetLastError());     \
    } while (0)

static inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Kernel attributes (cudaFuncSetAttribute) and occupancy figures belong to one device: a launcher
// sets them once per device.  `done` keeps one bit per device 0-63 (the setter runs on every call
// on a device above 63); two threads that set the same attribute at once do no harm.
template <class F>
inline int once_per_device(std::atomic<unsigned long long> &done, F &&set) {
    int dev = 0;
    BGPU_CHECK(cudaGetDevice(&dev));
    const unsigned long long bit = (dev >= 0 && dev < 64) ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return BGPU_OK;
    const int rc = set();
    if (rc == BGPU_OK && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return rc;
}
#define BGPU_ATTR_ONCE(...)                                                                           \
    do {                                                                                              \
        static std::atomic<unsigned long long> attr_done_{0};                                          \
        if (int rc_ = once_per_device(attr_done_, [&]() -> int { __VA_ARGS__; return BGPU_OK; })) return rc_; \
    } while (0)

// The bound of the triangular solves' device-side waits, in polls of the awaited flag (each
// followed by a 64 ns sleep), and the failure-path test's held block row (bgpu_set_wait_limit,
// bgpu_test_hold_trsv_row).
unsigned wait_limit();
int trsv_hold_row();

// ---- device helpers -------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// cp.async of 8 bytes with zero fill when `valid` is false (src is not read then).
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Bounded spin limit for device-side waits (about a second at B200 clocks with the
// nanosleep back-off below); a wait that runs out sets an error flag and returns.
#define BGPU_SPIN_LIMIT (1u << 22)

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
