// Shared helpers of the deepmr_b200 CUDA library: error reporting, launch
// accounting and small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>

#include "deepmr_b200.h"

namespace dmr {

// Per-thread last error message (dmr_last_error).
void set_error(const char *fmt, ...);

// Kernels launched by this library since load (dmr_launch_count).
extern std::atomic<int64_t> g_launches;

inline int cuda_fail(cudaError_t e, const char *what, const char *file, int line)
{
    set_error("%s:%d %s: %s", file, line, what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DMR_ERR_OOM : DMR_ERR_CUDA;
}

}  // namespace dmr

#define DMR_CUDA(call)                                                   \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) return dmr::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

// Call right after a <<<>>> launch: counts it and surfaces launch errors.
#define DMR_LAUNCHED(name)                                               \
    do {                                                                 \
        dmr::g_launches.fetch_add(1, std::memory_order_relaxed);         \
        cudaError_t e_ = cudaGetLastError();                             \
        if (e_ != cudaSuccess) return dmr::cuda_fail(e_, name, __FILE__, __LINE__); \
    } while (0)

#define DMR_CHECK(cond, code, ...)                                       \
    do {                                                                 \
        if (!(cond)) {                                                   \
            dmr::set_error(__VA_ARGS__);                                 \
            return (code);                                               \
        }                                                                \
    } while (0)

#define DMR_TRY(expr)                                                    \
    do {                                                                 \
        int r_ = (expr);                                                 \
        if (r_ != DMR_OK) return r_;                                     \
    } while (0)

namespace dmr {

// Floor modulo for a possibly negative value and positive n.
__host__ __device__ __forceinline__ int pmod(int v, int n)
{
    int r = v % n;
    return r < 0 ? r + n : r;
}

__host__ __device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace dmr
