// Shared helpers for the sm_100a kernels and their C-ABI hosts.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace rb200 {

inline void check(cudaError_t status, const char* what) {
    if (status != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(status));
}
inline void require(bool ok, const char* message) {
    if (!ok) throw std::runtime_error(message);
}

// Index of the first element in [0, count) for which ok(i) is false, or count.
// Large host arrays (the per-cell validation of caller buffers) are scanned by
// all hardware threads in contiguous chunks; the result is the same index a
// serial scan finds.
template <class Pred> size_t firstFailure(size_t count, Pred ok) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t threads = count < (size_t(1) << 18) ? 1 : std::min<size_t>(hw, 64);
    if (threads == 1) {
        for (size_t i = 0; i < count; ++i)
            if (!ok(i)) return i;
        return count;
    }
    std::vector<size_t> first(threads, count);
    std::vector<std::thread> pool;
    const size_t chunk = (count + threads - 1) / threads;
    for (size_t t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            const size_t end = std::min(count, (t + 1) * chunk);
            for (size_t i = t * chunk; i < end; ++i)
                if (!ok(i)) { first[t] = i; return; }
        });
    for (auto& th : pool) th.join();
    return *std::min_element(first.begin(), first.end());
}

// 148 SMs on B200; grids for grid-stride kernels are sized in whole waves of
// resident blocks rather than by the problem size alone.
constexpr int kSmCount = 148;

inline unsigned gridFor(size_t n, unsigned block, unsigned maxBlocksPerSm = 8) {
    const size_t need = (n + block - 1) / block;
    const size_t cap = size_t(kSmCount) * maxBlocksPerSm * 16;
    return unsigned(need < cap ? (need ? need : 1) : cap);
}

__device__ __forceinline__ bool isFinite(double x) { return isfinite(x); }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// Warp-level double min/sum with full-warp shuffles (no shared memory).
__device__ __forceinline__ double warpMin(double v) {
    for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warpSum(double v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace rb200
