// Shared helpers for the sm_100a kernels and their C-ABI hosts.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace rb200 {

inline void check(cudaError_t status, const char* what) {
    if (status != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(status));
}
inline void require(bool ok, const char* message) {
    if (!ok) throw std::runtime_error(message);
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
