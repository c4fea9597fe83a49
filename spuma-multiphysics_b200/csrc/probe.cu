// Measurement helper: sustained FP64 fused multiply-add rate of this GPU, the
// roofline denominator of the FP64-bound flash (a plain copy and a tensor-core
// GEMM do not bound it). Each thread runs eight independent FMA chains.
#include "common.cuh"
#include "../../include/reactive_b200_probe.h"

namespace rb200 {
__global__ void fmaChains(int iterations, double seed, double* out) {
    double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
           a7 = a0 + 7;
    const double m = 0.999999999, c = 1e-9;
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
            a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains live
}
}  // namespace rb200

extern "C" int rb200_probe_fp64_fma_v1(int blocks, int threads, int iterations, double* scratch, void* stream,
                                       double* flopsPerLaunch) {
    if (blocks <= 0 || threads <= 0 || iterations <= 0 || !scratch || !flopsPerLaunch) return 1;
    rb200::fmaChains<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(iterations, 0.5, scratch);
    *flopsPerLaunch = 2.0 * 8 * 8 * double(iterations) * double(blocks) * double(threads);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
