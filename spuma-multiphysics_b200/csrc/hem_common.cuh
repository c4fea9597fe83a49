// Pieces shared by the HEM translation units: queue counters, work totals, the
// seed schedules and the per-cell output write.
#pragma once
#include "hem_flash.cuh"

namespace rb200 {
namespace {

enum Counter { Q_A = 0, Q_B, LIST, Q_C, FALLBACK, FAILED, NCOUNTERS = 8 };
enum Total { T_PHASES = 0, T_RESIDUALS, T_CANDIDATES, T_STABLE, T_FAILURES, T_ANALYTIC, T_FD, T_SUCCEEDED, NTOTALS = 8 };

// Work-queue kernels: 128 threads, at least four blocks per SM (<= 128
// registers a thread). With the EOS routines out of line, sixteen resident warps
// per SM hide the latency of the FP64 chains better than eight warps at 255
// registers, and spill nothing that matters.
constexpr int kPassThreads = 128;
#ifndef RB200_PASS_MINBLOCKS
#define RB200_PASS_MINBLOCKS 4
#endif
__constant__ double kSeeds[5] = {-1, .5, .95, .1, .9999};
__constant__ double kRestart[4] = {0.02, 0.25, 0.5, 0.75};

__device__ __forceinline__ void flushCounts(const Counts& n, unsigned long long* totals) {
    unsigned long long v[7] = {n.phases, n.residuals, n.candidates, n.stable, n.failures, n.analytic, n.fd};
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        unsigned long long x = v[i];
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(totals + i, x);
    }
}

// The outputs are written once and not read again by the flash: streaming
// stores (evict-first in L2), so they do not push the solver threads' stack
// frames out of L2 (bit-identical results, 2.7% off a 160^3 flash launch).
__device__ inline void writeOutputs(const ReactiveThermoState& s, size_t c, ReactiveThermoState* state,
                                    ReactiveTransportState* transport) {
    if (state) {
        const double* src = reinterpret_cast<const double*>(&s);
        double* dst = reinterpret_cast<double*>(state + c);
#pragma unroll
        for (int i = 0; i < int(sizeof(ReactiveThermoState) / sizeof(double)); ++i) __stcs(dst + i, src[i]);
    }
    if (transport) {
        const double t[7] = {s.p, s.T, s.rho, s.cv, s.soundFrozen, s.gasMass, 0.0};
        double* dst = reinterpret_cast<double*>(transport + c);
#pragma unroll
        for (int i = 0; i < 7; ++i) __stcs(dst + i, t[i]);
    }
}

}  // namespace
}  // namespace rb200
