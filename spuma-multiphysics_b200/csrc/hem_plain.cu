// The plain FP64 form of the HEM flash: one thread per cell runs that cell's
// whole candidate search (src/reactiveThermo/reactiveDeviceFlash.h:509-560, the
// reference's hemKernel layout, src/reactiveThermo/reactiveGpuHem.cuh:64-80),
// with no work queue and no pruning. It is the baseline the work-queue form is
// measured against, so it is built the way it runs fastest: in its own
// translation unit with every EOS and flash routine inlined (the queue form
// keeps them out of line) and the full register file per thread.
#include "hem_common.cuh"
#include "common.cuh"

namespace rb200 {
namespace {

__global__ void __launch_bounds__(kPassThreads, 1) flashPerCell(const HemConst* __restrict__ Cp,
                                                             const CellInput* __restrict__ in, size_t count,
                                                             const ReactiveThermoState* seed,
                                                             ReactiveThermoState* state,
                                                             ReactiveTransportState* transport, int* success,
                                                             unsigned* counters, unsigned long long* totals) {
    const HemConst& C = *Cp;
    Counts n;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        const CellInput x = in[c];
        ReactiveThermoState best{};
        double bestEntropy = 0;
        bool have = false, gasStable = false;
        for (int k = 0; k < 7; ++k) {
            if (k >= 2 && C.stableGasPrune && gasStable) break;
            Eval v;
            CandidateOut o{};
            bool ok;
            GasPoint g;
            bool known;
            if (k == 0) ok = frozenSolve(C, x, 0.0, C.stableGasPrune ? 4 : 0, v, o, n, g, known);
            else if (k == 1) ok = frozenSolve(C, x, x.q, 0, v, o, n, g, known);
            else ok = twoPhaseSolve(C, x, kSeeds[k - 2], -1.0, v, o, n);
            if (!ok) { ++n.failures; continue; }
            if (!stableAt(C, x.q, v.liqMass, v.p, v.T, n)) { ++n.failures; continue; }
            ++n.stable;
            if (k == 0) gasStable = v.gasMass > 0;
            if (!have || v.entropyD > bestEntropy) {
                have = true;
                bestEntropy = v.entropyD;
                stateFromEval(v, x.q, o, best);
            }
        }
        if (!have) {
            const double lower = fmax(C.Tmin, C.liquidTmin), upper = fmin(C.Tmax, C.liquidTc * (1 - 1e-10));
            for (int t = 0; t < 4 && upper > lower; ++t)
                for (int s = 0; s < 5; ++s) {
                    Eval v;
                    CandidateOut o{};
                    if (!twoPhaseSolve(C, x, kSeeds[s], lower + (upper - lower) * kRestart[t], v, o, n)
                        || !stableAt(C, x.q, v.liqMass, v.p, v.T, n)) { ++n.failures; continue; }
                    ++n.stable;
                    if (!have || v.entropyD > bestEntropy) {
                        have = true;
                        bestEntropy = v.entropyD;
                        stateFromEval(v, x.q, o, best);
                    }
                }
        }
        if (have) {
            writeOutputs(best, c, state, transport);
        } else {
            if (state) state[c] = seed[c];
            if (transport) writeOutputs(seed[c], c, nullptr, transport);
            atomicAdd(counters + FAILED, 1u);
        }
        if (success) success[c] = have ? 1 : 0;
    }
    flushCounts(n, totals);
}

}  // namespace

void launchPlainFlash(const HemConst* cst, const CellInput* in, size_t count, const ReactiveThermoState* seed,
                      ReactiveThermoState* state, ReactiveTransportState* transport, int* success,
                      unsigned* counters, unsigned long long* totals, cudaStream_t s) {
    flashPerCell<<<unsigned((count + kPassThreads - 1) / kPassThreads), kPassThreads, 0, s>>>(
        cst, in, count, seed, state, transport, success, counters, totals);
    check(cudaGetLastError(), "flashPerCell");
}

}  // namespace rb200
