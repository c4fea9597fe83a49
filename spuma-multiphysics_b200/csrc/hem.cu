// reactive_gpu_hem_* C ABI on B200: candidate-parallel pure-fluid UV flash.
//
// Launch sequence per batch (all on one stream, no host synchronisation, no
// allocation; capturable in a CUDA graph):
//   1 inputs     per cell: (rho, e, seed p/T/liquid mass)
//   2 queue      persistent lane-level work queue over (candidate, cell) items:
//                all seven candidates of every cell; with the model's
//                stableGasPrune option, the all-gas/all-liquid items first, then
//   3 compact    the cells the all-gas candidate does not decide, and
//   4 queue      their five two-phase seeds
//   5 select     first maximum entropy among stable candidates, in reference
//                order; cells without one are queued for the restart search
//   6 pass C     persistent queue over (queued cell, 4 restart temperatures),
//                each running the 5 seeds and keeping its first best
//   7 select     over the 4 restarts; cells still without a candidate fail
// Candidate records live in HBM (192 B each); every loop in the solvers is
// bounded and no thread waits on another, so every launch terminates.
#include "hem_flash.cuh"
#include "hem_common.cuh"
#include "hem_queue.cuh"
#include "hem_mixture.h"
#include "common.cuh"
#include "../../include/reactive_b200_hem.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace rb200 {
// The plain one-thread-per-cell form (hem_plain.cu).
void launchPlainFlash(const HemConst* cst, const CellInput* in, size_t count, const ReactiveThermoState* seed,
                      ReactiveThermoState* state, ReactiveTransportState* transport, int* success,
                      unsigned* counters, unsigned long long* totals, cudaStream_t s);
namespace {

struct CandRecord {
    ReactiveThermoState st;
    double entropyD;
    int status;  // 0 not converged, 1 converged but unstable, 2 converged and stable
    int pad;
};
static_assert(sizeof(CandRecord) == 192, "candidate record layout");

// Warp-wide dynamic fetch of 32 consecutive items from a device counter.
__device__ __forceinline__ unsigned fetchItems(unsigned* counter) {
    unsigned base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(counter, 32u);
    return __shfl_sync(0xffffffffu, base, 0);
}

__global__ void inputsFromHost(const HemConst* __restrict__ Cp, const double* q, const double* energy,
                               const ReactiveThermoState* guess, size_t count, int ns, CellInput* in) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        double rho = 0;
        for (int k = 0; k < ns; ++k) rho += q[c * ns + k];
        const ReactiveThermoState g = guess[c];
        in[c] = CellInput{rho, energy[c], g.p, g.T, g.liquidMass[0], twoPhaseImpossible(*Cp, rho, energy[c])};
    }
}

// Inputs of a device-resident batch named by `order` (global cell indices):
// q holds ns masses per cell, energy the bulk internal energy density; the
// seeds are gathered too (a failed cell returns its seed). A capillary entry
// that asks for a pressure jump or the frozen partition sets *unsupported.
__global__ void inputsFromResident(const HemConst* __restrict__ Cp, const double* q, const double* energy,
                                   const ReactiveThermoState* seed, const ReactiveGpuHemCapillaryInputV2* capillary,
                                   const uint32_t* order, size_t count, int ns, CellInput* in,
                                   ReactiveThermoState* guess, unsigned* unsupported) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(blockDim.x) * gridDim.x) {
        const size_t c = order[i];
        if (capillary && !(capillary[c].pressureJump == 0.0 && capillary[c].equilibrium == 1)) atomicOr(unsupported, 1u);
        double rho = 0;
        for (int k = 0; k < ns; ++k) rho += q[c * size_t(ns) + k];
        const ReactiveThermoState g = seed[c];
        guess[i] = g;
        in[i] = CellInput{rho, energy[c], g.p, g.T, g.liquidMass[0], twoPhaseImpossible(*Cp, rho, energy[c])};
    }
}

// Results of a resident batch to output[order[i]].
__global__ void scatterResident(const ReactiveThermoState* state, const int* success, const uint32_t* order,
                                size_t count, ReactiveGpuHemOutputV1* output) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(blockDim.x) * gridDim.x) {
        ReactiveGpuHemOutputV1& o = output[order[i]];
        o.state = state[i];
        o.success = success[i];
        o.reserved = 0;
    }
}

// Flash inputs of cell c from the SoA conserved rows: the mass density, the
// internal energy density E - |m|^2/(2 rho) and the seed's p, T and liquid mass.
// Streaming loads (evict-first in L2): each is read once here, and the
// single-phase pass keeps its threads' stack frames in L2 better without them
// (1.9% off a 160^3 step).
__device__ __forceinline__ CellInput conservedInput(const HemConst& C, const double* cons, size_t stride, size_t c,
                                                    int ns, const ReactiveThermoState* seed) {
    double rho = 0;
    for (int k = 0; k < ns; ++k) rho += __ldcs(cons + size_t(k) * stride + c);
    const double mx = __ldcs(cons + size_t(ns) * stride + c), my = __ldcs(cons + size_t(ns + 1) * stride + c),
                 mz = __ldcs(cons + size_t(ns + 2) * stride + c), E = __ldcs(cons + size_t(ns + 3) * stride + c);
    const double e = E - .5 * (mx * mx + my * my + mz * mz) / rho;
    return CellInput{rho, e, __ldcs(&seed[c].p), __ldcs(&seed[c].T), __ldcs(&seed[c].liquidMass[0]),
                     twoPhaseImpossible(C, rho, e)};
}

__global__ void inputsFromConserved(const HemConst* __restrict__ Cp, const double* cons, size_t stride, size_t count,
                                    int ns, const ReactiveThermoState* seed, CellInput* in) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x)
        in[c] = conservedInput(*Cp, cons, stride, c, ns, seed);
}

struct MainRecords {
    CandRecord* rec;
    size_t count;
    __device__ CandRecord& at(const QueueLane& L) const { return rec[size_t(L.kind) * count + L.cell]; }
    __device__ void state(const QueueLane& L, const Eval& v) const {
        CandRecord& r = at(L);
        stateFromEval(v, L.x.q, L.o, r.st);
        r.entropyD = v.entropyD;
    }
    __device__ void status(const QueueLane& L, int code) const { at(L).status = code; }
};

// Lanes of a warp that help line searches once the queue is drained.
constexpr int kLineHelpers = 8;

__device__ __forceinline__ int nthSetBit(unsigned mask, int n) {
    for (int i = 0; i < n; ++i) mask &= mask - 1;
    return __ffs(mask) - 1;
}

// Persistent lane-level queue over items (kind, cell): kinds [kindBase,
// kindBase+kinds), cells 0..count-1 or list[0..counters[LIST]) when list != null.
// Items are kind-major, so consecutive items share a candidate kind.
//
// Once a warp's lanes find the queue empty, up to kLineHelpers of its idle lanes
// evaluate the next trial fractions of the warp's line searches (frozen-partition
// and two-phase Newton) beside the searching lanes' own trials (the r-th helper
// takes searching lane r mod S, trial offset 1 + r / S). A searching lane whose
// own trial is rejected walks its helpers' trials in order and takes the first
// that passes the same acceptance test: the search ends on the same fraction with
// the same evaluation (the same routine on the same inputs) as the serial search,
// in fewer rounds of a lone lane's FP64 latency.
__global__ void __launch_bounds__(kPassThreads, RB200_PASS_MINBLOCKS) passQueue(const HemConst* __restrict__ Cp,
                                                          const CellInput* __restrict__ in, size_t count,
                                                          const unsigned* __restrict__ list, int kindBase, int kinds,
                                                          CandRecord* rec, unsigned* counters, int queueSlot,
                                                          unsigned long long* totals) {
    const HemConst& C = *Cp;
    Counts n;
    const unsigned cells = list ? counters[LIST] : unsigned(count);
    const unsigned total = unsigned(kinds) * cells;
    const MainRecords records{rec, count};
    const int stallLimitGas = C.stableGasPrune ? 4 : 0;
    const unsigned lane = threadIdx.x & 31u;
    __shared__ Eval helpEval[kPassThreads / 32][kLineHelpers];
    __shared__ signed char helpResult[kPassThreads / 32][kLineHelpers];  // -1 no trial, 0 failed/skipped, 1 evaluated
    const unsigned warp = threadIdx.x >> 5;
    QueueLane L;
    L.st = Q_FREE;
    L.req = REQ_NONE;
    L.known = false;
    Eval v;
    bool pending = false, exhausted = cells == 0;
    // A short queue (fewer items than 32 per resident warp) is spread over the
    // warps: a warp takes at most `cap` items per fetch, so a few long items (the
    // frozen all-gas solves of cells inside the saturation dome late in a run) land
    // in different warps whose other lanes, once the queue is drained, evaluate
    // their line-search trials. Which lane runs an item changes no result.
    const unsigned gridWarps = gridDim.x * (blockDim.x >> 5);
    const unsigned cap = min(32u, max(1u, (total + gridWarps - 1) / gridWarps));
    for (;;) {
        for (int round = 0; round < 2; ++round) {
            bool need = L.st == Q_FREE && !exhausted;
            unsigned mask = __ballot_sync(0xffffffffu, need);
            if (unsigned(__popc(mask)) > cap) {
                unsigned rest = mask, take = 0;
                for (unsigned i = 0; i < cap; ++i) { take |= rest & (0u - rest); rest &= rest - 1; }
                mask = take;
                need = (mask >> lane) & 1u;
            }
            if (mask) {
                unsigned base = 0;
                if (lane == unsigned(__ffs(mask) - 1)) base = atomicAdd(counters + queueSlot, unsigned(__popc(mask)));
                base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
                if (need) {
                    const unsigned item = base + __popc(mask & ((1u << lane) - 1));
                    if (item < total) {
                        const unsigned kind = unsigned(kindBase) + item / cells, slot = item % cells;
                        L.kind = int(kind);
                        L.cell = list ? list[slot] : slot;
                        L.x = in[L.cell];
                        L.o = CandidateOut{};
                        L.mass = kind == 1 ? L.x.q : 0.0;
                        L.st = kind >= 2 ? Q_TP_START : Q_FZ_START;
                        L.req = REQ_NONE;
                        L.known = false;
                        if (kind >= 2 && L.x.noTwoPhase) {
                            // outside every saturation tie line: the seed cannot converge
                            ++n.candidates;
                            ++n.failures;
                            records.status(L, 0);
                            L.st = Q_FREE;
                        }
                    } else exhausted = true;
                }
            }
            // the item counter only grows: once one lane finds the queue drained, it
            // is drained for every lane of the warp (capped fetches would otherwise
            // discover it one lane at a time)
            exhausted = __any_sync(0xffffffffu, exhausted);
            if (L.st != Q_FREE && !pending) pending = plan(C, L, v, records, n, stallLimitGas);
        }
        const bool any = __any_sync(0xffffffffu, pending);
        if (!any) {
            if (__all_sync(0xffffffffu, L.st == Q_FREE && exhausted)) break;
            continue;
        }
        // line-search helpers (a warp-uniform decision)
        const bool tpSearch = pending && L.req == REQ_POINT && L.st == Q_TP_LS_AFTER;
        const bool fzSearch = pending && L.req == REQ_POINT && L.st == Q_FZ_LS_AFTER;
        const bool search = tpSearch || fzSearch;
        const bool idle = !pending && L.st == Q_FREE && exhausted;
        const unsigned searchMask = __ballot_sync(0xffffffffu, search);
        const unsigned idleMask = __ballot_sync(0xffffffffu, idle);
        const int nS = __popc(searchMask), nH = searchMask ? min(__popc(idleMask), kLineHelpers) : 0;
        // one evaluation per lane at one call site: the lane's own request or a helper's trial
        bool point = pending && L.req == REQ_POINT;
        double eq = L.x.q, erm = L.rm, erp = L.rp, erT = L.rT;
        bool erv = L.rv;
        Eval* out = &v;
        // A lane's own trial passes its kept gas-point terms (L.known); a helper's
        // trial below passes none. The two agree bit for bit only because L.known
        // is set solely in Q_SG_FINAL, never in a line-search state: a searching
        // lane (tpSearch / fzSearch) has L.known false here.
        const GasPoint* kept = L.known ? &L.g : nullptr;
        int helpSlot = -1;
        if (nH > 0) {
            const int r = idle ? __popc(idleMask & ((1u << lane) - 1)) : kLineHelpers;
            const bool helper = idle && r < nH;
            const int target = helper ? nthSetBit(searchMask, r % nS) : int(lane);
            const double a0 = __shfl_sync(0xffffffffu, L.a0, target), a1 = __shfl_sync(0xffffffffu, L.a1, target);
            const double a2 = __shfl_sync(0xffffffffu, L.a2, target), s0 = __shfl_sync(0xffffffffu, L.s0, target);
            const double s1 = __shfl_sync(0xffffffffu, L.s1, target), s2 = __shfl_sync(0xffffffffu, L.s2, target);
            const double f0 = __shfl_sync(0xffffffffu, L.frac, target), q = __shfl_sync(0xffffffffu, L.x.q, target);
            const double mass = __shfl_sync(0xffffffffu, L.mass, target);
            const int k0 = __shfl_sync(0xffffffffu, L.k, target);
            const bool tp = __shfl_sync(0xffffffffu, tpSearch, target);
            if (helper) {
                helpSlot = r;
                const int offset = 1 + r / nS;
                signed char result = -1;  // beyond the search's 30 trials
                if (k0 + offset < 30) {
                    double frac = f0;
                    for (int m = 0; m < offset; ++m) frac *= .5;
                    if (tp && !(a2 + frac * s2 >= 0 && a2 + frac * s2 < 1)) result = 0;  // skipped, no evaluation
                    else {
                        point = true;
                        eq = q;
                        if (tp) {
                            erm = (a2 + frac * s2) * q;
                            erp = exp(a0 + frac * s0);
                            erT = exp(a1 + frac * s1);
                            erv = true;
                        } else {
                            erm = mass;
                            erp = a0 * exp(frac * s0);
                            erT = a1 * exp(frac * s1);
                            erv = false;
                        }
                        out = &helpEval[warp][r];
                        kept = nullptr;
                    }
                }
                helpResult[warp][r] = result;
            }
        }
        if (point) {
            const bool ok = evaluate(C, eq, erm, erp, erT, erv, *out, n, kept);
            if (helpSlot >= 0) helpResult[warp][helpSlot] = ok ? 1 : 0;
            else L.ok = ok;
        } else if (pending) {
            if (L.req == REQ_PROBE) L.ok = gasProbe(C, L.x.q, L.x.e, L.rT, L.pF, L.pCv, L.pP, L.pCp, L.g, n);
            else L.ok = tangentStable(C, L.rp, L.rT, n);
        }
        if (pending) {
            L.req = REQ_NONE;
            pending = false;
        }
        __syncwarp();
        if (nH > 0 && search) {
            double t0, t1, t2;
            const bool own = tpSearch ? tpAccepts(v, L.ok, L.x.e, L.scale, L.prev, L.frac, t0, t1, t2)
                                      : fzAccepts(C, v, L.ok, L.x.e, L.scale, L.prev, L.frac);
            if (!own) {
                // the serial search's next trials, in order, from the helpers
                const int rank = __popc(searchMask & ((1u << lane) - 1));
                bool found = false;
                for (int r = rank; r < nH && !found; r += nS) {
                    const signed char result = helpResult[warp][r];
                    if (result < 0) break;
                    if (tpSearch) ++n.residuals;
                    ++L.k;
                    L.frac *= .5;
                    const Eval& h = helpEval[warp][r];
                    if (result > 0 && (tpSearch ? tpAccepts(h, true, L.x.e, L.scale, L.prev, L.frac, t0, t1, t2)
                                                : fzAccepts(C, h, true, L.x.e, L.scale, L.prev, L.frac))) {
                        v = h;
                        if (fzSearch) {  // the frozen step moves to the trial point itself
                            L.rp = L.a0 * exp(L.frac * L.s0);
                            L.rT = L.a1 * exp(L.frac * L.s1);
                        }
                        found = true;
                    }
                }
                L.ok = found;  // none accepted: the search resumes after the last trial taken
            }
        }
        __syncwarp();
    }
    flushCounts(n, totals);
}

__device__ __forceinline__ bool gasDecides(const HemConst& C, const CandRecord& gas) {
    return C.stableGasPrune && gas.status == 2 && gas.st.gasMass > 0;
}

// Cells whose two-phase seeds provably fail (the two-phase bound) have only
// their all-gas and all-liquid candidates: one thread per cell solves them
// through the same out-of-line solvers the work queue's state machines restate
// (bit for bit the queue's candidates), selects as selectCandidates does (the
// stable candidate of larger entropy, the all-gas one on a tie) and writes the
// outputs; a cell with neither goes to the restart list. The other cells are
// listed for the work queue.
__device__ __forceinline__ void appendTo(unsigned* list, unsigned* counter, bool take, unsigned value) {
    const unsigned mask = __ballot_sync(0xffffffffu, take);
    unsigned slot = 0;
    if ((threadIdx.x & 31) == 0 && mask) slot = atomicAdd(counter, unsigned(__popc(mask)));
    slot = __shfl_sync(0xffffffffu, slot, 0);
    if (take) list[slot + __popc(mask & ((1u << (threadIdx.x & 31)) - 1))] = value;
}

//
// FROM_CONSERVED: the pass forms each cell's inputs itself from the SoA conserved
// rows and the seeds (as inputsFromConserved does) and stores them in `in` only
// for the cells it hands to the work queue or the restart search, the two later
// readers of `in`; the cells it decides never write their inputs. `seed` may be
// `state` (an in-place recovery): a thread reads its own cell's seed before it
// writes that cell's state and touches no other cell's.
template <bool FROM_CONSERVED>
__global__ void __launch_bounds__(kPassThreads, RB200_PASS_MINBLOCKS) passSinglePhase(const HemConst* __restrict__ Cp,
                                                                CellInput* __restrict__ in,
                                                                const double* __restrict__ cons, size_t stride,
                                                                const ReactiveThermoState* seed,
                                                                size_t count, ReactiveThermoState* state,
                                                                ReactiveTransportState* transport, int* success,
                                                                unsigned* list, unsigned* fallback, unsigned* counters,
                                                                unsigned long long* totals) {
    const HemConst& C = *Cp;
    Counts n;
    for (size_t base = blockIdx.x * size_t(blockDim.x); base < count; base += size_t(blockDim.x) * gridDim.x) {
        const size_t c = base + threadIdx.x;
        bool queue = false, restart = false;
        if (c < count) {
            const CellInput x = FROM_CONSERVED ? conservedInput(C, cons, stride, c, 1, seed) : in[c];
            if (!x.noTwoPhase) queue = true;
            else {
                double bestEntropy = 0;
                bool have = false;
                for (int kind = 0; kind < 2; ++kind) {
                    const double mass = kind ? x.q : 0.0;
                    Eval v;
                    CandidateOut o{};
                    GasPoint g;
                    bool known = false;
                    const bool floor = kind == 1 && x.q * (1 + 1e-12) < C.liquidFloor;
                    if (floor || !frozenSolve(C, x, mass, 0, v, o, n, g, known)) {
                        ++n.failures;
                        continue;
                    }
                    const bool stable = stableAt(C, x.q, v.liqMass, v.p, v.T, n, known ? &g : nullptr);
                    if (!stable) {
                        ++n.failures;
                        continue;
                    }
                    ++n.stable;
                    if (!have || v.entropyD > bestEntropy) {
                        // the best so far goes straight to the outputs (a later, better
                        // candidate overwrites it); a cell with none keeps its state
                        have = true;
                        bestEntropy = v.entropyD;
                        ReactiveThermoState st;
                        stateFromEval(v, x.q, o, st);
                        writeOutputs(st, c, state, transport);
                    }
                }
                n.candidates += 5;  // the two-phase seeds, failed without their solves
                n.failures += 5;
                if (have) {
                    if (success) __stcs(success + c, 1);
                } else restart = true;
            }
            if (FROM_CONSERVED && (queue || restart)) in[c] = x;
        }
        appendTo(list, counters + LIST, queue, unsigned(c));
        appendTo(fallback, counters + FALLBACK, restart, unsigned(c));
    }
    flushCounts(n, totals);
}

__global__ void compactSeedCells(const HemConst* __restrict__ Cp, const CandRecord* rec, size_t count,
                                 unsigned* list, unsigned* counters) {
    const HemConst& C = *Cp;
    for (size_t base = blockIdx.x * size_t(blockDim.x); base < count; base += size_t(blockDim.x) * gridDim.x) {
        const size_t c = base + threadIdx.x;
        const bool need = c < count && !gasDecides(C, rec[c]);
        const unsigned mask = __ballot_sync(0xffffffffu, need);
        unsigned slot = 0;
        if ((threadIdx.x & 31) == 0 && mask) slot = atomicAdd(counters + LIST, unsigned(__popc(mask)));
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (need) list[slot + __popc(mask & ((1u << (threadIdx.x & 31)) - 1))] = unsigned(c);
    }
}

// Selection over every cell, or (list) over the cells the work queue solved.
__global__ void selectCandidates(const HemConst* __restrict__ Cp, const CandRecord* rec, size_t count,
                                 const unsigned* list, ReactiveThermoState* state, ReactiveTransportState* transport,
                                 int* success, unsigned* fallback, unsigned* counters) {
    const HemConst& C = *Cp;
    const size_t items = list ? counters[LIST] : count;
    for (size_t base = blockIdx.x * size_t(blockDim.x); base < items; base += size_t(blockDim.x) * gridDim.x) {
        const size_t i = base + threadIdx.x;
        const size_t c = i < items ? (list ? list[i] : i) : count;  // lanes past the end select nothing
        int best = -1;
        double bestEntropy = 0;
        if (c < count) {
            const int kinds = gasDecides(C, rec[c]) ? 2 : 7;
            for (int k = 0; k < kinds; ++k) {
                const CandRecord& r = rec[size_t(k) * count + c];
                if (r.status == 2 && (best < 0 || r.entropyD > bestEntropy)) { best = k; bestEntropy = r.entropyD; }
            }
            if (best >= 0) {
                writeOutputs(rec[size_t(best) * count + c].st, c, state, transport);
                if (success) success[c] = 1;
            }
        }
        const bool need = c < count && best < 0;
        const unsigned mask = __ballot_sync(0xffffffffu, need);
        unsigned slot = 0;
        if ((threadIdx.x & 31) == 0 && mask) slot = atomicAdd(counters + FALLBACK, unsigned(__popc(mask)));
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (need) fallback[slot + __popc(mask & ((1u << (threadIdx.x & 31)) - 1))] = unsigned(c);
    }
}

// Pass C: restart temperatures x queued cells; each item runs the five seeds.
__global__ void __launch_bounds__(kPassThreads, RB200_PASS_MINBLOCKS) passRestarts(const HemConst* __restrict__ Cp,
                                                             const CellInput* __restrict__ in,
                                                             const unsigned* __restrict__ fallback, CandRecord* fb,
                                                             size_t capacity, unsigned* counters,
                                                             unsigned long long* totals) {
    const HemConst& C = *Cp;
    Counts n;
    const unsigned queued = counters[FALLBACK];
    const unsigned total = 4u * queued;
    const double lower = fmax(C.Tmin, C.liquidTmin), upper = fmin(C.Tmax, C.liquidTc * (1 - 1e-10));
    for (;;) {
        const unsigned base = fetchItems(counters + Q_C);
        if (base >= total) break;
        const unsigned item = base + (threadIdx.x & 31);
        if (item < total) {
            const unsigned t = item / queued, slot = item % queued;
            const CellInput x = in[fallback[slot]];
            CandRecord* out = fb + size_t(t) * capacity + slot;
            out->status = 0;
            if (x.noTwoPhase) {  // no restart seed can converge either
                n.candidates += 5;
                n.failures += 5;
            } else if (upper > lower) {
                const double restartT = lower + (upper - lower) * kRestart[t];
                bool have = false;
                double bestEntropy = 0;
                for (int s = 0; s < 5; ++s) {
                    Eval v;
                    CandidateOut o{};
                    const bool ok = twoPhaseSolve(C, x, kSeeds[s], restartT, v, o, n);
                    if (!ok) { ++n.failures; continue; }
                    const bool stable = stableAt(C, x.q, v.liqMass, v.p, v.T, n);
                    if (!stable) { ++n.failures; continue; }
                    ++n.stable;
                    if (!have || v.entropyD > bestEntropy) {
                        have = true;
                        bestEntropy = v.entropyD;
                        stateFromEval(v, x.q, o, out->st);
                        out->entropyD = v.entropyD;
                        out->status = 2;
                    }
                }
            }
        }
    }
    flushCounts(n, totals);
}

// Vector-Jacobian product of the flash's transport-state outputs with respect
// to the cell's conserved variables, by the implicit function theorem at the
// converged candidate (no Newton unrolling). The candidate is read from the
// state: two-phase (gas and liquid mass) with unknowns x = (ln p, ln T, beta)
// and residual F = (V - 1, E - e, mu_l/RT - mu_g/RT); an all-gas or all-liquid
// partition with x = (ln p, ln T) and F = (V - 1, E - e), where V and E are
// the evaluation's volume and energy densities at the cell's density q and e is
// the internal energy density of the conserved state. With y(x, q) = (p, T, cv,
// frozen sound, gas mass) and ybar the adjoint of the outputs:
//   F_x^T lambda = y_x^T ybar,  qbar_rho = ybar . y_q - lambda . F_q + rhobar,
//   ebar = lambda_1 (dF_1/de = -1),
// then e = E - |m|^2 / (2 rho) carries ebar to rho, m and E. The partials of
// the closed-form evaluation are central differences (step 1e-6 in ln p, ln T
// and beta, 1e-6 q in q).
struct VjpPoint {
    double F[3], y[5];
};
__device__ inline bool vjpPoint(const HemConst& C, int kind, double q, double e, const double x[3], VjpPoint& o,
                                Counts& n) {
    Eval v;
    const double mass = kind == 2 ? x[2] * q : (kind == 1 ? q : 0.0);
    if (!evaluate(C, q, mass, exp(x[0]), exp(x[1]), kind == 2, v, n)) return false;
    o.F[0] = v.volume - 1;
    o.F[1] = v.energy - e;
    o.F[2] = kind == 2 ? v.muL - v.muG : 0.0;
    o.y[0] = v.p; o.y[1] = v.T; o.y[2] = v.cv; o.y[3] = v.soundFrozen; o.y[4] = v.gasMass;
    return fin(o.F[2]);
}

// The implicit-function adjoint of a single-phase cell in (T, rho) form. At the
// cell's density q the phase's state is a function of T alone, fixed by the
// energy residual F(T; q, e) = q e(T, q) - e = 0, so dT/de = 1/F_T and
// dT/dq = -F_q/F_T; the outputs y = (p, T, cv, frozen sound, gas mass) are
// those of the flash's evaluation of that phase at (T, q) (the (T, rho)
// evaluation needs no cubic root). Central differences of 1e-6 relative in T,
// and in q at fixed T. With lambda = sum(ybar y_T) / F_T: rhoBar +=
// sum(ybar y_q) - lambda F_q and eBar = lambda. False where an evaluation
// fails; the (ln p, ln T) form then runs.
__device__ inline bool singlePhaseVjp(const HemConst& C, int kind, double q, double e, double T, const double ybar[5],
                                      double& rhoBar, double& eBar) {
    const PureSpecies& sp = kind == 0 ? C.gas : C.liq;
    const double Tp = T * (1 + 1e-6), Tm = T * (1 - 1e-6), qp = q * (1 + 1e-6), qm = q * (1 - 1e-6);
    double F[4], y[4][5];
#pragma unroll 1
    for (int i = 0; i < 4; ++i) {
        const double Ti = i == 0 ? Tp : (i == 1 ? Tm : T), qi = i == 2 ? qp : (i == 3 ? qm : q);
        PhaseProps s;
        int phase;
        if (prTrho(sp, Ti, qi, false, s, phase) != EOS_OK) return false;
        // the flash's single-phase sums (mass qi at density qi: unit volume)
        const double vp = -s.kappaT, vt = s.alpha, cpD = qi * s.cp;
        const double cv = (cpD + Ti * vt * vt / vp) / qi;
        const double specific = 1 / qi, adiabatic = vp / qi + Ti * (vt / qi) * (vt / qi) / s.cp;
        F[i] = qi * s.e - e;
        y[i][0] = s.p;
        y[i][1] = Ti;
        y[i][2] = cv;
        y[i][3] = sqrt(-specific * specific / adiabatic);
        y[i][4] = kind == 0 ? qi : 0.0;
    }
    const double hT = Tp - Tm, hq = qp - qm;
    const double FT = (F[0] - F[1]) / hT, Fq = (F[2] - F[3]) / hq;
    double dot = 0, dq = 0;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        dot += ybar[r] * (y[0][r] - y[1][r]) / hT;
        dq += ybar[r] * (y[2][r] - y[3][r]) / hq;
    }
    const double lambda = dot / FT;
    if (!fin(lambda) || !fin(dq) || !fin(Fq) || FT == 0) return false;
    rhoBar += dq - lambda * Fq;
    eBar = lambda;
    return true;
}

__global__ void hemStateVjp(const HemConst* __restrict__ Cp, const double* __restrict__ cons, size_t stride,
                            size_t count, const ReactiveThermoState* __restrict__ state,
                            const ReactiveTransportState* __restrict__ bar, double* qBar, size_t barStride,
                            unsigned* failed) {
    const HemConst& C = *Cp;
    Counts n;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        const double q = cons[c], mx = cons[stride + c], my = cons[2 * stride + c], mz = cons[3 * stride + c],
                     E = cons[4 * stride + c];
        const double m2 = mx * mx + my * my + mz * mz;
        const double e = E - .5 * m2 / q;
        const ReactiveThermoState s = state[c];
        const ReactiveTransportState b = bar[c];
        const bool gas = s.gasMass > 0, liquid = s.liquidMass[0] > 0;
        const int kind = gas && liquid ? 2 : (liquid ? 1 : 0);
        const int nx = kind == 2 ? 3 : 2;
        const double x[3] = {log(s.p), log(s.T), kind == 2 ? s.liquidMass[0] / q : 0.0};
        const double ybar[5] = {b.p, b.T, b.cv, b.sound, b.gasMass};
        {
            double rhoBar = b.rho, eBar = 0;
            if (kind != 2 && singlePhaseVjp(C, kind, q, e, s.T, ybar, rhoBar, eBar)) {
                qBar[c] += rhoBar + eBar * .5 * m2 / (q * q);
                qBar[barStride + c] += -eBar * mx / q;
                qBar[2 * barStride + c] += -eBar * my / q;
                qBar[3 * barStride + c] += -eBar * mz / q;
                qBar[4 * barStride + c] += eBar;
                continue;
            }
        }
        double Fx[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, yx[5][3], Fq[3], yq[5];
        bool ok = true;
#pragma unroll 1
        for (int i = 0; i < 4 && ok; ++i) {
            if (i < 3 && i >= nx) continue;
            const bool onQ = i == 3;
            const double h = onQ ? 1e-6 * q : 1e-6;
            double xp[3] = {x[0], x[1], x[2]}, xm[3] = {x[0], x[1], x[2]};
            double qp = q, qm = q;
            if (onQ) { qp += h; qm -= h; } else { xp[i] += h; xm[i] -= h; }
            VjpPoint a, bm;
            ok = vjpPoint(C, kind, qp, e, xp, a, n) && vjpPoint(C, kind, qm, e, xm, bm, n);
            if (!ok) break;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double d = (a.F[r] - bm.F[r]) / (2 * h);
                if (onQ) Fq[r] = d; else Fx[r][i] = d;
            }
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                const double d = (a.y[r] - bm.y[r]) / (2 * h);
                if (onQ) yq[r] = d; else yx[r][i] = d;
            }
        }
        double lambda[3] = {0, 0, 0};
        if (ok) {
            // F_x^T lambda = y_x^T ybar
            double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, rhs[3] = {0, 0, 0};
#pragma unroll
            for (int i = 0; i < 3; ++i) {
#pragma unroll
                for (int j = 0; j < 3; ++j) A[i][j] = i < nx && j < nx ? Fx[j][i] : 0.0;
                double acc = 0;
#pragma unroll
                for (int r = 0; r < 5; ++r) acc += i < nx ? yx[r][i] * ybar[r] : 0.0;
                rhs[i] = acc;
            }
            ok = solveSmall(A, rhs, nx, lambda);
        }
        if (!ok) {
            if (failed) atomicAdd(failed, 1u);
            continue;
        }
        double rhoBar = b.rho;
#pragma unroll
        for (int r = 0; r < 5; ++r) rhoBar += ybar[r] * yq[r];
#pragma unroll
        for (int r = 0; r < 3; ++r) rhoBar -= r < nx ? lambda[r] * Fq[r] : 0.0;
        const double eBar = lambda[1];  // dF_1/de = -1 and F_x^T lambda carries y's e-dependence
        qBar[c] += rhoBar + eBar * .5 * m2 / (q * q);
        qBar[barStride + c] += -eBar * mx / q;
        qBar[2 * barStride + c] += -eBar * my / q;
        qBar[3 * barStride + c] += -eBar * mz / q;
        qBar[4 * barStride + c] += eBar;
    }
}

// Failed cells get their seed state back, so one contiguous copy of the
// results leaves them unchanged in the caller's array; succeeded (optional)
// counts the other cells.
__global__ void keepFailed(const ReactiveThermoState* __restrict__ seed, const int* __restrict__ success,
                           size_t count, ReactiveThermoState* __restrict__ out,
                           unsigned long long* succeeded = nullptr) {
    unsigned mine = 0;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        if (!success[c]) out[c] = seed[c];
        else ++mine;
    }
    if (succeeded) {
        mine = __reduce_add_sync(0xffffffffu, mine);
        if ((threadIdx.x & 31) == 0 && mine) atomicAdd(succeeded, (unsigned long long)mine);
    }
}

__global__ void selectRestarts(const CandRecord* fb, size_t capacity, const unsigned* fallback,
                               const ReactiveThermoState* seed, ReactiveThermoState* state,
                               ReactiveTransportState* transport, int* success, unsigned* counters) {
    const unsigned queued = counters[FALLBACK];
    for (unsigned slot = blockIdx.x * blockDim.x + threadIdx.x; slot < queued; slot += blockDim.x * gridDim.x) {
        const size_t c = fallback[slot];
        int best = -1;
        double bestEntropy = 0;
        for (int t = 0; t < 4; ++t) {
            const CandRecord& r = fb[size_t(t) * capacity + slot];
            if (r.status == 2 && (best < 0 || r.entropyD > bestEntropy)) { best = t; bestEntropy = r.entropyD; }
        }
        if (best >= 0) {
            writeOutputs(fb[size_t(best) * capacity + slot].st, c, state, transport);
            if (success) success[c] = 1;
        } else {
            if (seed && state) writeOutputs(seed[c], c, state, nullptr);
            if (transport && seed) writeOutputs(seed[c], c, nullptr, transport);
            if (success) success[c] = 0;
            atomicAdd(counters + FAILED, 1u);
        }
    }
}

// One thread per cell running the whole search in order (the layout of the
// reference's hemKernel, src/reactiveTransport/reactiveGpuHem.cuh:64-80): the
// plain form the candidate-parallel passes are measured against. No pruning.

// ------------------------------------------------------------------ host
std::string validateAndDerive(const ReactiveB200HemModel& m, HemConst& C);

// Saturation tie lines of a pure fluid on a temperature grid, one thread per
// temperature: the pressure where the chemical potentials of the smallest and
// largest cubic roots agree, by bisection in ln p (below it the liquid root has
// the higher potential or only a vapour-like root exists; above it the reverse
// or only a liquid-like root). out[5 i..5 i+4] = {valid, v_l, v_g, u_l, u_g}.
// Per temperature: resolved flag, liquid and gas specific volumes, liquid and gas
// specific internal energies, saturation pressure.
constexpr int kSatFields = 6;

__global__ void domeSaturation(const HemConst* __restrict__ Cp, int n, double T0, double dT, double* out) {
    const HemConst& C = *Cp;
    const PureSpecies& sp = C.gas;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += blockDim.x * gridDim.x) {
        double* o = out + kSatFields * size_t(i);
        o[0] = 0;
        const double T = T0 + dT * i;
        TTerms t;
        if (tTerms(sp, T, t) != EOS_OK) continue;
        const double Tcm = sp.a * kOmegaB / (sp.b * kOmegaA * kGas), pc = kOmegaB * kGas * Tcm / sp.b;
        double lo = log(1e-9 * pc), hi = log(2.0 * pc);
        bool ok = true;
        for (int it = 0; it < 160 && ok; ++it) {
            const double lp = .5 * (lo + hi);
            Roots r;
            if (cubicRoots(sp, T, exp(lp), t.aa, r) != EOS_OK) { ok = false; break; }
            if (r.count >= 2) {
                PhaseProps L, G;
                int ph;
                if (prTrhoT(sp, t, sp.W / r.lo, true, L, ph) != EOS_OK || prTrhoT(sp, t, sp.W / r.hi, true, G, ph) != EOS_OK) {
                    ok = false;
                    break;
                }
                if (L.mu > G.mu) lo = lp; else hi = lp;
            } else if (r.liquid && !r.gas) hi = lp;
            else lo = lp;
        }
        if (!ok) continue;
        const double p = exp(.5 * (lo + hi));
        Roots r;
        PhaseProps L, G;
        int ph;
        if (cubicRoots(sp, T, p, t.aa, r) != EOS_OK || r.count < 2 || prTrhoT(sp, t, sp.W / r.lo, true, L, ph) != EOS_OK
            || prTrhoT(sp, t, sp.W / r.hi, true, G, ph) != EOS_OK)
            continue;
        if (!(fabs(L.mu - G.mu) <= 1e-9 * kGas * T) || !(G.rho < L.rho)) continue;
        o[1] = 1 / L.rho; o[2] = 1 / G.rho; o[3] = L.e; o[4] = G.e; o[5] = p;
        o[0] = 1;
    }
}

struct HemDevice {
    std::mutex entry;
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t capacity = 0;
    bool hostPath = false;
    HemConst hostConst{};
    HemConst* cst = nullptr;
    CellInput* in = nullptr;
    CandRecord* rec = nullptr;  // 7 x capacity
    CandRecord* fb = nullptr;   // 4 x capacity
    unsigned* list = nullptr;
    unsigned* fallback = nullptr;
    unsigned* counters = nullptr;
    unsigned long long* totals = nullptr;
    // host-path staging
    double* dq = nullptr;
    double* de = nullptr;
    ReactiveThermoState* dguess = nullptr;
    ReactiveThermoState* dout = nullptr;
    int* dsuccess = nullptr;
    int passBlocks = 0;
    int domeBuilt = 0;  // grid points of the two-phase bound (0: none for this model)
    size_t bytes = 0;
    std::vector<void*> blocks;
    // a model image beyond the pure fluid: the multi-species flash (hem_mixture.cu)
    MixtureFlash* mixture = nullptr;
    // a pure-fluid handle's capillary batches (pressure jumps, the frozen
    // partition, the capillary boundary search): the same engine on the same
    // image, created by the first such batch when the image is in its scope
    std::unique_ptr<ReactiveB200HemModel> image;
    MixtureFlash* capillaryEngine = nullptr;
    MixtureFlash* capillaryFlash() {
        if (mixture) return mixture;
        if (!capillaryEngine && image) {
            std::string why;
            capillaryEngine = mixtureCreate(*image, capacity, device, why);
            if (!capillaryEngine) image.reset();  // outside its scope
            else bytes += mixtureDeviceBytes(capillaryEngine);
        }
        return capillaryEngine;
    }

    template <class T> T* alloc(size_t n) {
        void* p = nullptr;
        check(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
        blocks.push_back(p);
        bytes += n * sizeof(T);
        return static_cast<T*>(p);
    }
    ~HemDevice() {
        if (mixture) mixtureDestroy(mixture);
        if (capillaryEngine) mixtureDestroy(capillaryEngine);
        if (stream) cudaStreamSynchronize(stream);
        if (down) cudaStreamSynchronize(down);
        for (void* p : blocks) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
        if (up) cudaStreamDestroy(up);
        if (down) cudaStreamDestroy(down);
    }
    cudaStream_t up = nullptr, down = nullptr;  // host-path copy streams
    void ensureHostPath() {
        if (hostPath) return;
        check(cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaStreamCreateWithFlags(&down, cudaStreamNonBlocking), "cudaStreamCreate");
        dq = alloc<double>(capacity);
        de = alloc<double>(capacity);
        dguess = alloc<ReactiveThermoState>(capacity);
        dout = alloc<ReactiveThermoState>(capacity);
        dsuccess = alloc<int>(capacity);
        hostPath = true;
    }
    void launchPerCell(size_t count, const ReactiveThermoState* seed, ReactiveThermoState* state,
                       ReactiveTransportState* transport, int* success, cudaStream_t s) {
        check(cudaMemsetAsync(counters, 0, NCOUNTERS * sizeof(unsigned), s), "memset counters");
        launchPlainFlash(cst, in, count, seed, state, transport, success, counters, totals, s);
    }
    // Launches steps 2-7 for `count` prepared inputs, or, given the SoA conserved
    // rows of a pure fluid (cons, stride), forms the inputs first: inside the
    // single-phase pass when the two-phase bound is on, else with
    // inputsFromConserved.
    void launchSearch(size_t count, const ReactiveThermoState* seed, ReactiveThermoState* state,
                      ReactiveTransportState* transport, int* success, cudaStream_t s,
                      const double* cons = nullptr, size_t stride = 0) {
        check(cudaMemsetAsync(counters, 0, NCOUNTERS * sizeof(unsigned), s), "memset counters");
        const unsigned* selectList = !hostConst.stableGasPrune && hostConst.domeN ? list : nullptr;
        const bool fused = cons && !hostConst.stableGasPrune && hostConst.domeN;
        if (cons && !fused) {
            inputsFromConserved<<<gridFor(count, 256), 256, 0, s>>>(cst, cons, stride, count, 1, seed, in);
            check(cudaGetLastError(), "inputs");
        }
        if (hostConst.stableGasPrune) {
            // all-gas and all-liquid first; the seeds only for cells the gas does not decide
            passQueue<<<passBlocks, kPassThreads, 0, s>>>(cst, in, count, nullptr, 0, 2, rec, counters, Q_A, totals);
            check(cudaGetLastError(), "passQueue");
            compactSeedCells<<<gridFor(count, 256), 256, 0, s>>>(cst, rec, count, list, counters);
            check(cudaGetLastError(), "compactSeedCells");
            passQueue<<<passBlocks, kPassThreads, 0, s>>>(cst, in, count, list, 2, 5, rec, counters, Q_B, totals);
            check(cudaGetLastError(), "passQueue");
        } else if (hostConst.domeN) {
            // single-phase cells one thread each (selected and written there), the
            // rest through the work queue and the selection below
            if (fused)
                passSinglePhase<true><<<passBlocks, kPassThreads, 0, s>>>(cst, in, cons, stride, seed, count, state,
                                                                          transport, success, list, fallback,
                                                                          counters, totals);
            else
                passSinglePhase<false><<<passBlocks, kPassThreads, 0, s>>>(cst, in, nullptr, 0, nullptr, count, state,
                                                                           transport, success, list, fallback,
                                                                           counters, totals);
            check(cudaGetLastError(), "passSinglePhase");
            passQueue<<<passBlocks, kPassThreads, 0, s>>>(cst, in, count, list, 0, 7, rec, counters, Q_A, totals);
            check(cudaGetLastError(), "passQueue");
        } else {
            passQueue<<<passBlocks, kPassThreads, 0, s>>>(cst, in, count, nullptr, 0, 7, rec, counters, Q_A, totals);
            check(cudaGetLastError(), "passQueue");
        }
        selectCandidates<<<gridFor(count, 256), 256, 0, s>>>(cst, rec, count, selectList, state, transport, success,
                                                             fallback, counters);
        check(cudaGetLastError(), "selectCandidates");
        passRestarts<<<passBlocks, kPassThreads, 0, s>>>(cst, in, fallback, fb, capacity, counters, totals);
        check(cudaGetLastError(), "passRestarts");
        selectRestarts<<<gridFor(count, 256), 256, 0, s>>>(fb, capacity, fallback, seed, state, transport, success,
                                                           counters);
        check(cudaGetLastError(), "selectRestarts");
    }
};

// The two-phase admissibility bound of a pure fluid (HemConst::dome*): the
// saturation tie lines on 4,096 temperatures from the liquid range's lower end
// to its critical end, then per point of a 8,192-point log grid in specific
// volume the largest and smallest specific internal energy of the tie lines
// through it (and of the tie-line ends between it and its neighbours). Tie
// lines are straight in (v, u) with positive slope, so an interval's extremes
// sit at its ends or at a tie line's end inside it. The tie lines above the
// last resolved temperature lie in the box of the last one. Margins: 1e-3 of
// the largest latent energy plus ten energy tolerances, 1e-4 plus ten volume
// tolerances in v. Not built (no bound) for two tables, a loose chemical
// tolerance, a liquid range past the cubic's critical temperature, or any
// unresolved temperature below the last resolved one. The same tie lines give
// the saturation-pressure table of the all-gas stability shortcut
// (gasStableBelowSaturation), which lives and switches with the bound.
void buildDome(HemDevice& d) {
    HemConst& C = d.hostConst;
    C.domeN = 0;
    const PureSpecies& sp = C.gas;
    const double Tcm = sp.a * kOmegaB / (sp.b * kOmegaA * kGas);
    const double T0 = std::max(C.Tmin, C.liquidTmin), T1 = std::min(C.Tmax, C.liquidTc * (1 - 1e-10));
    if (!C.samePure || !(C.mutol <= 1e-5) || !(C.liquidTc * (1 - 1e-10) <= Tcm) || !(T1 > T0)) return;
    constexpr int nT = 4096, nV = 8192;
    const double dT = (T1 - T0) / (nT - 1);
    double* dev = nullptr;
    check(cudaMalloc(&dev, sizeof(double) * kSatFields * nT), "cudaMalloc");
    domeSaturation<<<nT / 128, 128, 0, d.stream>>>(d.cst, nT, T0, dT, dev);
    std::vector<double> t(kSatFields * nT);
    cudaError_t e1 = cudaGetLastError();
    cudaError_t e2 = cudaMemcpyAsync(t.data(), dev, sizeof(double) * kSatFields * nT, cudaMemcpyDeviceToHost,
                                     d.stream);
    cudaError_t e3 = cudaStreamSynchronize(d.stream);
    cudaFree(dev);
    check(e1, "domeSaturation");
    check(e2, "D2H dome");
    check(e3, "sync");
    int last = -1;
    for (int i = 0; i < nT; ++i)
        if (t[kSatFields * i] == 1) {
            if (last != i - 1) return;  // a gap below a resolved temperature
            last = i;
        }
    if (last < 1 || last < nT - 8) return;
    double vlo = HUGE_VAL, vhi = 0, latent = 0;
    for (int i = 0; i <= last; ++i) {
        vlo = std::min(vlo, t[kSatFields * i + 1]);
        vhi = std::max(vhi, t[kSatFields * i + 2]);
        latent = std::max(latent, t[kSatFields * i + 4] - t[kSatFields * i + 3]);
    }
    if (!(vlo > 0 && vhi > vlo && latent > 0)) return;
    const double lnV0 = std::log(vlo), step = std::log(vhi / vlo) / (nV - 1);
    std::vector<double> up(nV, -HUGE_VAL), lo(nV, HUGE_VAL), vgrid(nV);
    for (int j = 0; j < nV; ++j) vgrid[j] = std::exp(lnV0 + j * step);
    auto index = [&](double v) { return int(std::floor((std::log(v) - lnV0) / step)); };
    auto touch = [&](int j, double u) {
        for (int k = j; k <= j + 1; ++k)
            if (k >= 0 && k < nV) { up[k] = std::max(up[k], u); lo[k] = std::min(lo[k], u); }
    };
    for (int i = 0; i <= last; ++i) {
        const double* ti = &t[kSatFields * i];
        const double vl = ti[1], vg = ti[2], ul = ti[3], ug = ti[4];
        for (int j = std::max(0, index(vl)); j <= std::min(nV - 1, index(vg) + 1); ++j) {
            const double vj = vgrid[j];
            if (vj < vl || vj > vg) continue;
            const double u = ul + (ug - ul) * (vj - vl) / (vg - vl);
            up[j] = std::max(up[j], u);
            lo[j] = std::min(lo[j], u);
        }
        touch(index(vl), ul);
        touch(index(vg), ug);
    }
    {  // the critical end above the last resolved temperature
        const double* tl = &t[kSatFields * last];
        const double vl = tl[1], vg = tl[2], ul = tl[3], ug = tl[4];
        for (int j = std::max(0, index(vl)); j <= std::min(nV - 1, index(vg) + 1); ++j) {
            up[j] = std::max(up[j], ug);
            lo[j] = std::min(lo[j], ul);
        }
    }
    std::vector<double> packed(2 * nV + nT, 0.0);
    std::copy(up.begin(), up.end(), packed.begin());
    std::copy(lo.begin(), lo.end(), packed.begin() + nV);
    // saturation pressures where the phases are well apart (Z_g - Z_l >= 0.05)
    for (int i = 0; i <= last; ++i) {
        const double T = T0 + dT * i, p = t[kSatFields * i + 5];
        const double dz = p * sp.W * (t[kSatFields * i + 2] - t[kSatFields * i + 1]) / (kGas * T);
        if (p > 0 && dz >= .05) packed[2 * nV + i] = p;
    }
    double* table = d.alloc<double>(2 * nV + nT);
    check(cudaMemcpyAsync(table, packed.data(), sizeof(double) * (2 * nV + nT), cudaMemcpyHostToDevice, d.stream),
          "H2D dome");
    C.domeUp = table;
    C.domeLo = table + nV;
    C.domeLnV0 = lnV0;
    C.domeInvStep = 1 / step;
    C.domeVlo = vlo;
    C.domeVhi = vhi;
    C.domeMarginU = 1e-3 * latent + 10 * C.etol * std::max(1e5, 2000 * C.Tmax);
    C.domeMarginV = 1e-4 + 10 * C.vtol;
    C.domeN = nV;
    C.satP = table + 2 * nV;
    C.satN = nT;
    C.satT0 = T0;
    C.satInvStep = 1 / dT;
    d.domeBuilt = nV;
    check(cudaMemcpyAsync(d.cst, &C, sizeof(HemConst), cudaMemcpyHostToDevice, d.stream), "H2D constants");
    check(cudaStreamSynchronize(d.stream), "sync");
}

void* create(const void* raw, size_t bytes, size_t capacity, bool hostPath, char* error, size_t size) {
    try {
        require(raw && bytes == sizeof(ReactiveB200HemModel) && capacity && capacity <= UINT32_MAX / 8,
                "Invalid CUDA HEM model/capacity");
        ReactiveB200HemModel m;
        std::memcpy(&m, raw, sizeof(m));
        std::unique_ptr<HemDevice> d(new HemDevice);
        const std::string why = validateAndDerive(m, d->hostConst);
        int count = 0;
        check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
        require(count > 0, "No CUDA device");
        check(cudaGetDevice(&d->device), "cudaGetDevice");
        if (!why.empty()) {
            // not the pure-fluid scope: the multi-species flash, if the image is within its scope
            std::string whyMixture;
            d->mixture = mixtureCreate(m, capacity, d->device, whyMixture);
            if (!d->mixture) throw std::runtime_error(why + "; " + whyMixture);
            d->capacity = capacity;
            d->bytes = mixtureDeviceBytes(d->mixture);
            return d.release();
        }
        check(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        d->capacity = capacity;
        d->image.reset(new ReactiveB200HemModel(m));
        d->cst = d->alloc<HemConst>(1);
        d->in = d->alloc<CellInput>(capacity);
        d->rec = d->alloc<CandRecord>(7 * capacity);
        d->fb = d->alloc<CandRecord>(4 * capacity);
        d->list = d->alloc<unsigned>(capacity);
        d->fallback = d->alloc<unsigned>(capacity);
        d->counters = d->alloc<unsigned>(NCOUNTERS);
        d->totals = d->alloc<unsigned long long>(NTOTALS);
        check(cudaMemcpyAsync(d->cst, &d->hostConst, sizeof(HemConst), cudaMemcpyHostToDevice, d->stream), "H2D");
        check(cudaMemsetAsync(d->totals, 0, NTOTALS * sizeof(unsigned long long), d->stream), "memset");
        int perSm = 0, sms = 0;
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, passQueue, kPassThreads, 0), "occupancy");
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device), "attribute");
        d->passBlocks = std::max(1, perSm) * std::max(1, sms);
        if (hostPath) d->ensureHostPath();
        buildDome(*d);
        check(cudaStreamSynchronize(d->stream), "sync");
        return d.release();
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return nullptr;
    }
}

// Model validation (the reference's validModel, src/reactiveThermo/reactiveDeviceFlash.h:80-108,
// for the tables this build evaluates) and the derived device constants.
bool finiteD(double x) { return std::isfinite(x); }

std::string species(const ReactiveB200Table& t, PureSpecies& sp) {
    if (t.ns != 1) return "HEM table must hold one species";
    const ReactiveB200Species& s = t.species[0];
    if (!finiteD(t.refPressure) || t.refPressure <= 0) return "Invalid HEM table reference pressure";
    if (!finiteD(s.molecularWeight) || s.molecularWeight <= 0 || !finiteD(s.a) || s.a <= 0 || !finiteD(s.b)
        || s.b <= 0 || !finiteD(s.kappa) || s.regionCount <= 0 || s.regionCount > kMaxRegions)
        return "Invalid HEM species data";
    if (t.aBinary[0][0] != s.a) return "Invalid HEM binary a";
    sp.a = s.a; sp.b = s.b; sp.kappa = s.kappa; sp.W = s.molecularWeight; sp.refP = t.refPressure;
    sp.Tc = s.a * kOmegaB / (s.b * kOmegaA * kGas);
    sp.invW = 1.0 / sp.W;
    sp.invL = 1.0 / (2.0 * kSqrt2 * sp.b);
    sp.invL2 = 1.0 / (2.0 * kSqrt2 * sp.b * sp.b);
    sp.invTc = 1.0 / sp.Tc;
    sp.invRefP = 1.0 / sp.refP;
    {
        const double pc = kOmegaB * kGas * sp.Tc / sp.b;
        sp.vc = kOmegaVc * kGas * sp.Tc / pc;
    }
    sp.regionCount = s.regionCount;
    for (int r = 0; r < s.regionCount; ++r) {
        const auto& g = s.regions[r];
        if ((g.polynomial != 7 && g.polynomial != 9) || !finiteD(g.minimumTemperature)
            || !finiteD(g.maximumTemperature) || g.minimumTemperature <= 0
            || g.maximumTemperature <= g.minimumTemperature
            || (r && g.minimumTemperature < s.regions[r - 1].minimumTemperature))
            return "Invalid HEM NASA region";
        for (int j = 0; j < g.polynomial; ++j) if (!finiteD(g.coefficient[j])) return "Invalid HEM NASA coefficient";
        sp.polynomial[r] = g.polynomial;
        sp.regionMin[r] = g.minimumTemperature;
        for (int j = 0; j < 9; ++j) sp.coeff[r][j] = g.coefficient[j];
    }
    sp.regionMaxLast = s.regions[s.regionCount - 1].maximumTemperature;
    return "";
}

// Host copy of the pure-fluid cubic used only to place the reported-phase line
// (same relations as the device code, evaluated once per table).
struct HostRoots { double lo; int signedCount; bool ok; };
HostRoots hostRoots(const PureSpecies& sp, double T, double p) {
    HostRoots out{0, 0, false};
    const double sq = std::sqrt(T / sp.Tc), f = 1.0 + sp.kappa * (1.0 - sq);
    if (std::fabs(f) <= 1e-14) return out;
    const double q0 = std::fabs(f), aa = sp.a * q0 * q0;
    const double b = sp.b, b2 = b * b, RTp = kGas * T / p, aap = aa / p, bn = b - RTp;
    const double cn = -(2.0 * RTp * b - aap + 3.0 * b2), dn = b2 * RTp + b2 * b - aap * b;
    const double center = -bn / 3.0, delta2 = (bn * bn - 3.0 * cn) / 9.0;
    const double q = 2.0 * bn * bn * bn / 27.0 - bn * cn / 3.0 + dn;
    const double delta = delta2 > 0 ? std::sqrt(delta2) : 0, h = 2.0 * delta * delta2;
    double disc = q * q - h * h;
    if (std::fabs(std::fabs(h) - std::fabs(q)) < 1e-10) {
        if (disc > 1e-10) return out;
        disc = 0;
    }
    auto cubic = [&](double V) { return ((V + bn) * V + cn) * V + dn; };
    auto polish = [&](double x) {
        for (int n = 0; n < 12; ++n) {
            const double r = cubic(x), d = (3.0 * x + 2.0 * bn) * x + cn;
            if (std::fabs(d) <= 1e-300) break;
            const double step = r / d;
            x -= step;
            if (std::fabs(step) <= 4e-15 * std::max(1.0, std::fabs(x))) break;
        }
        return x;
    };
    std::vector<double> raw;
    int side = 0;
    if (std::fabs(disc) < 1e-14) {
        if (!(delta2 > 0) || q == 0) return out;
        const bool gasSide = q < 0;
        const double pair = center + (gasSide ? -1.0 : 1.0) * delta;
        double x = center + (gasSide ? 2.0 : -2.0) * delta;
        bool conv = false;
        for (int n = 0; n < 24; ++n) {
            const double fx = cubic(x), dfx = (3.0 * x + 2.0 * bn) * x + cn;
            if (!std::isfinite(fx) || !std::isfinite(dfx) || std::fabs(dfx) <= 1e-300) return out;
            const double step = fx / dfx;
            x -= step;
            if (std::fabs(step) <= 4e-15 * std::max(1.0, std::fabs(x))) { conv = true; break; }
        }
        if (!conv || !(x > b) || !(std::fabs(x - pair) > 1e-3 * std::max(std::fabs(x), std::fabs(pair)))) return out;
        raw.push_back(x);
        side = gasSide ? 1 : -1;
    } else if (disc > 1e-14 || !(delta2 > 0)) {
        const double sd = .5 * std::sqrt(std::max(0.0, disc));
        raw.push_back(polish(center + std::cbrt(-.5 * q + sd) + std::cbrt(-.5 * q - sd)));
    } else {
        const double arg = std::min(1.0, std::max(-1.0, -.5 * q / (delta * delta * delta)));
        const double theta = std::acos(arg) / 3.0;
        for (int i = 0; i < 3; ++i) raw.push_back(polish(center + 2.0 * delta * std::cos(theta + i * 2.0 * kPi / 3.0)));
    }
    std::sort(raw.begin(), raw.end());
    std::vector<double> phys;
    for (double v : raw) if (std::isfinite(v) && v > b) phys.push_back(v);
    if (phys.empty()) return out;
    out.lo = phys[0];
    out.ok = true;
    if (side) out.signedCount = side;
    else if (phys.size() >= 2) out.signedCount = int(phys.size());
    else {
        const double Tcm = sp.Tc, pc = kOmegaB * kGas * Tcm / b, vc = kOmegaVc * kGas * Tcm / pc;
        out.signedCount = (T > Tcm ? phys[0] < vc : phys[0] < center) ? -1 : 1;
    }
    return out;
}

std::string phaseLine(PureSpecies& sp) {
    const double tc = sp.a * kOmegaB / (sp.b * kOmegaA * kGas), pc = kOmegaB * kGas * tc / sp.b;
    const double vc = kOmegaVc * kGas * tc / pc;
    double tmid = tc - 100.0;
    if (tmid < 0) tmid = .5 * tc;
    const double ratio = tc / tmid;
    double pp = pc * std::exp(-.8734 * ratio * ratio - 3.4522 * ratio + 4.2918), liquidVolume = -1;
    bool found = false;
    for (int it = 0; it < 100; ++it) {
        const HostRoots r = hostRoots(sp, tmid, pp);
        if (!r.ok) return "HEM reported-phase construction failed";
        if (r.signedCount == 1 || r.signedCount == 2) {
            found = pp > pc;
            liquidVolume = r.lo;
            pp *= 1.04;
            if (found) break;
        } else {
            liquidVolume = r.lo;
            found = true;
            break;
        }
    }
    if (!found || !(liquidVolume > 0)) return "HEM reported-phase construction failed";
    const double rc = sp.W / vc, rl = sp.W / liquidVolume, rg = sp.W / (kGas * tmid / pp);
    sp.tcLine = tc;
    sp.rhoC = rc;
    sp.dRho = rc - .5 * (rl + rg);
    sp.dT = tc - tmid;
    return std::isfinite(sp.dRho) && sp.dT > 0 ? "" : "HEM reported-phase construction failed";
}

std::string validateAndDerive(const ReactiveB200HemModel& m, HemConst& C) {
    if (m.ns != 1 || m.nl != 1 || m.condensable[0] != 0 || m.condensedKind[0] != 0 || m.condensedKind[1] != 0
        || m.boundaryRecovery != 0)
        return "HEM model outside this build's scope: one condensable species with its own pure liquid "
               "(ns=1, nl=1, no solid, boundaryRecovery=0)";
    if ((m.scalarRecovery != 0 && m.scalarRecovery != 1) || (m.analyticJacobian != 0 && m.analyticJacobian != 1)
        || (m.stableGasPrune != 0 && m.stableGasPrune != 1)
        || (m.enforceSpeciesTemperatureBounds != 0 && m.enforceSpeciesTemperatureBounds != 1))
        return "Invalid CUDA HEM model flags";
    if (!finiteD(m.Tmin) || !finiteD(m.Tmax) || !(m.Tmin > 0 && m.Tmax > m.Tmin) || !finiteD(m.pmin)
        || !finiteD(m.pmax) || !(m.pmin > 0 && m.pmax > m.pmin) || !(m.vtol > 0 && m.etol > 0 && m.mutol > 0)
        || !finiteD(m.vtol) || !finiteD(m.etol) || !finiteD(m.mutol))
        return "Invalid CUDA HEM model tables or domain";
    std::string why = species(m.phase[0], C.gas);
    if (why.empty()) why = species(m.phase[1], C.liq);
    if (!why.empty()) return why;
    if (m.weights[0] != m.phase[0].species[0].molecularWeight
        || m.phase[1].species[0].molecularWeight != m.weights[0])
        return "Invalid CUDA HEM species weights";
    if (!finiteD(m.liquidTmin[0]) || !finiteD(m.liquidTc[0]) || !(m.liquidTmin[0] > 0 && m.liquidTc[0] > m.liquidTmin[0]))
        return "Invalid CUDA HEM liquid range";
    why = phaseLine(C.gas);
    if (why.empty()) why = phaseLine(C.liq);
    if (!why.empty()) return why;
    C.Tmin = m.Tmin; C.Tmax = m.Tmax; C.pmin = m.pmin; C.pmax = m.pmax;
    C.vtol = m.vtol; C.etol = m.etol; C.mutol = m.mutol;
    C.liquidTmin = m.liquidTmin[0]; C.liquidTc = m.liquidTc[0];
    C.gasTmin = m.phase[0].species[0].regions[0].minimumTemperature;
    C.gasTmax = C.gas.regionMaxLast;
    C.enforceBounds = m.enforceSpeciesTemperatureBounds;
    C.scalarRecovery = m.scalarRecovery;
    C.analyticJacobian = m.analyticJacobian;
    C.stableGasPrune = m.stableGasPrune;
    C.samePure = std::memcmp(&C.gas, &C.liq, sizeof(PureSpecies)) == 0;
    // The line rho_mid(T) = rho_c + (T - Tc) dRho/dT is >= rho_c below Tc when dRho <= 0 (dT > 0).
    C.liquidFloor = (C.liq.dRho <= 0 && C.liquidTc * (1 - 1e-10) <= C.liq.tcLine) ? C.liq.rhoC * (1 - C.vtol) : 0.0;
    return "";
}

void readTotals(HemDevice& d, ReactiveGpuHemProfileV1& p, cudaStream_t s, unsigned long long* succeeded = nullptr) {
    unsigned long long t[NTOTALS] = {};
    unsigned ctr[NCOUNTERS] = {};
    check(cudaMemcpyAsync(t, d.totals, sizeof(t), cudaMemcpyDeviceToHost, s), "D2H totals");
    check(cudaMemcpyAsync(ctr, d.counters, sizeof(ctr), cudaMemcpyDeviceToHost, s), "D2H counters");
    check(cudaStreamSynchronize(s), "sync");
    check(cudaMemsetAsync(d.totals, 0, sizeof(t), s), "memset totals");
    p.phaseEvaluations = t[T_PHASES];
    p.residualEvaluations = t[T_RESIDUALS];
    p.flashCandidates = t[T_CANDIDATES];
    p.stableCandidates = t[T_STABLE];
    p.analyticJacobians = t[T_ANALYTIC];
    p.finiteDifferenceJacobians = t[T_FD];
    p.deviceFailures = ctr[FAILED];
    if (succeeded) *succeeded = t[T_SUCCEEDED];
}

}  // namespace
}  // namespace rb200

using rb200::HemDevice;

extern "C" {

const char* reactive_gpu_hem_numerical_policy_v1(void) {
    return "fp64-fma-rn-candidate-parallel-v1:prec-div=true:prec-sqrt=true:fast-math=false";
}
void* reactive_gpu_hem_create_v1(const void* model, size_t bytes, size_t capacity, char* error, size_t size) {
    return rb200::create(model, bytes, capacity, true, error, size);
}
void* reactive_gpu_hem_create_resident_v1(const void* model, size_t bytes, size_t capacity, char* error,
                                          size_t size) {
    return rb200::create(model, bytes, capacity, false, error, size);
}
size_t reactive_gpu_hem_device_bytes_v1(void* raw) { return raw ? static_cast<HemDevice*>(raw)->bytes : 0; }
void reactive_gpu_hem_destroy_v1(void* raw) { delete static_cast<HemDevice*>(raw); }

int reactive_gpu_hem_run_v1(void* raw, const double* q, const double* energy, size_t count, ReactiveThermoState* states,
                            int* success, ReactiveGpuHemProfileV1* profile, char* error, size_t size) {
    try {
        rb200::require(raw && q && energy && states && success && profile && profile->abiVersion == 1
                           && profile->structBytes == sizeof(*profile),
                       "Invalid CUDA HEM batch arguments");
        auto& d = *static_cast<HemDevice*>(raw);
        std::lock_guard<std::mutex> lock(d.entry);
        rb200::require(count && count <= d.capacity, "CUDA HEM batch exceeds capacity");
        rb200::check(cudaSetDevice(d.device), "cudaSetDevice");
        if (d.mixture) {
            ReactiveGpuHemProfileV1 p{};
            p.abiVersion = 1;
            p.structBytes = sizeof(p);
            rb200::mixtureRun(d.mixture, q, energy, count, nullptr, states, success, p);
            *profile = p;
            return 0;
        }
        d.ensureHostPath();
        const auto begin = std::chrono::steady_clock::now();
        // Pipelined in chunks of at least 256Ki cells (up to 16): the uploads of
        // later chunks (copy stream up) and the downloads of finished ones (copy
        // stream down) overlap the flash of the current chunk; the chunks'
        // flashes run one after another on the handle's stream (they share the
        // queue scratch).
        const size_t chunks = std::min<size_t>(16, std::max<size_t>(1, count >> 18));
        const size_t per = (count + chunks - 1) / chunks;
        cudaStream_t s = d.stream;
        std::vector<cudaEvent_t> uploaded(chunks), computed(chunks);
        cudaEvent_t start, end, first, last;
        for (auto* e : {&start, &end, &first, &last}) rb200::check(cudaEventCreate(e), "event");
        for (size_t i = 0; i < chunks; ++i) {
            rb200::check(cudaEventCreateWithFlags(&uploaded[i], cudaEventDisableTiming), "event");
            rb200::check(cudaEventCreateWithFlags(&computed[i], cudaEventDisableTiming), "event");
        }
        rb200::check(cudaEventRecord(start, d.up), "event");
        for (size_t i = 0; i < chunks; ++i) {
            const size_t off = i * per, n = std::min(per, count - off);
            rb200::check(cudaMemcpyAsync(d.dq + off, q + off, n * sizeof(double), cudaMemcpyHostToDevice, d.up), "H2D q");
            rb200::check(cudaMemcpyAsync(d.de + off, energy + off, n * sizeof(double), cudaMemcpyHostToDevice, d.up),
                         "H2D e");
            rb200::check(cudaMemcpyAsync(d.dguess + off, states + off, n * sizeof(ReactiveThermoState),
                                         cudaMemcpyHostToDevice, d.up), "H2D seed");
            rb200::check(cudaEventRecord(uploaded[i], d.up), "event");
        }
        for (size_t i = 0; i < chunks; ++i) {
            const size_t off = i * per, n = std::min(per, count - off);
            rb200::check(cudaStreamWaitEvent(s, uploaded[i], 0), "wait");
            if (i == 0) rb200::check(cudaEventRecord(first, s), "event");
            rb200::check(cudaMemsetAsync(d.dsuccess + off, 0, n * sizeof(int), s), "memset");
            rb200::inputsFromHost<<<rb200::gridFor(n, 256), 256, 0, s>>>(d.cst, d.dq + off, d.de + off, d.dguess + off,
                                                                         n, 1,
                                                                         d.in);
            rb200::check(cudaGetLastError(), "inputs");
            d.launchSearch(n, d.dguess + off, d.dout + off, nullptr, d.dsuccess + off, s);
            // a failed cell leaves the caller's state unchanged: its seed goes back
            rb200::keepFailed<<<rb200::gridFor(n, 256), 256, 0, s>>>(d.dguess + off, d.dsuccess + off, n,
                                                                     d.dout + off, d.totals + rb200::T_SUCCEEDED);
            rb200::check(cudaGetLastError(), "keepFailed");
            rb200::check(cudaEventRecord(computed[i], s), "event");
            if (i + 1 == chunks) rb200::check(cudaEventRecord(last, s), "event");
            rb200::check(cudaStreamWaitEvent(d.down, computed[i], 0), "wait");
            rb200::check(cudaMemcpyAsync(states + off, d.dout + off, n * sizeof(ReactiveThermoState),
                                         cudaMemcpyDeviceToHost, d.down), "D2H states");
            rb200::check(cudaMemcpyAsync(success + off, d.dsuccess + off, n * sizeof(int), cudaMemcpyDeviceToHost,
                                         d.down), "D2H success");
        }
        rb200::check(cudaEventRecord(end, d.down), "event");
        rb200::check(cudaEventSynchronize(end), "sync");
        ReactiveGpuHemProfileV1 p{};
        p.abiVersion = 1;
        p.structBytes = sizeof(p);
        unsigned long long succeeded = 0;
        rb200::readTotals(d, p, s, &succeeded);
        float total = 0, kernel = 0;
        cudaEventElapsedTime(&total, start, end);
        cudaEventElapsedTime(&kernel, first, last);
        for (auto e : {start, end, first, last}) cudaEventDestroy(e);
        for (size_t i = 0; i < chunks; ++i) { cudaEventDestroy(uploaded[i]); cudaEventDestroy(computed[i]); }
        p.batches = 1;
        p.submitted = count;
        p.succeeded = succeeded;
        p.deviceFailures = count - p.succeeded;
        p.transferBytes = count * (2 * sizeof(double) + 2 * sizeof(ReactiveThermoState) + sizeof(int));
        p.deviceBytes = d.bytes;
        p.hostBytes = count * sizeof(ReactiveThermoState);
        p.kernelSeconds = kernel / 1000.;
        p.copySeconds = std::max(0.f, total - kernel) / 1000.;  // copy time not hidden behind the flash
        p.wallSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
        *profile = p;
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}

// src/reactiveTransport/reactiveGpuHem.cuh:354-358, 227-241: the capillary
// batch. Every cell is the reference's capillary recovery (recoverCapillary):
// the gas at p - color*jump, the liquid at p + (1 - color)*jump, UV equilibrium
// with the boundary search, or the frozen partition at the seed's liquid masses.
// It runs on the multi-species engine (hem_mixture.cu), for a pure-fluid handle
// one made from the same image. A pure-fluid image outside that engine's scope
// takes equilibrium batches without a jump on its own fast path (the plain UV
// flash) and refuses the rest.
int reactive_gpu_hem_run_v2(void* raw, const double* q, const double* energy,
                            const ReactiveGpuHemCapillaryInputV2* capillary, size_t count, ReactiveThermoState* states,
                            int* success, ReactiveGpuHemProfileV1* profile, char* error, size_t size) {
    try {
        rb200::require(capillary != nullptr, "Null CUDA HEM capillary input");
        rb200::require(raw && q && energy && states && success && profile && profile->abiVersion == 1
                           && profile->structBytes == sizeof(*profile),
                       "Invalid CUDA HEM batch arguments");
        auto& d = *static_cast<HemDevice*>(raw);
        bool plain = true;
        for (size_t c = 0; c < count; ++c) {
            const auto& in = capillary[c];
            rb200::require(std::isfinite(in.color) && in.color >= 0 && in.color <= 1 && std::isfinite(in.pressureJump)
                               && (in.equilibrium == 0 || in.equilibrium == 1),
                           "Invalid CUDA HEM capillary cell input");
            plain = plain && in.pressureJump == 0.0 && in.equilibrium == 1;
        }
        rb200::MixtureFlash* engine = nullptr;
        {
            std::lock_guard<std::mutex> lock(d.entry);
            rb200::require(count && count <= d.capacity, "CUDA HEM batch exceeds capacity");
            rb200::check(cudaSetDevice(d.device), "cudaSetDevice");
            engine = d.capillaryFlash();
            if (engine) {
                ReactiveGpuHemProfileV1 p{};
                p.abiVersion = 1;
                p.structBytes = sizeof(p);
                rb200::mixtureRun(engine, q, energy, count, capillary, states, success, p);
                *profile = p;
                return 0;
            }
        }
        rb200::require(plain, "Capillary pressure jumps and the frozen partition need a model image within the "
                              "multi-species flash's scope");
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
    return reactive_gpu_hem_run_v1(raw, q, energy, count, states, success, profile, error, size);
}
// src/reactiveTransport/reactiveGpuHem.cuh:403-408: the capillary primitive
// initialisation (every record's equilibrium 0) on the multi-species engine.
int reactive_gpu_hem_initialize_tp_v1(void* raw, double* q, double* energy,
                                      const ReactiveGpuHemCapillaryInputV2* capillary, size_t count,
                                      ReactiveThermoState* states, int* success, ReactiveGpuHemProfileV1* profile,
                                      char* error, size_t size) {
    try {
        rb200::require(q && energy && capillary, "Null CUDA primitive input");
        rb200::require(raw && states && success && profile && profile->abiVersion == 1
                           && profile->structBytes == sizeof(*profile),
                       "Invalid CUDA HEM batch arguments");
        auto& d = *static_cast<HemDevice*>(raw);
        for (size_t c = 0; c < count; ++c) {
            const auto& in = capillary[c];
            rb200::require(std::isfinite(in.color) && in.color >= 0 && in.color <= 1 && std::isfinite(in.pressureJump)
                               && in.equilibrium == 0,
                           "Invalid CUDA HEM capillary cell input");
        }
        std::lock_guard<std::mutex> lock(d.entry);
        rb200::require(count && count <= d.capacity, "CUDA HEM batch exceeds capacity");
        rb200::check(cudaSetDevice(d.device), "cudaSetDevice");
        rb200::MixtureFlash* engine = d.capillaryFlash();
        rb200::require(engine, "Capillary primitive initialisation needs a model image within the multi-species "
                               "flash's scope");
        ReactiveGpuHemProfileV1 p{};
        p.abiVersion = 1;
        p.structBytes = sizeof(p);
        rb200::mixtureInitialize(engine, q, energy, count, capillary, states, success, p);
        *profile = p;
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}
// The reference's device-resident batch (src/reactiveThermo/reactiveGpuHem.h:72-84).
// With capillary records (or a multi-species handle) it runs on the
// multi-species engine; a pure-fluid image outside that engine's scope takes
// UV equilibrium without a pressure jump (capillary NULL, or pressureJump = 0
// and equilibrium = 1 for every named cell) on its fast path: gather the named
// cells, the work-queue search, failed cells keep their seed, scatter to
// output[cell]. Synchronous on the handle's stream; only batch totals reach
// the host.
int reactive_gpu_hem_run_resident_v1(void* raw, const double* q, const double* energy, const ReactiveThermoState* seed,
                                     const ReactiveGpuHemCapillaryInputV2* capillary, const uint32_t* order,
                                     size_t count, ReactiveGpuHemOutputV1* output, ReactiveGpuHemProfileV1* profile,
                                     char* error, size_t size) {
    try {
        rb200::require(raw && q && energy && seed && order && output && profile && profile->abiVersion == 1
                           && profile->structBytes == sizeof(*profile),
                       "Invalid resident CUDA HEM batch arguments");
        auto& d = *static_cast<HemDevice*>(raw);
        std::lock_guard<std::mutex> lock(d.entry);
        rb200::require(count && count <= d.capacity, "Resident CUDA HEM batch exceeds capacity");
        rb200::check(cudaSetDevice(d.device), "cudaSetDevice");
        // the capillary recovery (and every batch of a multi-species handle) on the
        // multi-species engine; a pure-fluid image outside its scope keeps the fast path
        rb200::MixtureFlash* engine = d.mixture ? d.mixture : (capillary ? d.capillaryFlash() : nullptr);
        if (engine) {
            ReactiveGpuHemProfileV1 p{};
            p.abiVersion = 1;
            p.structBytes = sizeof(p);
            rb200::mixtureRunResident(engine, q, energy, seed, capillary, order, count, output, p);
            *profile = p;
            return 0;
        }
        d.ensureHostPath();  // gathered seeds, results and flags
        const auto begin = std::chrono::steady_clock::now();
        cudaStream_t s = d.stream;
        unsigned* unsupported = d.counters + rb200::FAILED;  // reset by the search before its own use
        rb200::check(cudaMemsetAsync(unsupported, 0, sizeof(unsigned), s), "memset");
        rb200::inputsFromResident<<<rb200::gridFor(count, 256), 256, 0, s>>>(d.cst, q, energy, seed, capillary, order,
                                                                            count,
                                                                            1, d.in, d.dguess, unsupported);
        rb200::check(cudaGetLastError(), "inputs");
        unsigned flag = 0;
        rb200::check(cudaMemcpyAsync(&flag, unsupported, sizeof(flag), cudaMemcpyDeviceToHost, s), "D2H flag");
        rb200::check(cudaStreamSynchronize(s), "sync");
        rb200::require(!flag, "Capillary pressure jumps and the frozen partition are not part of this B200 build");
        cudaEvent_t first, last;
        rb200::check(cudaEventCreate(&first), "event");
        rb200::check(cudaEventCreate(&last), "event");
        rb200::check(cudaEventRecord(first, s), "event");
        rb200::check(cudaMemsetAsync(d.dsuccess, 0, count * sizeof(int), s), "memset");
        d.launchSearch(count, d.dguess, d.dout, nullptr, d.dsuccess, s);
        rb200::keepFailed<<<rb200::gridFor(count, 256), 256, 0, s>>>(d.dguess, d.dsuccess, count, d.dout);
        rb200::check(cudaGetLastError(), "keepFailed");
        rb200::scatterResident<<<rb200::gridFor(count, 256), 256, 0, s>>>(d.dout, d.dsuccess, order, count, output);
        rb200::check(cudaGetLastError(), "scatter");
        rb200::check(cudaEventRecord(last, s), "event");
        ReactiveGpuHemProfileV1 p{};
        p.abiVersion = 1;
        p.structBytes = sizeof(p);
        rb200::readTotals(d, p, s);  // synchronises
        float kernel = 0;
        cudaEventElapsedTime(&kernel, first, last);
        cudaEventDestroy(first);
        cudaEventDestroy(last);
        p.batches = 1;
        p.submitted = count;
        p.succeeded = count - p.deviceFailures;
        p.deviceBytes = d.bytes;
        p.kernelSeconds = kernel / 1000.;
        p.wallSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
        *profile = p;
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}

int reactive_gpu_hem_run_device_v3(void* raw, const double* conserved, size_t stride, size_t count, size_t variables,
                                   const ReactiveThermoState* seed, ReactiveThermoState* state,
                                   ReactiveTransportState* transport, int* success, void*, int flags, void* stream,
                                   char* error, size_t size) {
    try {
        rb200::require(raw && conserved && seed && (state || transport) && count && stride >= count
                           && variables >= 5,
                       "Invalid device HEM batch arguments");
        auto& d = *static_cast<HemDevice*>(raw);
        rb200::require(!d.mixture, "The multi-species flash runs through reactive_gpu_hem_run_v1, run_v2 and run_resident_v1 only");
        std::lock_guard<std::mutex> lock(d.entry);
        rb200::require(count <= d.capacity, "Device HEM batch exceeds capacity");
        auto s = static_cast<cudaStream_t>(stream);
        if (flags & 2) {
            rb200::inputsFromConserved<<<rb200::gridFor(count, 256), 256, 0, s>>>(d.cst, conserved, stride, count, 1,
                                                                                 seed, d.in);
            rb200::check(cudaGetLastError(), "inputs");
            d.launchPerCell(count, seed, state, transport, success, s);
        } else
            d.launchSearch(count, seed, state, transport, success, s, conserved, stride);
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}

int reactive_gpu_hem_two_phase_bound_v3(void* raw, int request, int* active, char* error, size_t size) {
    try {
        rb200::require(raw && request >= -1 && request <= 1, "Invalid two-phase bound request");
        auto& d = *static_cast<HemDevice*>(raw);
        rb200::require(!d.mixture, "The multi-species flash runs through reactive_gpu_hem_run_v1, run_v2 and run_resident_v1 only");
        std::lock_guard<std::mutex> lock(d.entry);
        rb200::require(request != 1 || d.domeBuilt, "This model has no two-phase bound (see the header)");
        if (request >= 0) {
            d.hostConst.domeN = request ? d.domeBuilt : 0;
            rb200::check(cudaMemcpyAsync(d.cst, &d.hostConst, sizeof(d.hostConst), cudaMemcpyHostToDevice, d.stream),
                         "H2D constants");
            rb200::check(cudaStreamSynchronize(d.stream), "sync");
        }
        if (active) *active = d.hostConst.domeN ? 1 : 0;
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}

int reactive_gpu_hem_vjp_device_v3(void* raw, const double* conserved, size_t stride, size_t count, size_t variables,
                                   const ReactiveThermoState* state, const ReactiveTransportState* transportBar,
                                   double* conservedBar, size_t barStride, unsigned* failed, void* stream, char* error,
                                   size_t size) {
    try {
        rb200::require(raw && conserved && state && transportBar && conservedBar && count && stride >= count
                           && barStride >= count && variables == 5,
                       "Invalid HEM VJP arguments (pure fluid: variables = 5)");
        auto& d = *static_cast<HemDevice*>(raw);
        rb200::require(!d.mixture, "The multi-species flash runs through reactive_gpu_hem_run_v1, run_v2 and run_resident_v1 only");
        std::lock_guard<std::mutex> lock(d.entry);
        auto s = static_cast<cudaStream_t>(stream);
        rb200::hemStateVjp<<<rb200::gridFor(count, 128), 128, 0, s>>>(d.cst, conserved, stride, count, state,
                                                                      transportBar, conservedBar, barStride, failed);
        rb200::check(cudaGetLastError(), "hemStateVjp");
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}

int reactive_gpu_hem_autotune_v3(void* raw, const double* conserved, size_t stride, size_t count, size_t variables,
                                 const ReactiveThermoState* seed, void* stream, int* blocksPerSm, char* error,
                                 size_t size) {
    try {
        rb200::require(raw && conserved && seed && count && stride >= count && variables >= 5,
                       "Invalid HEM autotune arguments");
        auto& d = *static_cast<HemDevice*>(raw);
        rb200::require(!d.mixture, "The multi-species flash runs through reactive_gpu_hem_run_v1, run_v2 and run_resident_v1 only");
        std::lock_guard<std::mutex> lock(d.entry);
        rb200::require(count <= d.capacity, "CUDA HEM batch exceeds capacity");
        rb200::check(cudaSetDevice(d.device), "cudaSetDevice");
        auto s = static_cast<cudaStream_t>(stream);
        int perSm = 0, sms = 0;
        rb200::check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, rb200::passQueue, rb200::kPassThreads, 0),
                     "occupancy");
        rb200::check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d.device), "attribute");
        d.ensureHostPath();  // scratch outputs of the timed runs
        cudaEvent_t a, b;
        rb200::check(cudaEventCreate(&a), "event");
        rb200::check(cudaEventCreate(&b), "event");
        float best = 1e30f;
        int keep = std::max(1, perSm);
        for (int k = 1; k <= std::max(1, perSm); ++k) {
            d.passBlocks = k * sms;
            for (int r = 0; r < 2; ++r) {  // the first run warms up
                rb200::check(cudaEventRecord(a, s), "event");
                d.launchSearch(count, seed, d.dout, nullptr, d.dsuccess, s, conserved, stride);
                rb200::check(cudaEventRecord(b, s), "event");
                rb200::check(cudaEventSynchronize(b), "event");
            }
            float ms = 0;
            rb200::check(cudaEventElapsedTime(&ms, a, b), "event");
            if (ms < best) { best = ms; keep = k; }
        }
        d.passBlocks = keep * sms;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (blocksPerSm) *blocksPerSm = keep;
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}

int reactive_gpu_hem_run_counters_v3(void* raw, ReactiveGpuHemProfileV1* profile, void* stream, char* error,
                                     size_t size) {
    try {
        rb200::require(raw && profile, "Invalid HEM counter query");
        auto& d = *static_cast<HemDevice*>(raw);
        rb200::require(!d.mixture, "The multi-species flash runs through reactive_gpu_hem_run_v1, run_v2 and run_resident_v1 only");
        std::lock_guard<std::mutex> lock(d.entry);
        ReactiveGpuHemProfileV1 p{};
        p.abiVersion = 1;
        p.structBytes = sizeof(p);
        rb200::readTotals(d, p, static_cast<cudaStream_t>(stream));
        p.deviceBytes = d.bytes;
        *profile = p;
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Flash without any allocation, for callers that cannot call cudaMalloc.
//
// Some callers of the HEM cannot allocate device memory when they need a flash:
// a solver that owns the whole device through its own memory pool and forbids
// other allocations. For them this entry point runs the
// same work-queue flash as reactive_gpu_hem_run_device_v3 with no handle: its
// scratch (the derived model constants, per-cell inputs, candidate records,
// lists and queue counters) lives in one file-scope __device__ array sized for
// at most kStaticHemCells cells (about 9 MB). Every GPU that loads this library
// holds that array until the process exits.
//
// Every call looks up the array's device address with cudaGetSymbolAddress for
// the current device (a cheap lookup, and never stale: after a cudaDeviceReset,
// or under another context, the module is loaded again at a new address). The
// first call on a device loads this library's device code there if it is not
// loaded yet and queries the flash kernel's occupancy (kept per device): make
// that first call before capturing any stream. Every call uses the same array
// and finds the previous call's contents there; the queue counters and work
// totals are cleared at the start of each call, and every candidate record a
// call selects from is written by that call. Calls that overlap on the GPU (two
// streams, two host threads) race on the array: serialise them.
namespace rb200 {
namespace {
constexpr size_t kStaticHemCells = 4096;
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kStaticConst = 0;
constexpr size_t kStaticIn = align256(kStaticConst + sizeof(HemConst));
constexpr size_t kStaticRec = align256(kStaticIn + kStaticHemCells * sizeof(CellInput));
constexpr size_t kStaticFb = align256(kStaticRec + 7 * kStaticHemCells * sizeof(CandRecord));
constexpr size_t kStaticList = align256(kStaticFb + 4 * kStaticHemCells * sizeof(CandRecord));
constexpr size_t kStaticFallback = align256(kStaticList + kStaticHemCells * sizeof(unsigned));
constexpr size_t kStaticCounters = align256(kStaticFallback + kStaticHemCells * sizeof(unsigned));
constexpr size_t kStaticTotals = align256(kStaticCounters + NCOUNTERS * sizeof(unsigned));
constexpr size_t kStaticBytes = align256(kStaticTotals + NTOTALS * sizeof(unsigned long long));

static __device__ __align__(256) unsigned char staticHemScratch[kStaticBytes];

std::mutex staticHemMutex;
int staticHemBlocks[64] = {};  // work-queue grid per device ordinal (0: not yet queried)

// Device address of the scratch array on the current device.
unsigned char* staticScratch() {
    void* ptr = nullptr;
    check(cudaGetSymbolAddress(&ptr, staticHemScratch), "cudaGetSymbolAddress(static HEM scratch)");
    require(ptr != nullptr, "Static HEM scratch has no device address");
    return static_cast<unsigned char*>(ptr);
}

// Persistent work-queue grid for the current device (queried once per device).
int staticQueueBlocks() {
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    require(device >= 0 && device < 64, "Device ordinal out of range for the static HEM flash");
    std::lock_guard<std::mutex> lock(staticHemMutex);
    if (!staticHemBlocks[device]) {
        int perSm = 0, sms = 0;
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, passQueue, kPassThreads, 0), "occupancy");
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attribute");
        staticHemBlocks[device] = std::max(1, perSm) * std::max(1, sms);
    }
    return staticHemBlocks[device];
}

__global__ void storeConstants(HemConst c, HemConst* dst) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *dst = c;
}
}  // namespace
}  // namespace rb200

extern "C" int reactive_gpu_hem_run_static_v3(const void* model, size_t modelBytes, const double* conserved,
                                              size_t stride, size_t count, size_t variables,
                                              const ReactiveThermoState* seed, ReactiveThermoState* state,
                                              ReactiveTransportState* transport, int* success, void* stream,
                                              char* error, size_t size) {
    using namespace rb200;
    try {
        require(model && modelBytes == sizeof(ReactiveB200HemModel), "Invalid HEM model image");
        require(conserved && seed && (state || transport) && count && stride >= count && variables >= 5,
                "Invalid static HEM batch arguments");
        if (count > kStaticHemCells)
            throw std::runtime_error("Static HEM batch of " + std::to_string(count) + " cells exceeds the maximum of "
                                     + std::to_string(kStaticHemCells) + "; split the batch or use a handle");
        ReactiveB200HemModel m;
        std::memcpy(&m, model, sizeof(m));
        HemConst hostConst{};
        const std::string why = validateAndDerive(m, hostConst);
        require(why.empty(), why.c_str());
        unsigned char* base = staticScratch();
        auto* cst = reinterpret_cast<HemConst*>(base + kStaticConst);
        auto* in = reinterpret_cast<CellInput*>(base + kStaticIn);
        auto* rec = reinterpret_cast<CandRecord*>(base + kStaticRec);
        auto* fb = reinterpret_cast<CandRecord*>(base + kStaticFb);
        auto* list = reinterpret_cast<unsigned*>(base + kStaticList);
        auto* fallback = reinterpret_cast<unsigned*>(base + kStaticFallback);
        auto* counters = reinterpret_cast<unsigned*>(base + kStaticCounters);
        auto* totals = reinterpret_cast<unsigned long long*>(base + kStaticTotals);
        auto s = static_cast<cudaStream_t>(stream);
        const int blocks = staticQueueBlocks();
        storeConstants<<<1, 1, 0, s>>>(hostConst, cst);
        check(cudaGetLastError(), "storeConstants");
        check(cudaMemsetAsync(counters, 0, NCOUNTERS * sizeof(unsigned), s), "clear counters");
        check(cudaMemsetAsync(totals, 0, NTOTALS * sizeof(unsigned long long), s), "clear totals");
        inputsFromConserved<<<gridFor(count, 256), 256, 0, s>>>(cst, conserved, stride, count, 1, seed, in);
        check(cudaGetLastError(), "inputs");
        if (hostConst.stableGasPrune) {
            passQueue<<<blocks, kPassThreads, 0, s>>>(cst, in, count, nullptr, 0, 2, rec, counters, Q_A, totals);
            compactSeedCells<<<gridFor(count, 256), 256, 0, s>>>(cst, rec, count, list, counters);
            passQueue<<<blocks, kPassThreads, 0, s>>>(cst, in, count, list, 2, 5, rec, counters, Q_B, totals);
        } else {
            passQueue<<<blocks, kPassThreads, 0, s>>>(cst, in, count, nullptr, 0, 7, rec, counters, Q_A, totals);
        }
        check(cudaGetLastError(), "passQueue");
        selectCandidates<<<gridFor(count, 256), 256, 0, s>>>(cst, rec, count, nullptr, state, transport, success,
                                                             fallback, counters);
        passRestarts<<<blocks, kPassThreads, 0, s>>>(cst, in, fallback, fb, kStaticHemCells, counters, totals);
        selectRestarts<<<gridFor(count, 256), 256, 0, s>>>(fb, kStaticHemCells, fallback, seed, state, transport,
                                                           success, counters);
        check(cudaGetLastError(), "select");
        return 0;
    } catch (const std::exception& e) {
        if (error && size) std::snprintf(error, size, "%s", e.what());
        return 1;
    }
}
