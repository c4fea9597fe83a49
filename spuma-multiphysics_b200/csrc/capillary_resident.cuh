// Device kernels of the resident capillary closure (the reference's
// reactive_transport_capillary_resident_*_v1, src/reactiveTransport/
// reactiveTransport.cpp:280-360 and :963-1127, over the host closure of
// src/reactiveFoam/reactiveCapillary.H:54-246): the outer iteration between the
// capillary HEM flash and the diffuse interface geometry with every per-cell
// array on the device. Each expression is the host closure's own, so with
// separate rounding (this translation unit's --fmad=false) every value is
// bitwise the host path's. An input the host path would reject only raises a
// flag; the caller then reruns the closure on the host path, which reports it.
#pragma once
#include <cstdint>
#include "../../include/reactive_b200_types.h"

namespace rb200 {
namespace capres {

constexpr unsigned kBadColor = 1u, kBadInput = 2u, kNonFinite = 4u;

__device__ __forceinline__ bool sameBits(double a, double b) {
    return __double_as_longlong(a) == __double_as_longlong(b);
}

// The liquid volume fraction of a recovered state, V_l / (V_l + V_g) from the
// phase masses and densities (reactiveCapillary.H:6-29).
__device__ inline double liquidColor(const ReactiveThermoState& s, unsigned* flags) {
    const double ml = s.liquidMass[0];
    if (!(isfinite(ml) && ml >= 0)) { atomicOr(flags, kBadColor); return 0; }
    double c = 0;
    if (ml > 0) {
        if (!(isfinite(s.rhoLiquid[0]) && s.rhoLiquid[0] > 0)) { atomicOr(flags, kBadColor); return 0; }
        c = ml / s.rhoLiquid[0];
    }
    const double gasVolume = s.gasMass > 0 ? s.gasMass / s.rhoGas : 0;
    const double sum = c + gasVolume;
    if (!(isfinite(sum) && sum > 0 && fabs(sum - 1) < 1e-6)) { atomicOr(flags, kBadColor); return 0; }
    c /= sum;
    if (!(isfinite(c) && c >= 0 && c <= 1)) atomicOr(flags, kBadColor);
    return c;
}

// The HEM scheduling key of a cell (src/reactiveTransport/reactiveHemBucket.h:13-18,
// performance only): active liquids, present species, dominant species.
__device__ inline unsigned hemBucket(const double* q, int ns, int activeLiquids) {
    unsigned present = 0, dominant = 0;
    for (int k = 0; k < ns; ++k) {
        if (q[k] > 0) ++present;
        if (q[k] > q[dominant]) dominant = unsigned(k);
    }
    const unsigned liquids = activeLiquids < 0 ? 0u : (activeLiquids > 3 ? 3u : unsigned(activeLiquids));
    return (liquids << 6) | ((present > 7 ? 7u : present) << 3) | (dominant > 7 ? 7u : dominant);
}

__global__ void identity(size_t n, uint32_t* x) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
        x[c] = uint32_t(c);
}

// The incoming states' color, then each seed carries the transported liquid
// inventory (every outer iteration seeds a cell with the same state).
__global__ void seedStates(size_t n, ReactiveThermoState* seed, const double* liquid, double* color,
                           unsigned* flags) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        color[c] = liquidColor(seed[c], flags);
        seed[c].liquidMass[0] = liquid[c];
    }
}

__global__ void pressureJump(size_t n, double sigma, const double* curvature, double* jump) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
        jump[c] = sigma * curvature[c];
}

// The iteration's inputs (color, jump, surface energy before the flash), the
// flash's bulk energy and capillary record, and the dirty set: every cell at
// iteration 0, later the cells whose three geometry inputs changed bitwise since
// their last flash. keys: dirty cells by heavy-first bucket (255 - bucket), the
// clean ones after them (256). One thread per cell (the ballot needs full warps).
__global__ void selectDirty(size_t n, int all, int equilibrium, int ns, const double* q,
                            const ReactiveThermoState* seed, const double* bulk, const double* color,
                            const double* jump, const double* surface, double* colorBefore, double* jumpBefore,
                            double* energyBefore, const double* flashedColor, const double* flashedJump,
                            const double* flashedEnergy, double* energy, ReactiveGpuHemCapillaryInputV2* capillary,
                            uint16_t* keys, unsigned long long* dirtyCount, unsigned* flags) {
    const size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    bool dirty = false;
    if (c < n) {
        const double cb = color[c], jb = jump[c], eb = surface[c];
        colorBefore[c] = cb;
        jumpBefore[c] = jb;
        energyBefore[c] = eb;
        dirty = all || !sameBits(cb, flashedColor[c]) || !sameBits(jb, flashedJump[c]) || !sameBits(eb, flashedEnergy[c]);
        energy[c] = bulk[c] - eb;
        ReactiveGpuHemCapillaryInputV2 in{};
        in.color = cb;
        in.pressureJump = jb;
        in.equilibrium = equilibrium;
        capillary[c] = in;
        if (!(isfinite(cb) && cb >= 0 && cb <= 1 && isfinite(jb))) atomicOr(flags, kBadInput);
        keys[c] = dirty ? uint16_t(255u - hemBucket(q + c * size_t(ns), ns, seed[c].activeLiquids)) : uint16_t(256u);
    }
    const unsigned mask = __ballot_sync(0xffffffffu, dirty);
    if ((threadIdx.x & 31u) == 0 && mask) atomicAdd(dirtyCount, (unsigned long long)__popc(mask));
}

// The flashed cells record the inputs they were flashed with.
__global__ void recordFlashed(size_t count, const uint32_t* order, const double* colorBefore,
                              const double* jumpBefore, const double* energyBefore, double* flashedColor,
                              double* flashedJump, double* flashedEnergy) {
    for (size_t j = blockIdx.x * size_t(blockDim.x) + threadIdx.x; j < count; j += size_t(gridDim.x) * blockDim.x) {
        const uint32_t c = order[j];
        flashedColor[c] = colorBefore[c];
        flashedJump[c] = jumpBefore[c];
        flashedEnergy[c] = energyBefore[c];
    }
}

// The candidate color of the flashed states.
__global__ void candidateColor(size_t n, const ReactiveGpuHemOutputV1* output, double* color, unsigned* flags) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
        color[c] = liquidColor(output[c].state, flags);
}

__global__ void gatherStates(size_t n, const ReactiveGpuHemOutputV1* output, ReactiveThermoState* states) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
        states[c] = output[c].state;
}

__global__ void relaxColor(size_t n, const double* colorBefore, double* color) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
        color[c] = .5 * (colorBefore[c] + color[c]);
}

// The closure residual: the largest change of color, of surface energy (scaled
// by max(|bulk energy|, 1e5 rho)) and of the pressure jump (scaled by max(p, 1))
// over the iteration. The maximum of non-negative doubles is taken on their bit
// patterns, which order like the values.
__global__ void closureResidual(size_t n, const double* candidate, const double* colorBefore, const double* surface,
                                const double* energyBefore, const double* jump, const double* jumpBefore,
                                const double* bulk, const ReactiveGpuHemOutputV1* output, unsigned long long* bits,
                                unsigned* flags) {
    const size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    unsigned long long local = 0;
    if (c < n) {
        const ReactiveThermoState& s = output[c].state;
        const double a = fabs(bulk[c]), b = s.rho * 1e5;
        const double bulkScale = a < b ? b : a;
        const double p = s.p < 1.0 ? 1.0 : s.p;
        const double x = fabs(candidate[c] - colorBefore[c]), y = fabs(surface[c] - energyBefore[c]) / bulkScale,
                     z = fabs(jump[c] - jumpBefore[c]) / p;
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) atomicOr(flags, kNonFinite);
        else local = (unsigned long long)__double_as_longlong(fmax(x, fmax(y, z)));
    }
    for (unsigned offset = 16; offset; offset >>= 1) {
        const unsigned long long other = __shfl_down_sync(0xffffffffu, local, offset);
        if (other > local) local = other;
    }
    if ((threadIdx.x & 31u) == 0 && local) atomicMax(bits, local);
}

}  // namespace capres
}  // namespace rb200
