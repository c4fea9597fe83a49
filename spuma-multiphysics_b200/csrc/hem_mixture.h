// Host interface of the multi-species HEM flash (hem_mixture.cu) for the
// reactive_gpu_hem_* entry points in hem.cu.
#pragma once
#include <cstddef>
#include <string>
#include "../../include/reactive_b200_types.h"

namespace rb200 {

struct MixtureFlash;

// A handle for a model image outside the pure-fluid scope: a Peng-Robinson gas of
// 1 to 4 species with 0 to 2 pure condensed liquids. Returns nullptr and the
// reason when the image is invalid or outside this build's scope.
MixtureFlash* mixtureCreate(const ReactiveB200HemModel& model, size_t capacity, int device, std::string& why);
void mixtureDestroy(MixtureFlash* flash);
size_t mixtureDeviceBytes(const MixtureFlash* flash);
// The reference's run_v1 / run_v2 contract on host arrays: q cell-major (count x
// ns species densities), energy the internal (bulk) energy density, capillary
// (optional, run_v2) each cell's color, pressure jump and equilibrium flag,
// already validated; states the seeds in and the results out (a failed cell
// keeps its seed), success per cell. Synchronous.
void mixtureRun(MixtureFlash* flash, const double* q, const double* energy, size_t count,
                const ReactiveGpuHemCapillaryInputV2* capillary, ReactiveThermoState* states, int* success,
                ReactiveGpuHemProfileV1& profile);
// The reference's initialize_tp_v1 contract (capillary records with
// equilibrium 0, already validated): q, energy and states become the
// normalised densities, their energy and the states only if every cell
// succeeds; success per cell either way.
void mixtureInitialize(MixtureFlash* flash, double* q, double* energy, size_t count,
                       const ReactiveGpuHemCapillaryInputV2* capillary, ReactiveThermoState* states, int* success,
                       ReactiveGpuHemProfileV1& profile);
// The reference's run_resident_v1 contract: DEVICE arrays indexed by cell,
// order[0..count) names the cells, each result goes to output[cell] (a failed
// cell gets its seed). Synchronous on the engine's stream; batch totals in profile.
void mixtureRunResident(MixtureFlash* flash, const double* q, const double* energy, const ReactiveThermoState* seed,
                        const ReactiveGpuHemCapillaryInputV2* capillary, const uint32_t* order, size_t count,
                        ReactiveGpuHemOutputV1* output, ReactiveGpuHemProfileV1& profile);

}  // namespace rb200
