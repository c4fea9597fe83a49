/* Plain-old-data structures shared by the transport and HEM C ABIs.
 *
 * Every struct here crosses the drop-in boundary and therefore keeps the exact
 * field order, types and sizes of the reference ABI it replaces; the static
 * size checks at the bottom pin them. Reference layouts (paths inside the
 * reference project):
 *   ReactiveTransportFace / State / Config  src/reactiveTransport/reactiveTransport.h:10-23
 *   ReactiveTransportPrimitive              src/reactiveTransport/reactiveTransport.h:77
 *   ReactiveTransportStats / Profile        src/reactiveTransport/reactiveTransport.h:73-83
 *   ReactiveTransportDeviceProfile          src/reactiveTransport/reactiveTransport.h:86-89
 *   ReactiveTransportOptionsV2 / MemoryV2   src/reactiveTransport/reactiveTransport.h:24-33
 *   ReactiveTransportToken                  src/reactiveTransport/reactiveTransport.h:34
 *   ReactiveTransportOptionsV21/ProfileV21  src/reactiveTransport/reactiveTransportV21.h:4-16
 *   ReactiveWaleOptionsV1 / ProfileV1       src/reactiveTransport/reactiveTurbulence.h:12-19
 *   ReactiveWaleScalarOptionsV1 / ProfileV1 src/reactiveTransport/reactiveTurbulence.h:28-35
 *   ReactiveCapillaryOptionsV1 / ProfileV1  src/reactiveTransport/reactiveTransport.h:38-47
 *   ReactiveCapillaryResidentViewV1         src/reactiveTransport/reactiveCapillaryResident.h:17-22
 *   ReactiveWalePrModelV1 / EpochV1 / ProfileV1 src/reactiveTransport/reactiveTurbulence.h:48-68
 *   ReactiveGasThermoSpecies/Region/Partition src/reactiveThermo/reactiveGasThermo.h:12-21
 *   ReactiveThermoState                     src/reactiveThermo/reactiveThermo.h:11-19
 *   ReactiveGpuHemProfileV1                 src/reactiveThermo/reactiveGpuHem.h:14-21
 *   ReactiveGpuHemCapillaryInputV2          src/reactiveThermo/reactiveGpuHem.h:59-62
 *   ReactiveGpuHemOutputV1                  src/reactiveThermo/reactiveGpuHem.h:78-80
 */
#ifndef REACTIVE_B200_TYPES_H
#define REACTIVE_B200_TYPES_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct ReactiveTransportFace {
    int64_t owner, neighbour, fixed;
    double normal[3], area, distance, ownerWeight;
    int kind; /* 0 internal/cyclic, 1 slipWall, 2 extrapolate, 3 fixedState */
} ReactiveTransportFace;

typedef struct ReactiveTransportState {
    double p, T, rho, cv, sound, gasMass, dilatation;
} ReactiveTransportState;

typedef struct ReactiveTransportConfig {
    size_t cells, species, variables, faces, fixed;
    double viscosity, conductivity, diffusivity, waveFactor, maxBytes;
    int mechanical;
} ReactiveTransportConfig;

typedef struct ReactiveTransportOptionsV2 {
    uint32_t abiVersion, structBytes;
    size_t bridgeCells;
    int recomputeGas;
    char physicalModelHash[65];
} ReactiveTransportOptionsV2;

typedef struct ReactiveTransportMemoryV2 {
    uint64_t liveBytes, peakBytes, bridgeBytes, conservedWorkspaceBytes, gasWorkspaceBytes;
    uint64_t rhsWorkspaceBytes, deviceToDeviceBytes, synchronizations;
} ReactiveTransportMemoryV2;

typedef struct ReactiveTransportToken { uint64_t attemptId, stageId, contentVersion; } ReactiveTransportToken;

typedef struct ReactiveTransportStats {
    uint64_t allocatedBytes, uploadedBytes, downloadedBytes, kernelLaunches;
    uint64_t stages, stepQueries;
} ReactiveTransportStats;

typedef struct ReactiveTransportPrimitive { double rho, u[3]; } ReactiveTransportPrimitive;

typedef struct ReactiveTransportProfile {
    uint64_t conservedUploads, conservedUploadBytes, conservedDownloadBytes;
    uint64_t stateUploadBytes, primitiveUploadBytes, gasUploadBytes;
    uint64_t boundaryPartitions, residentStages;
} ReactiveTransportProfile;

typedef struct ReactiveTransportDeviceProfile {
    uint64_t gasPropertyBuilds, gasPropertyCells, partitionUploadBytes, thermoTableBytes;
    uint64_t gasStatusChecks, cflFaceLaunches, transportFaceLaunches, faceWorkspaceBytes;
} ReactiveTransportDeviceProfile;

typedef struct ReactiveTransportOptionsV21 {
    uint32_t abiVersion, structBytes;
    size_t slotBytes, pinnedBudgetBytes, bridgeCellsOverride;
    uint32_t slots, blockThreads;
    int recomputeGas, detailedGasCounters;
    char physicalModelHash[65];
} ReactiveTransportOptionsV21;

typedef struct ReactiveTransportProfileV21 {
    uint64_t layoutTiles, layoutLaunches, memcpyCalls, payloadBytes;
    uint64_t nasaValidationEvaluations, nasaFaceEvaluations, temperatureBasisBuilds;
    uint64_t pinnedBytes, deviceStagingBytes, temperatureBasisBytes, eventWaits;
    uint64_t slotCells, slots, blockThreads, failedCalls;
} ReactiveTransportProfileV21;

typedef struct ReactiveWaleOptionsV1 {
    uint32_t abiVersion, structBytes;
    double Cw;
} ReactiveWaleOptionsV1;

typedef struct ReactiveWaleProfileV1 {
    uint32_t abiVersion, structBytes;
    uint64_t gradientBuilds, viscosityBuilds, cellsEvaluated, workspaceBytes;
} ReactiveWaleProfileV1;

typedef struct ReactiveWaleScalarOptionsV1 {
    uint32_t abiVersion, structBytes;
    double turbulentPrandtl, turbulentSchmidt;
} ReactiveWaleScalarOptionsV1;

typedef struct ReactiveWaleScalarProfileV1 {
    uint32_t abiVersion, structBytes;
    uint64_t fieldUploads, fieldUploadBytes, workspaceBytes;
} ReactiveWaleScalarProfileV1;

/* The diffuse capillary closure: surface tension sigma [N/m], the capillary
 * wave Courant number (0, 1], the geometry threshold on |grad c| * V^(1/3)
 * below which a cell has no interface normal, and the species whose liquid
 * inventory is conserved variable species+4. */
typedef struct ReactiveCapillaryOptionsV1 {
    uint32_t abiVersion, structBytes;
    double sigma, capillaryCfl, geometryEpsilon;
    int64_t condensableSpecies;
} ReactiveCapillaryOptionsV1;

typedef struct ReactiveCapillaryProfileV1 {
    uint32_t abiVersion, structBytes;
    uint64_t geometryBuilds, geometryCells, geometryKernels, faceFluxBuilds;
    uint64_t colorUploadBytes, geometryDownloadBytes, capillaryWorkspaceBytes;
} ReactiveCapillaryProfileV1;

/* The WALE Peng-Robinson scalar-property pass (src/reactiveTransport/reactiveTurbulence.h:48-68). */
typedef struct ReactiveWalePrModelV1 {
    uint32_t abiVersion, structBytes;
    const void* modelImage;
    size_t modelBytes;
    char physicalModelHash[65];
    const double* fixedCp;
    const double* fixedSpeciesH;  /* fixed-cell-major, species values per cell */
} ReactiveWalePrModelV1;

typedef struct ReactiveWalePrEpochV1 {
    uint32_t abiVersion, structBytes;
    /* the exact next RK input of stage properties; a CFL-only cp query outside an
     * attempt uses {0,0,0}, inside one {attemptId, UINT64_MAX, 0} */
    ReactiveTransportToken nextConserved;
    uint64_t thermoVersion, geometryVersion, boundaryVersion;
    int enthalpies;  /* 0: cp only (CFL); 1: cp and the effective species enthalpies */
} ReactiveWalePrEpochV1;

typedef struct ReactiveWalePrProfileV1 {
    uint32_t abiVersion, structBytes;
    uint64_t builds, cells, kernels, failures, inputUploadBytes, scratchBytes;
    double wallSeconds;
} ReactiveWalePrProfileV1;

typedef struct ReactiveGasThermoSpecies {
    uint64_t regionOffset, regionCount;
    double gasConstant;
    int polynomial;
} ReactiveGasThermoSpecies;

typedef struct ReactiveGasThermoRegion {
    double minimumTemperature, maximumTemperature, coefficient[9];
} ReactiveGasThermoRegion;

typedef struct ReactiveGasPartition { double liquidMass[2]; } ReactiveGasPartition;

typedef struct ReactiveThermoState {
    double p, T, rho, e, entropy;
    double soundFrozen, soundEquilibrium;
    double volumeResidual, energyResidual, chemicalResidual;
    double alphaGas, alphaLiquid[2];
    double rhoGas, rhoLiquid[2], liquidMass[2];
    double gasMass, cp, cv;
    int activeLiquids, iterations;
} ReactiveThermoState;

typedef struct ReactiveGpuHemProfileV1 {
    uint32_t abiVersion, structBytes;
    uint64_t batches, submitted, succeeded, cpuFallbacks, deviceFailures;
    uint64_t phaseEvaluations, residualEvaluations, flashCandidates, stableCandidates;
    uint64_t analyticJacobians, finiteDifferenceJacobians;
    uint64_t transferBytes, hostBytes, deviceBytes;
    double wallSeconds, kernelSeconds, copySeconds;
} ReactiveGpuHemProfileV1;

typedef struct ReactiveGpuHemCapillaryInputV2 {
    double color, pressureJump;
    int equilibrium;
} ReactiveGpuHemCapillaryInputV2;

typedef struct ReactiveGpuHemOutputV1 {
    ReactiveThermoState state; int success, reserved;
} ReactiveGpuHemOutputV1;

/* The device view of one resident capillary iteration
 * (src/reactiveTransport/reactiveCapillaryResident.h:17-22): DEVICE pointers for
 * reactive_gpu_hem_run_resident_v1 (the first `count` entries of `order` are the
 * cells to flash). */
typedef struct ReactiveCapillaryResidentViewV1 {
    uint32_t abiVersion, structBytes;
    const double* q;
    const double* energy;
    const ReactiveThermoState* seed;
    const ReactiveGpuHemCapillaryInputV2* capillary;
    const uint32_t* order;
    ReactiveGpuHemOutputV1* output;
    size_t count;
} ReactiveCapillaryResidentViewV1;

/* The HEM model image. The reference passes an opaque 47,448-byte POD image
 * (src/reactiveThermo/reactiveDeviceFlash.h:39-53, static_assert at :52);
 * this is the same layout so an exported image can be handed over unchanged. */
#define REACTIVE_B200_MAX_SPECIES 16
#define REACTIVE_B200_MAX_REGIONS 8
#define REACTIVE_B200_SOLID_POINTS 64
typedef struct ReactiveB200NasaRegion {
    double minimumTemperature, maximumTemperature;
    int polynomial;
    double coefficient[9];
} ReactiveB200NasaRegion;
typedef struct ReactiveB200Species {
    double molecularWeight, a, b, kappa;
    int regionCount;
    ReactiveB200NasaRegion regions[REACTIVE_B200_MAX_REGIONS];
} ReactiveB200Species;
typedef struct ReactiveB200Table {
    int ns;
    double refPressure;
    ReactiveB200Species species[REACTIVE_B200_MAX_SPECIES];
    double aBinary[REACTIVE_B200_MAX_SPECIES][REACTIVE_B200_MAX_SPECIES];
} ReactiveB200Table;
typedef struct ReactiveB200SolidModel {
    int enabled, n;
    double Tmin, Tmax, Tref, pref, pmax;
    double molarVolume, molecularWeight, hRef, sRef;
    double T[REACTIVE_B200_SOLID_POINTS], cp[REACTIVE_B200_SOLID_POINTS];
} ReactiveB200SolidModel;
typedef struct ReactiveB200HemModel {
    ReactiveB200Table phase[3];
    int ns, nl, condensable[2], boundaryRecovery, scalarRecovery, analyticJacobian;
    int stableGasPrune;
    double weights[REACTIVE_B200_MAX_SPECIES], liquidTmin[2], liquidTc[2];
    double Tmin, Tmax, pmin, pmax, vtol, etol, mutol;
    int condensedKind[2];
    int enforceSpeciesTemperatureBounds;
    ReactiveB200SolidModel solid[2];
} ReactiveB200HemModel;

#ifdef __cplusplus
}
static_assert(sizeof(ReactiveTransportFace) == 80, "face layout");
static_assert(sizeof(ReactiveTransportState) == 56, "state layout");
static_assert(sizeof(ReactiveThermoState) == 176, "thermo state layout");
static_assert(sizeof(ReactiveWaleScalarOptionsV1) == 24, "WALE scalar options layout");
static_assert(sizeof(ReactiveWaleScalarProfileV1) == 32, "WALE scalar profile layout");
static_assert(sizeof(ReactiveCapillaryOptionsV1) == 40, "capillary options layout");
static_assert(sizeof(ReactiveCapillaryProfileV1) == 64, "capillary profile layout");
static_assert(sizeof(ReactiveCapillaryResidentViewV1) == 64, "resident capillary view layout");
static_assert(sizeof(ReactiveWalePrModelV1) == 112, "WALE PR model layout");
static_assert(sizeof(ReactiveWalePrEpochV1) == 64, "WALE PR epoch layout");
static_assert(sizeof(ReactiveWalePrProfileV1) == 64, "WALE PR profile layout");
static_assert(sizeof(ReactiveGpuHemOutputV1) == 184, "HEM output layout");
static_assert(sizeof(ReactiveB200HemModel) == 47448, "HEM model image layout");
static_assert(offsetof(ReactiveB200HemModel, stableGasPrune) == 45004, "HEM model image layout");
static_assert(offsetof(ReactiveB200HemModel, weights) == 45008, "HEM model image layout");
#endif
#endif
