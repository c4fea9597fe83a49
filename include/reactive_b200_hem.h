/* reactive_gpu_hem_* : the HEM UV-flash C ABI exported by libreactive_b200.so.
 *
 * Model images, batch arrays, success flags and profile structs are those of the
 * reference ABI (src/reactiveThermo/reactiveGpuHem.h:40-84). This build flashes
 * one condensable species with its own pure liquid (ns = 1, nl = 1, no solid,
 * boundaryRecovery = 0, the pure-N2O configuration); create rejects other
 * images with an error message. Device or API errors never fall back to a CPU
 * flash. A failed cell leaves the caller's state unchanged and reports
 * success = 0.
 */
#ifndef REACTIVE_B200_HEM_H
#define REACTIVE_B200_HEM_H
#include "reactive_b200_types.h"
#ifdef __cplusplus
extern "C" {
#endif

/* src/reactiveThermo/reactiveGpuHem.h:40 (policy strings :31-37) */
const char* reactive_gpu_hem_numerical_policy_v1(void);
/* src/reactiveThermo/reactiveGpuHem.h:41 (impl. src/reactiveTransport/reactiveGpuHem.cuh:190-219) */
void* reactive_gpu_hem_create_v1(const void* model, size_t modelBytes, size_t capacity, char* error, size_t errorSize);
/* src/reactiveThermo/reactiveGpuHem.h:44 */
void* reactive_gpu_hem_create_resident_v1(const void* model, size_t modelBytes, size_t capacity, char* error,
    size_t errorSize);
/* src/reactiveThermo/reactiveGpuHem.h:46-47 */
size_t reactive_gpu_hem_device_bytes_v1(void* hem);
void reactive_gpu_hem_destroy_v1(void* hem);
/* src/reactiveThermo/reactiveGpuHem.h:51-52 (impl. reactiveGpuHem.cuh:227-353): q holds ns masses per
 * cell, energy the internal energy density, state the seed in / the result out. */
int reactive_gpu_hem_run_v1(void* hem, const double* q, const double* energy, size_t count,
    ReactiveThermoState* state, int* success, ReactiveGpuHemProfileV1* profile, char* error, size_t errorSize);
/* src/reactiveThermo/reactiveGpuHem.h:56-65, :72-84: the capillary batches. energy is the bulk
 * internal energy density (kinetic and surface energy removed); each cell's color in [0, 1],
 * pressure jump sigma*kappa [Pa] and equilibrium flag select the reference's capillary recovery
 * (recoverCapillary, reactiveDeviceFlash.h:572-588): the gas phase at p - color*jump, the liquid at
 * p + (1 - color)*jump, p the returned mechanical pressure; UV equilibrium with the boundary search,
 * or (equilibrium 0) the frozen partition at the seed's liquid masses; a nonzero jump needs one
 * pure liquid (else the cell fails). run_v2 rejects the batch ("Invalid CUDA HEM capillary cell
 * input") for a color outside [0, 1], a non-finite jump or an equilibrium flag other than 0/1.
 * These run on the multi-species engine, one thread per cell (for a pure-fluid handle, one made
 * from the same image, whose Newton Jacobian is always the bounded finite-difference one).
 * run_resident_v1: device pointers indexed by global cell, order[0..count) names the cells, each
 * result (state, success) goes to output[cell] (reserved untouched), a failed cell returns its
 * seed; capillary may be NULL for the plain flash; synchronous, batch totals in *profile.
 * initialize_tp_v1 (src/reactiveThermo/reactiveGpuHem.h:66-71, every record's equilibrium 0):
 * at each seed's (p, T) and liquid mass, with the gas at p - color*jump and the liquid at
 * p + (1 - color)*jump, the densities scaled so the phase volumes fill the cell; q, energy and
 * state become the normalised densities, their energy and the state only if every cell succeeds
 * (success per cell either way); on the same engine. */
int reactive_gpu_hem_run_v2(void* hem, const double* q, const double* energy,
    const ReactiveGpuHemCapillaryInputV2* capillary, size_t count, ReactiveThermoState* state, int* success,
    ReactiveGpuHemProfileV1* profile, char* error, size_t errorSize);
int reactive_gpu_hem_initialize_tp_v1(void* hem, double* q, double* energy,
    const ReactiveGpuHemCapillaryInputV2* capillary, size_t count, ReactiveThermoState* state, int* success,
    ReactiveGpuHemProfileV1* profile, char* error, size_t errorSize);
int reactive_gpu_hem_run_resident_v1(void* hem, const double* q, const double* energy,
    const ReactiveThermoState* seed, const ReactiveGpuHemCapillaryInputV2* capillary, const uint32_t* order,
    size_t count, ReactiveGpuHemOutputV1* output, ReactiveGpuHemProfileV1* profile, char* error, size_t errorSize);

/* ---- additive device-resident entry point (no reference counterpart; the
 * reference's resident HEM takes host-prepared q/energy arrays,
 * src/reactiveTransport/reactiveGpuHem.cuh:360-403). All pointers are DEVICE
 * memory. `conserved` is the transport's SoA conserved array (row k at
 * conserved + k*stride; species rows, three momentum rows, total energy), the
 * internal energy is formed on the device. seed/state are full thermo states;
 * transport (optional) receives the compact transport state. success (optional)
 * receives per-cell flags; failed cells copy their seed. Never synchronises or
 * allocates; safe to capture in a CUDA graph.
 * flags bit 1: run the plain form instead (one thread per cell running the whole
 * candidate search in order, no work queue, no pruning).
 * Work counters accumulate in either form (read with run_counters_v3). */
int reactive_gpu_hem_run_device_v3(void* hem, const double* conserved, size_t stride, size_t count,
    size_t variables, const ReactiveThermoState* seed, ReactiveThermoState* state,
    ReactiveTransportState* transport, int* success, void* reserved, int flags, void* stream,
    char* error, size_t errorSize);
/* Synchronises `stream` and reports the counters accumulated since the last call
 * (phase/residual evaluations, candidates, stable candidates, failures in
 * deviceFailures, Jacobians); resets them. */
int reactive_gpu_hem_run_counters_v3(void* hem, ReactiveGpuHemProfileV1* profile, void* stream, char* error,
    size_t errorSize);

/* Launch-shape autotuner of the work-queue flash (no reference counterpart).
 * Runs the flash of `count` cells (conserved SoA rows with `stride`, seeds as
 * run_device_v3 takes them) with 1, 2, ... up to the occupancy limit of
 * resident queue blocks per SM, times each on `stream` and keeps the fastest
 * for later launches (the results do not depend on it). Synchronous; allocates
 * the host-path scratch on the first call; call it before capturing a graph.
 * *blocksPerSm (may be NULL) receives the choice. */
int reactive_gpu_hem_autotune_v3(void* hem, const double* conserved, size_t stride, size_t count,
    size_t variables, const ReactiveThermoState* seed, void* stream, int* blocksPerSm, char* error,
    size_t errorSize);

/* Two-phase admissibility bound of the work-queue search (no reference
 * counterpart). For a pure fluid a two-phase candidate can only converge to a
 * mixture on a saturation tie line of the model's cubic (chemical potentials
 * equal to mutol, volume and energy to vtol and etol). At create the handle
 * tabulates the tie lines (4,096 temperatures over the liquid range) and bounds
 * the specific internal energy of the mixtures at each specific volume; a cell
 * outside that region, widened by 1e-3 of the latent energy and ten tolerances,
 * has its two-phase seeds (and restart seeds) recorded as failed without the
 * Newton solves, which could not converge. Results are the exhaustive search's
 * bit for bit; the work counters count the skipped seeds as failed candidates
 * without phase evaluations. On by default where the bound is built (a pure
 * fluid, mutol <= 1e-5, a liquid range ending at or below the cubic's critical
 * temperature); request 0 turns it off, 1 on, -1 queries; *active (may be NULL)
 * receives the state. The plain per-cell form and the static entry run the
 * exhaustive search. */
int reactive_gpu_hem_two_phase_bound_v3(void* hem, int request, int* active, char* error, size_t errorSize);
/* Vector-Jacobian product of the flash (no reference counterpart; the
 * reference's tangent precedent is its host IFT TangentContext,
 * src/reactiveThermo/reactiveDirectional.inc:81-106). At the converged states
 * `state` of cells with conserved SoA rows `conserved` (pure fluid, variables
 * 5), adds to conservedBar (SoA, stride barStride) the adjoint of the
 * transport-state outputs {p, T, rho, cv, frozen sound, gas mass} given in
 * transportBar, by the implicit function theorem on the converged candidate's
 * residual (two-phase (ln p, ln T, beta) or a single-phase (ln p, ln T)
 * partition). Cells whose derivative could not be formed add nothing and
 * increment *failed (device counter, may be NULL). Asynchronous on `stream`. */
int reactive_gpu_hem_vjp_device_v3(void* hem, const double* conserved, size_t stride, size_t count,
    size_t variables, const ReactiveThermoState* state, const ReactiveTransportState* transportBar,
    double* conservedBar, size_t barStride, unsigned* failed, void* stream, char* error, size_t errorSize);

/* Flash without any allocation. No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc when they need a flash, for example a solver
 * whose own memory pool owns the whole device and forbids other allocations. It
 * takes the model image and DEVICE
 * arrays like reactive_gpu_hem_run_device_v3 but needs no handle: its scratch is
 * one file-scope device array (about 9 MB, held by every GPU that loads this
 * library until the process exits) for at most 4,096 cells per call; larger
 * batches are rejected with an error. Every call looks up the array's address on
 * the current device; the first call on each device also loads this library's
 * device code there if needed and queries the flash kernel's occupancy, so make
 * it before any stream capture. Calls share the array: calls that overlap on the
 * GPU race and must be serialised. */
int reactive_gpu_hem_run_static_v3(const void* model, size_t modelBytes, const double* conserved, size_t stride,
    size_t count, size_t variables, const ReactiveThermoState* seed, ReactiveThermoState* state,
    ReactiveTransportState* transport, int* success, void* stream, char* error, size_t errorSize);

#ifdef __cplusplus
}
#endif
#endif
