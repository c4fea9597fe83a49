/* reactive_transport_* : the transport C ABI exported by libreactive_b200.so.
 *
 * Every entry point keeps the reference signature, argument meaning, error text
 * convention and return codes (0 ok, 1 error with text via
 * reactive_transport_error, 2 concurrent entry rejected, -1 null handle;
 * src/reactiveTransport/reactiveTransport.cpp:1471-1491). Host arrays are
 * cell-major and borrowed only for the duration of the synchronous call.
 * backend must be 1 (CUDA); backend 0 is rejected with an error because this
 * library has no CPU execution path.
 *
 * The *_v3 entry points are additive: they take DEVICE pointers and a CUDA
 * stream, never synchronise, and never allocate, so a caller can keep the
 * conserved state resident in HBM and capture a whole step in a CUDA graph.
 */
#ifndef REACTIVE_B200_TRANSPORT_H
#define REACTIVE_B200_TRANSPORT_H
#include "reactive_b200_types.h"
#ifdef __cplusplus
extern "C" {
#endif

/* src/reactiveTransport/reactiveTransport.h:118-121 (impl. reactiveTransport.cpp:1494-1499) */
void* reactive_transport_create(int backend, const ReactiveTransportConfig* config,
    const double* volume, const ReactiveTransportFace* faces, const double* fixedQ,
    const ReactiveTransportState* fixedStates, const double* fixedGasY,
    const double* fixedGasH, char* error, size_t errorSize);
/* src/reactiveTransport/reactiveTransport.h:60-63 (impl. reactiveTransport.cpp:1738-1743) */
void* reactive_transport_create_v2(int backend, const ReactiveTransportConfig* config,
    const ReactiveTransportOptionsV2* options, const double* volume, const ReactiveTransportFace* faces,
    const double* fixedQ, const ReactiveTransportState* fixedStates, const double* fixedY, const double* fixedH,
    char* error, size_t errorSize);
/* src/reactiveTransport/reactiveTransportV21.h:24-27 (impl. reactiveTransport.cpp:1792-1808) */
void* reactive_transport_create_v21(int backend, const ReactiveTransportConfig* config,
    const ReactiveTransportOptionsV21* options, const double* volume, const ReactiveTransportFace* faces,
    const double* fixedQ, const ReactiveTransportState* fixedStates, const double* fixedY, const double* fixedH,
    char* error, size_t errorSize);
/* src/reactiveTransport/reactiveTransport.h:122-125 */
void reactive_transport_destroy(void* transport);
const char* reactive_transport_error(void* transport);
int reactive_transport_is_cuda(void* transport);
int reactive_transport_stats(void* transport, ReactiveTransportStats* stats);
/* src/reactiveTransport/reactiveTransport.h:84, :90, :64; reactiveTransportV21.h:28 */
int reactive_transport_profile(void* transport, ReactiveTransportProfile* profile);
int reactive_transport_device_profile(void* transport, ReactiveTransportDeviceProfile* profile);
int reactive_transport_memory_v2(void* transport, ReactiveTransportMemoryV2* result);
int reactive_transport_profile_v21(void* transport, ReactiveTransportProfileV21* result);
/* src/reactiveTransport/reactiveTransport.h:126-127 (impl. reactiveTransport.cpp:1506-1512) */
int reactive_transport_stable_step(void* transport, const double* q,
    const ReactiveTransportState* state, double cfl, double maximum, double* dt);
/* src/reactiveTransport/reactiveTransport.h:108-110 (impl. reactiveTransport.cpp:1647-1667) */
int reactive_transport_stable_step_primitives(void* transport,
    const ReactiveTransportPrimitive* primitive, const ReactiveTransportState* state,
    double cfl, double maximum, double* dt);
/* src/reactiveTransport/reactiveTransport.h:131-133 (impl. reactiveTransport.cpp:1518-1524) */
int reactive_transport_stage(void* transport, double* q,
    const ReactiveTransportState* state, const double* gasY, const double* gasH,
    double dt, int stage, double* boundaryRate);
/* src/reactiveTransport/reactiveTransport.h:135-137 (impl. reactiveTransport.cpp:1513-1517) */
int reactive_transport_rhs(void* transport, const double* q,
    const ReactiveTransportState* state, const double* gasY, const double* gasH,
    double* rhs, double* boundaryRate);
/* src/reactiveTransport/reactiveTransport.h:106 (impl. reactiveTransport.cpp:1557-1565) */
int reactive_transport_upload_conserved(void* transport, const double* q, uint64_t version);
/* src/reactiveTransport/reactiveTransport.h:113-115 (impl. reactiveTransport.cpp:1710-1720) */
int reactive_transport_stage_resident(void* transport, const ReactiveTransportState* state,
    const double* gasY, const double* gasH, double dt, int stage,
    uint64_t inputVersion, uint64_t outputVersion, double* qOutput, double* boundaryRate);
/* src/reactiveTransport/reactiveTransport.h:67-72 (impl. reactiveTransport.cpp:1750-1789) */
int reactive_transport_begin_attempt(void* transport, const char* modelHash, uint64_t attemptId);
int reactive_transport_end_attempt(void* transport, uint64_t attemptId, int commit);
int reactive_transport_advance_resident_v2(void* transport, ReactiveTransportToken input,
    ReactiveTransportToken output, const ReactiveTransportState* state, const ReactiveGasPartition* partition,
    const double* gasY, const double* gasH, double dt, double* boundaryRate);
int reactive_transport_download_conserved(void* transport, ReactiveTransportToken token, double* output);
/* src/reactiveTransport/reactiveTransport.h:58-59 (impl. reactiveTransport.cpp:1636-1646) */
int reactive_transport_replace_stage_state_v1(void* transport, ReactiveTransportToken before,
    uint64_t replacementVersion, const double* conserved);
/* src/reactiveTransport/reactiveTurbulence.h:20-25 (impl. reactiveTransport.cpp:1668-1709) */
int reactive_transport_set_wale_v1(void* transport, const ReactiveWaleOptionsV1* options);
int reactive_transport_wale_profile_v1(void* transport, ReactiveWaleProfileV1* profile);
/* WALE scalar closure (src/reactiveTransport/reactiveTurbulence.h:26-45,
 * src/reactiveTransport/reactiveTransport.cpp:653-702, 1671-1681): the
 * turbulent heat flux rho nu_t cp / Pr_t grad T and the turbulent mixing of the
 * total species mass fractions rho nu_t / Sc_t grad Y (with its enthalpy flux)
 * on every non-slip face, and their diffusivities in the CFL step. Zero disables
 * a term. Installed once, after set_wale_v1 and before any stage; species
 * mixing needs variables == species + 4. The fields are the current mixture cp
 * (J/kg/K) and the effective species enthalpies (J/kg), cell-major, for the
 * cells and the fixed states (fixed pointers may be NULL without fixed
 * states). NULL enthalpies refresh cp only (enough for the CFL step) and
 * invalidate the previous enthalpies: a stage needs both. */
int reactive_transport_set_wale_scalars_v1(void* transport, const ReactiveWaleScalarOptionsV1* options);
int reactive_transport_wale_scalar_profile_v1(void* transport, ReactiveWaleScalarProfileV1* profile);
int reactive_transport_wale_scalar_fields_v1(void* transport, const double* cellCp,
    const double* cellSpeciesH, const double* fixedCp, const double* fixedSpeciesH);
int reactive_transport_wale_primitives_v1(void* transport, const ReactiveTransportPrimitive* primitive,
    const ReactiveTransportState* state, double* nut);
/* Out-of-scope reference entry points kept as stubs that return 1 with a
 * message, as the reference's own CPU build does for its CUDA-only paths
 * (src/reactiveTransport/reactiveTransport.cpp:1613-1630):
 * src/reactiveTransport/reactiveTransport.h:93-102 (NASA-generated gas properties),
 * src/reactiveTransport/reactiveTurbulence.h:47-85 (WALE PR properties). */
int reactive_transport_set_gas_thermo(void* transport, const ReactiveGasThermoSpecies* species,
    size_t count, const ReactiveGasThermoRegion* regions, size_t regionCount,
    const int64_t* liquidSpecies, size_t liquids);
int reactive_transport_stage_resident_gas(void* transport, const ReactiveTransportState* state,
    const ReactiveGasPartition* partition, double dt, int stage,
    uint64_t inputVersion, uint64_t outputVersion, double* qOutput, double* boundaryRate);
int reactive_transport_rhs_gas(void* transport, const double* q, const ReactiveTransportState* state,
    const ReactiveGasPartition* partition, double* rhs, double* boundaryRate);
int reactive_transport_gas_properties_resident(void* transport, const ReactiveTransportState* state,
    const ReactiveGasPartition* partition, double* gasY, double* gasH);
/* The diffuse capillary closure on the face graph (src/reactiveTransport/
 * reactiveTransport.h:48-54, reactiveTransport.cpp:859-962): a resolved material
 * color with its Green-Gauss interface geometry
 * (src/reactiveInterface/reactiveUnstructuredInterface.h) and the balanced
 * contact-preserving HLLC face core (reactiveBalancedCapillary.h:55-142). Install
 * once before stepping, on a non-mechanical model with one frozen liquid
 * inventory (variables = species + 5). Each geometry call replaces the cell and
 * fixed colors (each in [0, 1]) and rebuilds the gradient, normal, area density,
 * curvature and surface energy sigma |grad c| [J/m^3]; curvature and normalXYZ
 * (packed XYZ per cell) may be NULL. An identical request without normalXYZ
 * returns the published outputs without device work. Every stage then consumes
 * this exact geometry; a face whose balanced flux cannot be formed fails the host
 * entries with "Invalid capillary face flux" and sets bit 3 of the device status
 * word. The capillary model keeps the face graph (the structured box path needs
 * variables = species + 4). */
int reactive_transport_set_capillary_v1(void* transport, const ReactiveCapillaryOptionsV1* options);
int reactive_transport_capillary_geometry_v1(void* transport, const double* cellColor,
    const double* fixedColor, double* surfaceEnergy, double* curvature, double* normalXYZ);
int reactive_transport_capillary_profile_v1(void* transport, ReactiveCapillaryProfileV1* profile);
/* Entry points of the Cartesian implicit surface geometry, which the solver
 * references statically (so that a solver linked against this library resolves
 * every symbol it names); each returns 1 with a message, and the solver reaches
 * them only with that option selected. Struct arguments are opaque here.
 * src/reactiveTransport/reactiveCartesianTransport.h:34-35 (Cartesian descriptor),
 * :44-49 (implicit geometry). */
int reactive_transport_install_cartesian_v1(void* transport, const void* mesh);
int reactive_transport_cartesian_info_v1(void* transport, void* info);
int reactive_transport_set_implicit_v1(void* transport, const void* options);
int reactive_transport_implicit_coefficients_v1(void* transport, double* output, const double* restore,
    size_t count, size_t* required);
/* The WALE Peng-Robinson scalar properties of the one-liquid capillary model
 * (src/reactiveTransport/reactiveTurbulence.h:48-81, reactiveTransport.cpp:703-828):
 * install once, before stepping, after set_capillary_v1 and set_wale_scalars_v1,
 * with the model image (copied), the transport's physical model hash and the
 * fixed cells' cp / species enthalpies; then each stage's (or CFL query's)
 * properties from the accepted states: the state's cp and, with enthalpies, the
 * effective species enthalpies (h_k = (gas_k hbar_k + [k condensable] m_l h_l) / q_k,
 * hbar the gas mixture's partial molar enthalpies at p - c J, h_l the liquid's
 * at p + (1 - c) J), every state checked against the phases it implies. The
 * epoch names what the properties are for: the exact next RK input token of the
 * stage, or a CFL query ({0,0,0} outside an attempt, {attempt, UINT64_MAX, 0}
 * inside), the geometry build they were computed on, a thermo version that
 * never decreases and boundary version 1; stage and CFL entries refuse
 * properties of another epoch, a new geometry retires them, and host scalar
 * uploads are refused once installed. A failing cell fails the call ("WALE PR
 * GPU property cell N status S") and publishes nothing. v2: statesUnchanged != 0
 * reuses the previous call's device copy of the states. */
int reactive_transport_set_wale_pr_model_v1(void* transport, const ReactiveWalePrModelV1* model);
int reactive_transport_wale_pr_properties_v1(void* transport, const ReactiveWalePrEpochV1* epoch, const double* q,
    size_t qStride, const ReactiveThermoState* state);
int reactive_transport_wale_pr_properties_v2(void* transport, const ReactiveWalePrEpochV1* epoch, const double* q,
    size_t qStride, const ReactiveThermoState* state, int statesUnchanged);
int reactive_transport_wale_pr_profile_v1(void* transport, ReactiveWalePrProfileV1* profile);
/* The resident capillary closure (src/reactiveTransport/reactiveCapillaryResident.h:26-41,
 * reactiveTransport.cpp:963-1127): the outer iteration between the capillary HEM
 * flash and the diffuse geometry with every per-cell array on the device; the
 * caller keeps the iteration control (src/reactiveFoam/reactiveCapillary.H:54-115).
 * begin: q (`species` = the transport's species masses per cell), the
 * transported liquid inventory, the bulk energy (kinetic removed, surface energy
 * not), the incoming states and the fixed colors; builds the seeds (each state
 * carrying its cell's liquid inventory), their color and geometry.
 * select: snapshots the iteration's color, jump and surface energy, and fills the
 * view for reactive_gpu_hem_run_resident_v1: the bulk energy less the surface
 * energy, the capillary records, and `order` with the cells to flash first (all
 * at iteration 0, later those whose color, jump or surface energy changed
 * bitwise since their last flash; heavy-first by the HEM bucket key), `count` of them.
 * update (after a fully successful flash of `count` cells): records the flashed
 * inputs, the candidate color from the flashed states, its geometry, and the
 * residual max(|dc|, |dE_s| / max(|E_bulk|, 1e5 rho), |dJ| / max(p, 1)).
 * relax: the color becomes 0.5 (before + candidate), geometry rebuilt.
 * commit: downloads the states, color, surface energy and curvature; a later
 * identical geometry request reuses that geometry.
 * A nonzero *fallback means an input the host closure would reject (a color
 * that does not close, a non-finite value): nothing host-side changed and the
 * caller reruns the closure on the host path. Out-of-order calls return 1. */
int reactive_transport_capillary_resident_begin_v1(void* transport, size_t species, const double* q,
    const double* liquid, const double* bulk, const ReactiveThermoState* states, const double* fixedColor,
    double sigma, int equilibrium, int* fallback);
int reactive_transport_capillary_resident_select_v1(void* transport, int iteration,
    ReactiveCapillaryResidentViewV1* view, int* fallback);
int reactive_transport_capillary_resident_update_v1(void* transport, size_t count, double* residual,
    int* fallback);
int reactive_transport_capillary_resident_relax_v1(void* transport);
int reactive_transport_capillary_resident_commit_v1(void* transport, ReactiveThermoState* states,
    double* color, double* surfaceEnergy, double* curvature);

/* ---- additive device-resident entry points (no reference counterpart; the
 * reference's resident path is advance_resident_v2 + download_conserved,
 * src/reactiveTransport/reactiveTransport.cpp:1773-1789, which round-trips q
 * through the host between RK stages). Conserved arrays are SoA,
 * q[k*(cells+fixed)+c], with the fixed-state tail filled by
 * reactive_transport_fill_fixed_v3. */
int reactive_transport_layout_v3(void* transport, size_t* cells, size_t* fixed, size_t* variables,
    size_t* species);
int reactive_transport_fill_fixed_v3(void* transport, double* q, ReactiveTransportState* state, void* stream);
/* stage 0: qOut = qIn + dt L(qIn). stage 1: qOut = .5 qOut + .5 (qIn + dt L(qIn)),
 * i.e. qOut holds q^n on entry. boundaryRate (device, variables doubles) may be null.
 * Requires diffusivity 0 (molecular species diffusion takes host gas fractions). */
int reactive_transport_stage_device_v3(void* transport, const double* qIn, double* qOut,
    const ReactiveTransportState* state, double dt, int stage, double* boundaryRate, void* stream);
/* Writes the CFL step (or -1 when any face is invalid) to dt[0] on the device. */
int reactive_transport_stable_step_device_v3(void* transport, const double* q,
    const ReactiveTransportState* state, double cfl, double maximum, double* dt, void* stream);
/* The CFL query and the stage on the same device state in one call (no
 * reference counterpart): the results are those of
 * reactive_transport_stable_step_device_v3(q = qIn, state, cfl, maximum, dtOut)
 * followed by reactive_transport_stage_device_v3(qIn, qOut, state, dt, stage,
 * boundaryRate), bit for bit, with the cell primitives and (with WALE) the
 * velocity gradients and eddy viscosities formed once for both. dt is the step
 * taken; dtOut[0] receives the CFL step (or -1) on the device. */
int reactive_transport_stage_cfl_device_v3(void* transport, const double* qIn, double* qOut,
    const ReactiveTransportState* state, double dt, int stage, double* boundaryRate, double cfl,
    double maximumStep, double* dtOut, void* stream);
/* Structured Cartesian fast path of the device-resident entries (no reference
 * counterpart: the reference's Cartesian descriptor,
 * reactive_transport_install_cartesian_v1 in
 * src/reactiveTransport/reactiveCartesianTransport.h:34, serves its capillary
 * geometry, not the flux). At create the face list is checked for a uniform box in the
 * canonical ordering; when it is one, stage_device_v3 and
 * stable_step_device_v3 use cell-stencil kernels that read no face-work array
 * and give bitwise the same stage results as the face graph. request -1 only
 * queries, 0 selects the face graph, 1 the structured path (an error when the
 * face list is not such a box); *active (may be NULL) receives the selection. */
int reactive_transport_structured_v3(void* transport, int request, int* active);
/* Face flux of the structured path (no C-ABI counterpart: the reference applies
 * its HLLC core only inside the capillary option, reactive_transport_set_capillary_v1,
 * with the interface geometry). request -1 only queries, 0 selects HLL, 1 HLLC:
 * the reference's contact-preserving core with no capillary terms
 * (src/reactiveInterface/reactiveBalancedCapillary.h:55-142), falling back to
 * the HLL coefficients when the star speed leaves the wave fan. A face whose
 * HLLC state cannot be formed sets bit 1 of the status word. Selecting the face
 * graph returns to HLL; the rate VJP covers HLL only. *active (may be NULL)
 * receives the scheme. */
int reactive_transport_flux_v3(void* transport, int request, int* active);
/* Arithmetic of the structured path (no reference counterpart; the reference
 * transport is FP64 only). request -1 only queries, 0 selects FP64, 1 the mixed
 * form: velocity gradients, WALE eddy viscosity and face fluxes (HLL, traction,
 * conduction) in FP32, each cell's six face contributions summed with
 * compensation (Neumaier two-sum) and the stage update applied to the FP64
 * conserved state in FP64. The CFL step stays FP64. Mixed requires the
 * structured path; selecting the face graph returns to FP64. *active (may be
 * NULL) receives 1 for mixed. */
int reactive_transport_precision_v3(void* transport, int request, int* active);
/* Own cells of this handle (no reference counterpart; the reference runs one
 * domain): a z-slab of a larger box holds its own cells [begin, end) and halo
 * layers that a neighbour owns. The stage entries then update the own cells
 * only (the halo cells' outputs are left as they were, for the halo exchange
 * to overwrite), the CFL minimum covers the own cells only, and the boundary
 * ledger sums the boundary faces of own cells only. Gradients, eddy
 * viscosities and face fluxes still read every cell, so an own cell next to a
 * halo sees the same neighbours as in the undivided box. Default: every cell.
 * Requires begin < end <= cells. */
int reactive_transport_owned_cells_v3(void* transport, uint64_t begin, uint64_t end);
/* Vector-Jacobian product of the rate operator of the device stage entries (no
 * reference counterpart; the reference has no adjoint). With rate(q, state) the
 * per-cell right-hand side L that stage_device_v3 applies (q SoA with the fixed
 * tail, stride cells+fixed) and w its adjoint (SoA, stride cells), writes
 * qBar = (dL/dq)^T w (SoA, stride cells) and stateBar = (dL/dstate)^T w per cell
 * (the p, T, rho and sound fields the flux reads; the others are zero).
 * Structured path, the whole operator: HLL or HLLC (wave-speed and star-state
 * switches taken piecewise, on the branch the forward selects), viscous/WALE traction through the cells' velocity gradients and
 * eddy viscosities (with their own adjoints carried back through the WALE
 * relation and the Green-Gauss gradient to the neighbours' velocities), and
 * conduction. The derivative of the FP64 operator; a handle with the WALE
 * scalar closure is refused. The first call on a viscous handle allocates its
 * scratch. Asynchronous on `stream`. */
int reactive_transport_rate_vjp_v3(void* transport, const double* q, const ReactiveTransportState* state,
    const double* w, double* qBar, ReactiveTransportState* stateBar, void* stream);
/* Launch-shape autotuner of the structured path (no reference counterpart).
 * Times the candidates of the stage kernel (0: the shared-memory tiled form; or
 * the per-cell form with 64, 96 (the default), 128 threads a block), gradient
 * (64, 128, 256) and CFL (64, 128, 256) kernels on this handle's problem (q and
 * state as stage_device_v3 takes them; neither is modified) and keeps the
 * fastest for later launches; results do not depend on the choice. Synchronous;
 * allocates one scratch copy of q on the first call; call it before capturing
 * a graph. chosen (may be NULL) receives {stage, gradient, CFL} block sizes. */
int reactive_transport_autotune_v3(void* transport, const double* q, const ReactiveTransportState* state,
    void* stream, unsigned* chosen);
/* Query (request NULL) or set the structured path's launch shapes {stage, gradient,
 * CFL} (no reference counterpart): stage 0 is the shared-memory tiled stage
 * kernel, 1 the split stage (each interior face's flux once into the face
 * workspace, then the per-cell sums; 128 threads per cell without the
 * workspace), 64/96/128 the per-cell kernel's block size; gradient
 * and CFL block sizes 64/128/256. Results do not depend on them. active (may be
 * NULL) receives the shapes in use. */
int reactive_transport_launch_shapes_v3(void* transport, const unsigned* request, unsigned* active);
/* Device-resident refresh of the WALE scalar fields for the device stage
 * entries (no reference counterpart: the reference fills them from the host or
 * from its own PR property pass). Stream-ordered and allocation-free, so it can
 * sit inside a captured graph. Reads cp[c * cpStride] and h[c * hStride + k]
 * (k < species) for the cells c < cells and, when the fixed pointers are not
 * NULL, the same strides for the fixed states; NULL fixed pointers keep the
 * fixed values last set. cellCp is required when Pr_t > 0; NULL cellH
 * invalidates the enthalpies, except with one species, whose mixing carries no
 * flux. A cp that is not finite and positive or an enthalpy that is not finite
 * sets bit 2 of the status word. */
int reactive_transport_wale_scalar_fields_device_v3(void* transport, const double* cellCp, const double* cellH,
    const double* fixedCp, const double* fixedH, size_t cpStride, size_t hStride, void* stream);
/* Device status word: bit 0 = WALE gradient/viscosity/traction non-finite,
 * bit 1 = an HLLC face could not be formed, bit 2 = an invalid WALE scalar
 * field from wale_scalar_fields_device_v3, bit 3 = a capillary face flux or
 * liquid inventory that could not be formed. Reading
 * it synchronises the handle's work on `stream`; clear=1 resets it afterwards. */
int reactive_transport_status_v3(void* transport, unsigned* status, int clear, void* stream);

#ifdef __cplusplus
}
#endif
#endif
