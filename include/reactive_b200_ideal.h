/* Ideal-gas mixture closure on B200: thermodynamic states of an ideal-gas
 * multi-species cell from its conserved variables, for the two-species
 * (N2O/N2) box whose closure the Peng-Robinson HEM does not cover
 * (src/reactiveThermo/reactiveGpuHemModel.inc:5).
 *
 * No C-ABI counterpart in the reference: its device closure for this case is
 * the scalar plugin reactive_closure_scalar_run_v1
 * (src/reactiveThermo/reactiveClosureAcceleration.h:41-42), which takes
 * host-prepared, composition-premixed NASA coefficients per cell and returns
 * (p, T, e, cv) to the host. These entries run the same recovery
 * (src/reactiveTransport/reactiveClosureScalar.cuh:9-57 with pr = 0: NASA
 * h(T), cv(T) and p = rho r T; a T bracket of up to 24 doublings, then up to 70
 * safeguarded Newton steps on e(T) = e) directly on device-resident SoA
 * conserved arrays, mixing the species' own NASA tables per cell, and write
 * the transport states the stage entries read. */
#ifndef REACTIVE_B200_IDEAL_H
#define REACTIVE_B200_IDEAL_H
#include <stddef.h>
#include "reactive_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* gasTable: a ReactiveB200Table (the gas table of the HEM model image; up to
 * four species, NASA7/9 regions, molecular weights). Temperatures are
 * recovered within [Tmin, Tmax]; tolerance is the relative energy tolerance of
 * the Newton (the reference's .25 tolerance max(1e5, cp T) rule). Returns NULL
 * with a message on invalid input. */
void* reactive_ideal_gas_create_v3(const void* gasTable, size_t tableBytes, double Tmin, double Tmax,
    double tolerance, char* error, size_t errorSize);
void reactive_ideal_gas_destroy_v3(void* gas);

/* Device arrays: conserved SoA q[k*stride + c] with variables = species + 4
 * (species masses, momentum, total energy); Tseed/T per cell (T may alias
 * Tseed); transport receives {p, T, rho, cv, sound, gasMass = rho, 0}; success
 * per cell (may be NULL). Asynchronous on `stream`; no allocation. */
int reactive_ideal_gas_run_device_v3(void* gas, const double* conserved, size_t stride, size_t count,
    size_t variables, const double* Tseed, double* T, ReactiveTransportState* transport, int* success,
    void* stream, char* error, size_t errorSize);

/* Vector-Jacobian product of the closure at converged temperatures T:
 * conservedBar[k*barStride + c] += sum over the transport-state fields of
 * transportBar[c].field * d field / d q[k][c]. The temperature's dependence on
 * q is taken by the implicit function theorem on e(T, Y) = e, not through the
 * Newton iterations. */
int reactive_ideal_gas_vjp_device_v3(void* gas, const double* conserved, size_t stride, size_t count,
    size_t variables, const double* T, const ReactiveTransportState* transportBar, double* conservedBar,
    size_t barStride, void* stream, char* error, size_t errorSize);

#ifdef __cplusplus
}
#endif
#endif
