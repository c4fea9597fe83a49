/* Host-side helpers for callers of the host-array entry points (no reference
 * counterpart: the reference solver does this bookkeeping in its own parallel
 * loops, src/reactiveFoam/ReactiveFoam.C:419-420, :651-661, :732-751). Each runs
 * as a parallel loop over a persistent pool of host threads, synchronously,
 * with no device work. Return 0, or 1 for a null or inconsistent argument. */
#ifndef REACTIVE_B200_HOST_H
#define REACTIVE_B200_HOST_H
#include <stddef.h>
#include "reactive_b200_types.h"
#ifdef __cplusplus
extern "C" {
#endif
/* The pool's thread count. */
int reactive_b200_host_threads_v3(void);
/* dst[0..bytes) = src[0..bytes) (the regions must not overlap). */
int reactive_b200_host_copy_v3(void* dst, const void* src, size_t bytes);
/* The transport states of thermo states (p, T, rho, cv, frozen sound, gas mass,
 * dilatation 0) and, when primitives is not NULL, the primitives (rho of the
 * state, u = momentum / rho from the cell-major conserved rows q: species
 * masses, then three momentum components, qStride values per cell). */
int reactive_b200_host_transport_states_v3(const ReactiveThermoState* thermo, size_t count, const double* q,
    size_t qStride, size_t species, ReactiveTransportState* states, ReactiveTransportPrimitive* primitives);
/* The flash inputs of cell-major conserved rows: the species masses (masses
 * count x species, may be NULL) and the internal energy density E - |m|^2 / (2 rho). */
int reactive_b200_host_recovery_inputs_v3(const double* q, size_t count, size_t qStride, size_t species,
    double* masses, double* energy);
#ifdef __cplusplus
}
#endif
#endif
