/* Peng-Robinson mixture properties on B200 for the multi-species gas of the
 * reference's production case (air N2/O2, N2O and isopropanol in one PR phase).
 *
 * No C-ABI counterpart in the reference: its flash evaluates these properties
 * per state inside the device flash (ReactiveDevicePR::evaluateTrhoTrusted and
 * evaluateTPTrusted, src/reactiveThermo/reactiveDevicePR.h:474-609). This entry
 * runs the same evaluation over a batch of states, one thread per state, for
 * callers that need mixture properties on the device and as the first step of
 * the multi-species flash. */
#ifndef REACTIVE_B200_MIXTURE_H
#define REACTIVE_B200_MIXTURE_H
#include <stddef.h>
#include "reactive_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Properties of `count` states. All pointers are device pointers:
 *   table  a ReactiveB200Table (the HEM model image's gas-table layout) with
 *          1 to 4 species, uploaded by the caller; the host does not read it,
 *          so the caller validates it first (a table with another layout or a
 *          species count outside 1..4 gives status 1 per state, and a pointer
 *          that is not a device allocation of the table's size faults);
 *   T      temperatures [K];
 *   value  densities [kg/m^3] for mode 0 (T, rho, Y), pressures [Pa] for mode 1
 *          (T, p, Y) on the root `choice` picks (0: the largest, as the reference
 *          starts gas-side; 1 gas; 2 liquid);
 *   Y      mass fractions, 4 per state (entries past the table's species count
 *          are ignored; the table's entries must sum to 1 within 1e-12);
 *   out    19 doubles per state: T, p, W, V, rho, e, h, s, cp, cv, alpha,
 *          kappaT, sound, dp/dT, dp/dV, then the chemical potentials of the
 *          table's species [J/kmol] (per mass where the reference's State is);
 *   status the evaluator's code per state: 0 success, 1 invalid table,
 *          2 invalid input, 3 invalid composition, 4 no physical root,
 *          5 phase unavailable, 6 unstable state, 7 non-finite (the reference's
 *          ReactiveDevicePR::Status values);
 *   phase  the reported phase per state: -2 supercritical, -1 gas, 0 liquid.
 * out and phase are written only where status is 0. Asynchronous on `stream`;
 * no allocation. Returns 0, or 1 with a message on invalid arguments. */
int reactive_b200_mixture_properties_v3(const void* table, size_t count, const double* T, const double* value,
    const double* Y, int mode, int choice, double* out, int* status, int* phase, void* stream, char* error,
    size_t errorSize);

#ifdef __cplusplus
}
#endif
#endif
