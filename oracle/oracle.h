/* TEST INFRASTRUCTURE ONLY. CPU restatements of the reference algorithms on the
 * hot path, used by tests/ and by bench.py's CPU-baseline leg as the checker;
 * never linked or loaded by the product library.
 *
 * Parity pinning: transport_oracle.c is checked against the reference's own CPU
 * transport build (oracle/_ref/libreactiveTransport_ref.so) on the reference's
 * validation cases; flash_oracle.c is checked against the reference's device
 * flash compiled for the host (oracle/_ref/libref_flash.so). */
#ifndef RB200_ORACLE_H
#define RB200_ORACLE_H
#include "reactive_b200_types.h"

/* Face-loop transport operator: rhs (cell-major cells x variables), boundary
 * ledger (variables), optional per-cell WALE nu_t (waleCw < 0 disables WALE) and
 * optional per-cell CFL denominator sum_f area*speed. Returns 0, or a nonzero
 * code when a WALE value or a face speed is invalid. */
void oracle_set_flux_scheme(int scheme);
void oracle_set_wale_scalars(double pr, double sc, const double* cellCp, const double* fixedCp,
                             const double* cellH, const double* fixedH);
int oracle_hllc_face(double rhoL, const double uL[3], double pL, double aL, double EL, double rhoR,
                     const double uR[3], double pR, double aR, double ER, const double normal[3], double out[5]);
int oracle_transport_rhs(const ReactiveTransportConfig* cfg, const double* volume,
    const ReactiveTransportFace* faces, const double* fixedQ, const ReactiveTransportState* fixedStates,
    const double* fixedY, const double* fixedH, double waleCw,
    const double* q, const ReactiveTransportState* states, const double* gasY, const double* gasH,
    double* rhs, double* boundary, double* nut, double* denominator);

/* min over cells of min(maximum, cfl * V / denominator); -1 when invalid. */
double oracle_transport_stable_dt(const ReactiveTransportConfig* cfg, const double* volume,
    const ReactiveTransportFace* faces, const double* fixedQ, const ReactiveTransportState* fixedStates,
    double waleCw, const double* q, const ReactiveTransportState* states, double cfl, double maximum);

/* WALE nu_t for one velocity gradient g[3i+j] = du_i/dx_j; returns 0 on invalid input. */
int oracle_wale_nut(const double* g, double delta, double cw, double* nut);

/* Pure-component (ns = 1, nl = 1) HEM UV flash over `count` cells; q holds one
 * mass density per cell, energy the internal energy density, guess the seed
 * states. counters: 7 per cell (phases, residuals, candidates, stable, failures,
 * analytic Jacobians, finite-difference Jacobians), may be null. Returns 1 for a
 * model outside the pure-component scope. */
int oracle_flash_recover(const char* image, size_t count, const double* q, const double* energy,
    const ReactiveThermoState* guess, ReactiveThermoState* out, int* success, uint64_t* counters, int threads);
int oracle_pr_evaluate_tp(const char* image, int table, double T, double p, int choice, int chem,
    double* out, int* phase);

#endif
