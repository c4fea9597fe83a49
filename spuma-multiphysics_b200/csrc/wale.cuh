// Nicoud-Ducros WALE eddy viscosity, evaluated per cell on the device.
//
//   nu_t = (Cw*Delta)^2 (Sd:Sd)^(3/2) / ((S:S)^(5/2) + (Sd:Sd)^(5/4)),
//   S = sym(g), Sd = dev(sym(g g)), g[3i+j] = d u_i / d x_j, Delta = cbrt(V).
//
// Semantics follow src/reactiveTransport/reactiveWale.h: invariants are formed
// from g / max|g| so g*g cannot overflow or underflow on extreme unit scales
// (:87-136); nu_t = 0 exactly when Sd:Sd == 0, the gradient is zero, Cw == 0 or
// Delta == 0 (:157-161); the final (Cw^2 Delta^2 |g| ratio) product is assembled
// from frexp mantissas and a summed binary exponent so no intermediate squares
// overflow (:48-81). A non-finite result is an error, reported to the caller.
#pragma once
#include <cuda_runtime.h>

namespace rb200 {

// Returns false when the inputs or the result are not finite (the caller flags
// the cell as a WALE failure). R is double (the FP64 path) or float (the mixed
// path's FP32 WALE arithmetic); the operations are the same for both.
template <class R>
__device__ inline bool waleEddyViscosityT(const R g[9], R delta, R cw, R& nut) {
    nut = R(0);
    if (!isfinite(delta) || delta < R(0) || !isfinite(cw) || cw < R(0)) return false;
    R scale = R(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        if (!isfinite(g[i])) return false;
        scale = fmax(scale, fabs(g[i]));
    }
    if (scale == R(0) || cw == R(0) || delta == R(0)) return true;
    R h[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) h[i] = g[i] / scale;
    R sq[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            sq[3 * i + j] = h[3 * i] * h[j] + h[3 * i + 1] * h[3 + j] + h[3 * i + 2] * h[6 + j];
    const R trace = sq[0] + sq[4] + sq[8];
    R ss = R(0), dd = R(0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const R s = R(0.5) * (h[3 * i + j] + h[3 * j + i]);
            R d = R(0.5) * (sq[3 * i + j] + sq[3 * j + i]);
            if (i == j) d -= trace / R(3.0);
            ss += s * s;
            dd += d * d;
        }
    if (!isfinite(ss) || !isfinite(dd)) return false;
    if (dd == R(0)) return true;
    const R rootD = sqrt(dd);
    const R numerator = dd * rootD;                    // (Sd:Sd)^(3/2)
    const R denominator = ss * ss * sqrt(ss) + dd * sqrt(rootD);
    if (!(denominator > R(0)) || !isfinite(denominator) || !isfinite(numerator)) return false;
    const R ratio = numerator / denominator;
    if (ratio == R(0)) return true;
    int ec, ed, eg, er, em;
    const R mc = frexp(cw, &ec), md = frexp(delta, &ed);
    const R mg = frexp(scale, &eg), mr = frexp(ratio, &er);
    const R m = frexp(mc * mc * md * md * mg * mr, &em);
    nut = ldexp(m, 2 * ec + 2 * ed + eg + er + em);
    return isfinite(nut);
}

__device__ inline bool waleEddyViscosity(const double g[9], double delta, double cw, double& nut) {
    return waleEddyViscosityT<double>(g, delta, cw, nut);
}

}  // namespace rb200
