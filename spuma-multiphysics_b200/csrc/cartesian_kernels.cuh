// Structured fast path of the transport for a uniform Cartesian box.
//
// When the face list is a uniform nx x ny x nz box in natural cell order
// (c = i + nx (j + ny k); internal faces (c, c+1), (c, c+nx), (c, c+nx ny) with
// normals +x, +y, +z; boundary faces on the six box sides), the operator is
// evaluated by cell stencils instead of a face graph: no face-work array and no
// CSR incidence are read. One kernel forms the Green-Gauss velocity gradient and
// the WALE viscosity of a cell from its six neighbours; a second computes the six
// face fluxes of a cell (HLL, viscous/WALE traction, conduction), sums them and
// applies the SSPRK2 update, so the flux of an internal face is computed by both
// of its cells instead of being stored and re-read. Boundary sides keep their own
// face records (kind, fixed index, weight, distance, area); in the canonical
// ordering the boundary faces of each box side form one contiguous block.
//
// The face physics is that of transport_kernels.cuh
// (src/reactiveTransport/reactiveTransportKernels.h:290-560). With an
// axis-aligned unit normal every projection reduces to one component; the
// terms a face graph multiplies by a zero normal component are still formed
// and added here (they are signed zeros for finite data), and a cell's faces are
// summed in its face-graph incidence order, so for finite data both paths give
// bitwise identical stage results.
#pragma once
#include "transport_kernels.cuh"
#include "dual.cuh"

namespace rb200 {

constexpr int kCartMaxNs = 4;

struct CartView {
    int nx, ny, nz;
    size_t cells, fixed, all;
    double area[3], dist[3];      // internal faces per axis (ownerWeight 0.5)
    const double* invV;
    const ReactiveTransportFace* face;
    size_t sideBase[6];           // -x,+x,-y,+y,-z,+z: first face of the side block
    size_t boundaryBase, nBoundary;
    const ReactiveTransportPrimitive* primitive;  // cells + fixed (velocities, as the face-graph kernels use)
    double viscosity, conductivity, waveFactor;
    bool wale;
    double cw;
    int scheme;  // 0 HLL, 1 HLLC
    // WALE scalar closure: turbulent Prandtl / Schmidt numbers (0 disables a
    // term), mixture cp (all) and effective species enthalpies (SoA ns x all)
    bool sgs;
    double pr, sc;
    const double* mixCp;
    const double* spH;
    // cells [ownBegin, ownEnd) are this handle's own: the stage update, the CFL
    // minimum and the boundary ledger cover them only (a z-slab's halo layers
    // are read as neighbours, and written by the halo exchange)
    size_t ownBegin, ownEnd;
    // scratch of the split stage (cartFaceFluxes / cartRatesFromFaces /
    // cartRatesBoxSides): one flux per interior face and variable, SoA (axis,
    // variable) x cells, indexed by the face's owner (the lower cell), and the
    // layout below; null where the split is unavailable
    double* faceFlux;
};

struct CellData {
    double q[kCartMaxNs + 4];
    double u[3];
    double p, T, rho, cv, c;
    double cp, h[kCartMaxNs];  // WALE scalar closure only
};

// A cell's flux inputs in arithmetic type R (double, float, or a dual number
// for the adjoint), each rounded from the FP64 data once.
template <class R> struct CellT {
    R q[kCartMaxNs + 4];
    R u[3];
    R p, T, rho, cv, c;
    R cp, h[kCartMaxNs];  // WALE scalar closure only
};
template <int NS, class R, bool SGS = false> __device__ __forceinline__ CellT<R> asCell(const CellData& d) {
    CellT<R> r;
#pragma unroll
    for (int k = 0; k < NS + 4; ++k) r.q[k] = R(d.q[k]);
#pragma unroll
    for (int a = 0; a < 3; ++a) r.u[a] = R(d.u[a]);
    r.p = R(d.p); r.T = R(d.T); r.rho = R(d.rho); r.cv = R(d.cv); r.c = R(d.c);
    if constexpr (SGS) {
        r.cp = R(d.cp);
#pragma unroll
        for (int k = 0; k < NS; ++k) r.h[k] = R(d.h[k]);
    }
    return r;
}

// SGS: also the cell's mixture cp (when Pr_t > 0) and, with its conserved
// variables, its species enthalpies (when Sc_t > 0).
template <int NS, bool SGS = false>
__device__ __forceinline__ void loadCell(const CartView& v, const double* __restrict__ q,
                                         const ReactiveTransportState* __restrict__ st, size_t c, CellData& d,
                                         bool needQ) {
    if (needQ) {
#pragma unroll
        for (int k = 0; k < NS + 4; ++k) d.q[k] = q[size_t(k) * v.all + c];
    }
    if constexpr (SGS) {
        d.cp = v.pr > 0 ? v.mixCp[c] : 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) d.h[k] = needQ && v.sc > 0 ? v.spH[size_t(k) * v.all + c] : 0.0;
    }
    const ReactiveTransportPrimitive pr = v.primitive[c];
#pragma unroll
    for (int a = 0; a < 3; ++a) d.u[a] = pr.u[a];
    const ReactiveTransportState s = st[c];
    d.p = s.p; d.T = s.T; d.rho = s.rho; d.cv = s.cv; d.c = s.sound;
}

// Right state of a boundary face of kind 1 (slip: velocity and momentum
// mirrored), 2 (extrapolate: owner), 3 (fixed state).
template <int NS, bool SGS = false>
__device__ __forceinline__ void boundaryRight(const CartView& v, const double* __restrict__ q,
                                              const ReactiveTransportState* __restrict__ st,
                                              const ReactiveTransportFace& f, int axis, const CellData& L,
                                              CellData& R, bool needQ) {
    if (f.kind == 3) {
        loadCell<NS, SGS>(v, q, st, v.cells + size_t(f.fixed), R, needQ);
        return;
    }
    R = L;
    if (f.kind == 1) {
        // u - 2 (u.n) n with n = +-e_axis: the component along the axis changes sign
        R.u[axis] = L.u[axis] - 2 * L.u[axis];
        if (needQ) R.q[NS + axis] = L.q[NS + axis] - 2 * L.q[NS + axis];
    }
}

// Unit normal component d of a face with normal sgn*e_axis.
template <class R> __device__ __forceinline__ R nrm(int d, int axis, R sgn) { return d == axis ? sgn : R(0); }
template <class R> __device__ __forceinline__ R rmin(R a, R b) { return a < b ? a : b; }
template <class R> __device__ __forceinline__ R rmax(R a, R b) { return a > b ? a : b; }

// Neumaier's compensated sum: s + c carries the sum of all added x to about
// twice the working precision.
__device__ __forceinline__ void twoSum(float& s, float& c, float x) {
    const float t = s + x;
    c += fabsf(s) >= fabsf(x) ? (s - t) + x : (x - t) + s;
    s = t;
}

// Flux of all variables through a face with unit normal sgn*e_axis, times the
// area, seen from the owner (left) side (faceWork + faceFluxK of the face graph).
// gL/gR: gradients (9 components; gR only used for internal faces); nutL/nutR
// the WALE viscosities of the owner and right sides. R is the arithmetic type:
// double on the FP64 path (the face graph's exact operation sequence), float
// on the mixed path (inputs rounded to FP32 once, every operation in FP32).
// SGS adds the WALE scalar closure: the turbulent heat flux rho nu_t cp / Pr_t
// (T_R - T_L) / d and the turbulent species mixing of total mass fractions with
// its enthalpy flux, in the face graph's operation order
// (src/reactiveTransport/reactiveTransportKernels.h:150-168, :440-477).
template <int NS, class R, bool SGS = false>
__device__ __forceinline__ void faceFluxCart(const CartView& v, int axis, double sgnD, double areaD, double distD,
                                             double wD, int kind, bool internal, const CellT<R>& L,
                                             const CellT<R>& Rt, const R* gL, const R* gR, R nutL, R nutR, R* F,
                                             bool& bad, bool& faceBad) {
    const R sgn = R(sgnD), w = R(wD), dist = R(distD), area = R(areaD);
    const R unL = L.u[axis] * sgn, unR = Rt.u[axis] * sgn;
    const R aL = R(v.waveFactor) * L.c, aR = R(v.waveFactor) * Rt.c;
    const R left = rmin(R(0), rmin(unL - aL, unR - aR)), right = rmax(R(0), rmax(unL + aL, unR + aR));
    const R inv = R(1) / (right - left);
    R advL = right * (unL - left) * inv, advR = left * (right - unR) * inv;
    const R pL = L.p, pR = Rt.p;
    R pM = (right * pL - left * pR) * inv, pE = (right * pL * unL - left * pR * unR) * inv;
    if (v.scheme == 1) {
        // HLLC: the reference's contact-preserving core with no capillary terms
        // (src/reactiveInterface/reactiveBalancedCapillary.h:55-142, applied by
        // src/reactiveTransport/reactiveTransportKernels.h:357-417). The HLL
        // coefficients above stand when the star speed leaves the wave fan.
        const R rhoL = L.rho, rhoR = Rt.rho;
        const R den = rhoL * (left - unL) - rhoR * (right - unR);
        if (!(rhoL > R(0) && rhoR > R(0) && pL > R(0) && pR > R(0) && isfinite(den) && den != R(0)
              && right > left)) {
            faceBad = true;
        } else {
            const R star = (pR - pL + rhoL * unL * (left - unL) - rhoR * unR * (right - unR)) / den;
            if (isfinite(star) && star > left && star < right) {
                const bool useLeft = star >= R(0);
                const R rho = useLeft ? rhoL : rhoR, un = useLeft ? unL : unR, wave = useLeft ? left : right;
                const R p = useLeft ? pL : pR, E = useLeft ? L.q[NS + 3] : Rt.q[NS + 3];
                const bool supersonic = (useLeft && left >= R(0)) || (!useLeft && right <= R(0));
                R mass;
                if (supersonic) {
                    mass = rho * un;
                    pM = p;
                    pE = p * un;
                } else {
                    const R rhoStar = rho * (wave - un) / (wave - star);
                    const R pStar = p + rho * (wave - un) * (star - un);
                    const R eStar = ((wave - un) * E - p * un + pStar * star) / (wave - star);
                    mass = rhoStar * star;
                    pM = pStar + mass * (star - un);
                    pE = star * (eStar + pStar) - mass * E / rho;
                }
                advL = useLeft ? mass / rhoL : R(0);
                advR = useLeft ? R(0) : mass / rhoR;
            }
        }
    }
    R traction[3] = {R(0), R(0), R(0)}, energy = R(0);
    if (v.viscosity > 0 || v.wale) {
        const R* uL = L.u;
        const R* uR = Rt.u;
        R g[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) g[j] = internal ? w * gL[j] + (R(1) - w) * gR[j] : gL[j];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            R normal = R(0);
#pragma unroll
            for (int d = 0; d < 3; ++d) normal += g[i * 3 + d] * nrm(d, axis, sgn);
            const R target = (uR[i] - uL[i]) / (R(kind == 1 ? 2 : 1) * dist);
#pragma unroll
            for (int d = 0; d < 3; ++d) g[i * 3 + d] += nrm(d, axis, sgn) * (target - normal);
        }
        const R div = g[0] + g[4] + g[8];
        const R mu = R(v.viscosity) + (v.wale ? w * L.rho * nutL + (R(1) - w) * Rt.rho * nutR : R(0));
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int d = 0; d < 3; ++d)
                traction[i] += mu * (g[3 * i + d] + g[3 * d + i] - (i == d ? R(2) * div / R(3) : R(0)))
                    * nrm(d, axis, sgn);
        if (kind == 1) {
            R dot = R(0);
#pragma unroll
            for (int d = 0; d < 3; ++d) dot += traction[d] * nrm(d, axis, sgn);
#pragma unroll
            for (int d = 0; d < 3; ++d) traction[d] = dot * nrm(d, axis, sgn);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) energy -= traction[d] * (w * uL[d] + (R(1) - w) * uR[d]);
    }
    if (v.conductivity > 0 && kind != 1) energy -= R(v.conductivity) * (Rt.T - L.T) / dist;
    R sgsJ[NS], sgsD = R(0), sgsSum = R(0), sgsCarrierFlux = R(0);
#pragma unroll
    for (int k = 0; k < NS; ++k) sgsJ[k] = R(0);
    if constexpr (SGS) {
        if (v.pr > 0 && kind != 1) {
            const R rhoNut = w * L.rho * nutL + (R(1) - w) * Rt.rho * nutR;
            const R cp = w * L.cp + (R(1) - w) * Rt.cp;
            energy -= rhoNut * cp / R(v.pr) * (Rt.T - L.T) / dist;
        }
        if (v.sc > 0 && kind != 1) {
            const R rhoNut = w * L.rho * nutL + (R(1) - w) * Rt.rho * nutR;
            sgsD = -rhoNut / R(v.sc) / dist;
            R largest = R(-1), yL[NS], yR[NS];
            int carrier = 0;
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                yL[k] = L.q[k] / L.rho;
                yR[k] = Rt.q[k] / Rt.rho;
                sgsSum += sgsD * (yR[k] - yL[k]);
                const R y = w * yL[k] + (R(1) - w) * yR[k];
                if (y > largest) { largest = y; carrier = k; }
            }
            R hc = R(0);
#pragma unroll
            for (int k = 0; k < NS; ++k)
                if (k == carrier) hc = w * L.h[k] + (R(1) - w) * Rt.h[k];
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                if (k == carrier) continue;
                const R J = sgsD * (yR[k] - yL[k]) - (w * yL[k] + (R(1) - w) * yR[k]) * sgsSum;
                sgsCarrierFlux -= J;
                energy += J * ((w * L.h[k] + (R(1) - w) * Rt.h[k]) - hc);
                sgsJ[k] = J;
            }
#pragma unroll
            for (int k = 0; k < NS; ++k)
                if (k == carrier) sgsJ[k] = sgsCarrierFlux;
        }
    }
    if (v.wale) {
        bad |= !isfinite(energy) || !isfinite(sgsD) || !isfinite(sgsSum) || !isfinite(sgsCarrierFlux);
#pragma unroll
        for (int d = 0; d < 3; ++d) bad |= !isfinite(traction[d]);
    }
#pragma unroll
    for (int k = 0; k < NS + 4; ++k) {
        R flux = advL * L.q[k] + advR * Rt.q[k];
        if (k >= NS && k < NS + 3) flux += pM * nrm(k - NS, axis, sgn);
        if (k == NS + 3) flux += pE;
        if (k < NS) {
            // species diffusion: no molecular term on this path, the mixing flux when on
            R diffusion = R(0);
            if (sgsD != R(0)) diffusion += sgsJ[k];
            flux += diffusion;
        } else if (k < NS + 3) flux -= traction[k - NS];
        else if (k == NS + 3) flux += energy;
        F[k] = flux * area;
    }
}

__device__ __forceinline__ void cellCoords(const CartView& v, size_t c, int& i, int& j, int& k) {
    i = int(c % size_t(v.nx));
    const size_t r = c / size_t(v.nx);
    j = int(r % size_t(v.ny));
    k = int(r / size_t(v.ny));
}

// Face record of box side s (-x,+x,-y,+y,-z,+z) at cell (i, j, k).
__device__ __forceinline__ const ReactiveTransportFace& sideFace(const CartView& v, int s, int i, int j, int k) {
    const size_t lateral = s < 2 ? size_t(j) + size_t(v.ny) * k
                                 : (s < 4 ? size_t(i) + size_t(v.nx) * k : size_t(i) + size_t(v.nx) * j);
    return v.face[v.sideBase[s] + lateral];
}

// The n-th side of a cell in its face-graph incidence order for the canonical
// ordering: internal faces are sorted by (owner, neighbour), so a cell meets the
// faces it neighbours (-z, -y, -x) before those it owns (+x, +y, +z); the
// boundary faces follow in side-block order (-x, +x, -y, +y, -z, +z). n < 6
// walks the internal sides, n >= 6 the boundary sides.
__device__ __forceinline__ int sideOf(int n) {
    constexpr int order[6] = {4, 2, 0, 1, 3, 5};
    return n < 6 ? order[n] : n - 6;
}

__device__ __forceinline__ bool hasNeighbour(const CartView& v, int s, int i, int j, int k) {
    const int coord = s < 2 ? i : (s < 4 ? j : k);
    const int dim = s < 2 ? v.nx : (s < 4 ? v.ny : v.nz);
    return (s & 1) ? coord + 1 < dim : coord > 0;
}

__device__ __forceinline__ size_t neighbourOf(const CartView& v, int s, size_t c) {
    const size_t step = s < 2 ? 1 : (s < 4 ? size_t(v.nx) : size_t(v.nx) * v.ny);
    return (s & 1) ? c + step : c - step;
}

// Green-Gauss gradient (and the WALE viscosity) of every cell, in arithmetic
// type R (stored as R: 9 gradient components and nu_t per cell).
template <int NS, class R>
__global__ void __launch_bounds__(256) cartGradients(CartView v, const ReactiveTransportState* __restrict__ st,
                                                     R* __restrict__ grad, R* __restrict__ nut, unsigned* error) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        int i, j, k;
        cellCoords(v, c, i, j, k);
        CellData C;
        loadCell<NS>(v, nullptr, st, c, C, false);
        R g[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        const R iv = R(v.invV[c]);
#pragma unroll
        for (int n = 0; n < 12; ++n) {
            const int s = sideOf(n);
            const bool interior = hasNeighbour(v, s, i, j, k);
            if (interior != (n < 6)) continue;
            const int axis = s >> 1;
            R uf[3], scale, sgn;
            if (interior) {
                // internal face: owner is the lower cell, normal +e_axis; this cell's
                // incidence sign is +1 on its upper side (owner), -1 on its lower side
                const ReactiveTransportPrimitive pn = v.primitive[neighbourOf(v, s, c)];
                const bool owner = s & 1;
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    uf[a] = owner ? R(.5) * R(C.u[a]) + (R(1) - R(.5)) * R(pn.u[a])
                                  : R(.5) * R(pn.u[a]) + (R(1) - R(.5)) * R(C.u[a]);
                scale = R(owner ? 1.0 : -1.0) * R(v.area[axis]) * iv;
                sgn = R(1);
            } else {
                const ReactiveTransportFace& f = sideFace(v, s, i, j, k);
                CellData Rt;
                boundaryRight<NS>(v, nullptr, st, f, axis, C, Rt, false);
                const R w = R(f.ownerWeight);
#pragma unroll
                for (int a = 0; a < 3; ++a) uf[a] = w * R(C.u[a]) + (R(1) - w) * R(Rt.u[a]);
                scale = R(1.0) * R(f.area) * iv;
                sgn = (s & 1) ? R(1) : R(-1);
            }
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d) g[3 * a + d] += uf[a] * nrm(d, axis, sgn) * scale;
        }
#pragma unroll
        for (int jj = 0; jj < 9; ++jj) grad[size_t(jj) * v.cells + c] = g[jj];
        if (v.wale) {
            const R volume = R(1) / iv;
            R delta = R(0), nu = R(0);
            bool ok = isfinite(volume) && volume > R(0);
            if (ok) { delta = cbrt(volume); ok = isfinite(delta) && delta > R(0); }
            ok = ok && waleEddyViscosityT<R>(g, delta, R(v.cw), nu);
            if (!ok || !isfinite(nu) || nu < R(0) || !isfinite(R(C.rho) * nu)) atomicOr(error, 1u);
            else nut[c] = nu;
        }
    }
}

// The flux of side s of cell c and this cell's incidence sign for it.
template <int NS, class R, bool SGS = false>
__device__ __forceinline__ void sideFlux(const CartView& v, const double* __restrict__ q,
                                         const ReactiveTransportState* __restrict__ st,
                                         const R* __restrict__ grad, const R* __restrict__ nut, size_t c,
                                         int s, bool interior, int i, int j, int k, const CellData& C,
                                         const R* gC, R nutC, R* F, double& sign, bool& bad, bool& faceBad) {
    const int axis = s >> 1;
    const bool viscous = v.viscosity > 0 || v.wale;
    if (interior) {
        const size_t nb = neighbourOf(v, s, c);
        CellData N;
        loadCell<NS, SGS>(v, q, st, nb, N, true);
        R gN[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (viscous) {
#pragma unroll
            for (int jj = 0; jj < 9; ++jj) gN[jj] = grad[size_t(jj) * v.cells + nb];
        }
        const R nutN = v.wale ? nut[nb] : R(0);
        const CellT<R> cc = asCell<NS, R, SGS>(C), cn = asCell<NS, R, SGS>(N);
        if (s & 1) {  // this cell owns the face
            faceFluxCart<NS, R, SGS>(v, axis, 1.0, v.area[axis], v.dist[axis], .5, 0, true, cc, cn, gC, gN, nutC,
                                     nutN, F, bad, faceBad);
            sign = -1;
        } else {
            faceFluxCart<NS, R, SGS>(v, axis, 1.0, v.area[axis], v.dist[axis], .5, 0, true, cn, cc, gN, gC, nutN,
                                     nutC, F, bad, faceBad);
            sign = 1;
        }
    } else {
        const ReactiveTransportFace& f = sideFace(v, s, i, j, k);
        CellData Rt;
        boundaryRight<NS, SGS>(v, q, st, f, axis, C, Rt, true);
        // a boundary face's right-side WALE viscosity is the owner's
        faceFluxCart<NS, R, SGS>(v, axis, (s & 1) ? 1.0 : -1.0, f.area, f.distance, f.ownerWeight, f.kind, false,
                                 asCell<NS, R, SGS>(C), asCell<NS, R, SGS>(Rt), gC, gC, nutC, nutC, F, bad, faceBad);
        sign = -1;
    }
}

// Sum of the six face fluxes of every cell and the SSPRK2 update:
// mode 0 rate -> out (stride outStride), 1 out = q + dt rate,
// 2 out = .5 out + .5 (q + dt rate) (out holds q^n).
// R = double: the face graph's FP64 sums. R = float (mixed): FP32 face fluxes,
// summed per cell with Neumaier compensation (the sum and its error term are
// added in FP64), divided by the volume in FP64, and the update applied to the
// FP64 conserved state in FP64. Each internal face's FP32 flux is computed from
// the same inputs by both of its cells, so it cancels exactly between them.
template <int NS, class R, bool SGS = false>
__global__ void __launch_bounds__(128) cartRates(CartView v, const double* __restrict__ q,
                                                 const ReactiveTransportState* __restrict__ st,
                                                 const R* __restrict__ grad, const R* __restrict__ nut,
                                                 double* out, size_t outStride, int mode, double dt,
                                                 unsigned* error) {
    constexpr bool fp64 = sizeof(R) == sizeof(double);
    const bool viscous = v.viscosity > 0 || v.wale;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        if (c < v.ownBegin || c >= v.ownEnd) continue;
        int i, j, k;
        cellCoords(v, c, i, j, k);
        CellData C;
        loadCell<NS, SGS>(v, q, st, c, C, true);
        R gC[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (viscous) {
#pragma unroll
            for (int jj = 0; jj < 9; ++jj) gC[jj] = grad[size_t(jj) * v.cells + c];
        }
        const R nutC = v.wale ? nut[c] : R(0);
        const double iv = v.invV[c];
        R rate[NS + 4], comp[NS + 4];
#pragma unroll
        for (int kk = 0; kk < NS + 4; ++kk) rate[kk] = comp[kk] = R(0);
        bool bad = false, faceBad = false;
#pragma unroll
        for (int n = 0; n < 12; ++n) {
            const int s = sideOf(n);
            const bool interior = hasNeighbour(v, s, i, j, k);
            if (interior != (n < 6)) continue;
            R F[NS + 4];
            double sign;
            sideFlux<NS, R, SGS>(v, q, st, grad, nut, c, s, interior, i, j, k, C, gC, nutC, F, sign, bad, faceBad);
#pragma unroll
            for (int kk = 0; kk < NS + 4; ++kk) {
                if constexpr (fp64) rate[kk] += sign * F[kk] * iv;
                else twoSum(rate[kk], comp[kk], sign > 0 ? F[kk] : -F[kk]);
            }
        }
        if (bad) atomicOr(error, 1u);
        if (faceBad) atomicOr(error, 2u);
#pragma unroll
        for (int kk = 0; kk < NS + 4; ++kk) {
            const double r = fp64 ? double(rate[kk]) : (double(rate[kk]) + double(comp[kk])) * iv;
            const size_t o = size_t(kk) * outStride + c;
            if (mode == 0) out[o] = r;
            else if (mode == 1) out[o] = C.q[kk] + dt * r;
            else out[o] = .5 * out[o] + .5 * (C.q[kk] + dt * r);
        }
    }
}

// ---------------------------------------------------------------------------
// The stage split in three launches, each interior face's flux evaluated once
// instead of once by each of its two cells. cartFaceFluxes: the owner (lower
// cell) of every +x/+y/+z interior face with an own cell on either side
// evaluates it in the owner orientation, exactly the call both cells' per-cell
// evaluations make (faceFluxCart, the same inputs), into v.faceFlux.
// cartRatesFromFaces and cartRatesBoxSides: every own cell sums its six faces
// in its face-graph incidence order (-z, -y, -x, +x, +y, +z, then the box
// sides, evaluated as cartRates does) with the same signs and scaling, and
// applies the same update: the results are bitwise cartRates<NS, R>'s (FP64,
// and FP32 faces with the compensated sums continued in the same order).
// (defined with the CFL kernels below)
template <bool SGS = false>
__device__ __forceinline__ double faceSpeedCart(const CartView& v, int axis, double sgn, double dist, double w,
                                                int kind, const CellData& L, const CellData& R, double nutL,
                                                double nutR);

// The split stage's scratch in v.faceFlux, in doubles: the face fluxes
// (3 NQ cells), the box-side cells' partial sums (NQ cells), with the CFL pass
// the +x/+y/+z face speeds (3 cells), the box-side cells' partial
// denominators (cells) and the per-block step minima of both kernels.
constexpr size_t kSplitStepPartials = 2 * size_t(kSmCount) * 8 * 16;
__host__ __device__ inline size_t splitSpeedOffset(int nq, size_t cells) { return 4 * size_t(nq) * cells; }
__host__ __device__ inline size_t splitDenominatorOffset(int nq, size_t cells) { return (4 * size_t(nq) + 3) * cells; }
__host__ __device__ inline size_t splitStepOffset(int nq, size_t cells) { return (4 * size_t(nq) + 4) * cells; }
__host__ __device__ inline size_t splitScratchDoubles(int nq, size_t cells, bool cflPass) {
    return cflPass ? splitStepOffset(nq, cells) + kSplitStepPartials : 4 * size_t(nq) * cells;
}

// One block's minimum of m into partial[block] (all threads of the block).
__device__ __forceinline__ void blockMinimum(double m, double* partial) {
    __shared__ double warpValues[32];
    m = warpMin(m);
    if ((threadIdx.x & 31) == 0) warpValues[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? warpValues[threadIdx.x] : HUGE_VAL;
        m = warpMin(m);
        if (threadIdx.x == 0) partial[blockIdx.x] = m;
    }
}

// A cell's CFL step from its face-speed denominator, as cartSteps forms it.
__device__ __forceinline__ double cellStep(const CartView& v, size_t c, double denominator, bool bad, double cfl,
                                           double maximumStep) {
    double step = denominator > 0 ? dmin(maximumStep, cfl / (v.invV[c] * denominator)) : maximumStep;
    if (bad || !isfinite(denominator) || denominator < 0) step = -1;
    return isfinite(step) && step > 0 ? step : -1.0;
}

// With `cfl` > 0 the split stage also forms the CFL step of the same state
// (cartSteps' per-cell steps from the same face speeds, each face's speed
// evaluated once): the minimum over both kernels' block minima
// (minimumReduce) is bitwise cartSteps'.
// Four blocks of 128 per SM (at most 128 registers) measured 7% faster at
// 160^3 than the compiler's own 151 registers at three.
#ifndef RB200_FACE_MINBLOCKS
#define RB200_FACE_MINBLOCKS 4
#endif
template <int NS, class R, bool SGS = false>
__global__ void __launch_bounds__(128, RB200_FACE_MINBLOCKS) cartFaceFluxes(CartView v, const double* __restrict__ q,
                                                      const ReactiveTransportState* __restrict__ st,
                                                      const R* __restrict__ grad, const R* __restrict__ nut,
                                                      unsigned* error, bool cflPass) {
    constexpr int NQ = NS + 4;
    const bool viscous = v.viscosity > 0 || v.wale;
    R* flux = reinterpret_cast<R*>(v.faceFlux);
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        int i, j, k;
        cellCoords(v, c, i, j, k);
        const bool ownC = c >= v.ownBegin && c < v.ownEnd;
        bool any = false;
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const int s = 2 * axis + 1;
            if (!hasNeighbour(v, s, i, j, k)) continue;
            const size_t nb = neighbourOf(v, s, c);
            any = any || ownC || (nb >= v.ownBegin && nb < v.ownEnd);
        }
        if (!any) continue;
        CellData C;
        loadCell<NS, SGS>(v, q, st, c, C, true);
        R gC[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (viscous) {
#pragma unroll
            for (int jj = 0; jj < 9; ++jj) gC[jj] = grad[size_t(jj) * v.cells + c];
        }
        const R nutC = v.wale ? nut[c] : R(0);
        const CellT<R> cc = asCell<NS, R, SGS>(C);
        bool bad = false, faceBad = false;
#pragma unroll 1
        for (int axis = 0; axis < 3; ++axis) {
            const int s = 2 * axis + 1;
            if (!hasNeighbour(v, s, i, j, k)) continue;
            const size_t nb = neighbourOf(v, s, c);
            if (!ownC && !(nb >= v.ownBegin && nb < v.ownEnd)) continue;
            CellData N;
            loadCell<NS, SGS>(v, q, st, nb, N, true);
            R gN[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
            if (viscous) {
#pragma unroll
                for (int jj = 0; jj < 9; ++jj) gN[jj] = grad[size_t(jj) * v.cells + nb];
            }
            const R nutN = v.wale ? nut[nb] : R(0);
            R F[NQ];
            faceFluxCart<NS, R, SGS>(v, axis, 1.0, v.area[axis], v.dist[axis], .5, 0, true, cc,
                                     asCell<NS, R, SGS>(N), gC, gN, nutC, nutN, F, bad, faceBad);
#pragma unroll
            for (int kk = 0; kk < NQ; ++kk) flux[(size_t(axis) * NQ + kk) * v.cells + c] = F[kk];
            if (cflPass)
                v.faceFlux[splitSpeedOffset(NQ, v.cells) + size_t(axis) * v.cells + c] =
                    faceSpeedCart<SGS>(v, axis, 1.0, v.dist[axis], .5, 0, C, N, double(nutC), double(nutN));
        }
        if (bad) atomicOr(error, 1u);
        if (faceBad) atomicOr(error, 2u);
    }
}

// A cell's sums over its faces, as cartRates forms them: FP64 adds each face's
// sign * F / V; FP32 (mixed) keeps the Neumaier pair (sum, error) of the signed
// fluxes and divides by the volume at the end in FP64.
template <class R> struct FaceSums {
    R rate, comp;
    __device__ __forceinline__ void add(double sign, R F, double iv) {
        if constexpr (sizeof(R) == sizeof(double)) rate += sign * F * iv;
        else twoSum(rate, comp, sign > 0 ? F : -F);
    }
    __device__ __forceinline__ double value(double iv) const {
        if constexpr (sizeof(R) == sizeof(double)) return double(rate);
        else return (double(rate) + double(comp)) * iv;
    }
};

// Every own cell's interior faces in its incidence order (-z, -y, -x, +x, +y,
// +z) from the face fluxes, and for a cell off the box sides the update. A
// cell on a box side leaves its partial sums in the scratch after the face
// fluxes (variable-major, stride cells; FP32: the sums then their errors) for
// cartRatesBoxSides, which adds its box-side faces in cartRates' order and
// applies the update: the two kernels together give cartRates' sums bit for
// bit, and this one stays light (no boundary flux code, far fewer registers).
template <int NS, class R>
__global__ void __launch_bounds__(256) cartRatesFromFaces(CartView v, const double* __restrict__ q, double* out,
                                                          size_t outStride, int mode, double dt, double cfl,
                                                          double maximumStep) {
    constexpr int NQ = NS + 4;
    const R* __restrict__ flux = reinterpret_cast<const R*>(v.faceFlux);
    R* partial = reinterpret_cast<R*>(v.faceFlux + size_t(3) * NQ * v.cells);
    const double* speed = v.faceFlux + splitSpeedOffset(NQ, v.cells);
    double* denominators = v.faceFlux + splitDenominatorOffset(NQ, v.cells);
    const bool cflPass = cfl > 0;
    double m = maximumStep;  // as cartSteps starts its minimum
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        if (c < v.ownBegin || c >= v.ownEnd) continue;
        int i, j, k;
        cellCoords(v, c, i, j, k);
        const bool edge = i == 0 || i + 1 == v.nx || j == 0 || j + 1 == v.ny || k == 0 || k + 1 == v.nz;
        const double iv = v.invV[c];
        FaceSums<R> sum[NQ];
#pragma unroll
        for (int kk = 0; kk < NQ; ++kk) sum[kk] = FaceSums<R>{R(0), R(0)};
#pragma unroll
        for (int n = 0; n < 6; ++n) {
            const int s = sideOf(n);
            if (!hasNeighbour(v, s, i, j, k)) continue;
            const int axis = s >> 1;
            const size_t owner = (s & 1) ? c : neighbourOf(v, s, c);
            const double sign = (s & 1) ? -1 : 1;
#pragma unroll
            for (int kk = 0; kk < NQ; ++kk) sum[kk].add(sign, flux[(size_t(axis) * NQ + kk) * v.cells + owner], iv);
        }
        if (cflPass) {
            // cartSteps' denominator over the interior faces, in the same order
            double denominator = 0;
            bool bad = false;
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                const int s = sideOf(n);
                if (!hasNeighbour(v, s, i, j, k)) continue;
                const int axis = s >> 1;
                const size_t owner = (s & 1) ? c : neighbourOf(v, s, c);
                const double sp = speed[size_t(axis) * v.cells + owner];
                if (!isfinite(sp) || sp < 0) bad = true;
                else if (!bad) denominator += v.area[axis] * sp;
            }
            if (edge) denominators[c] = bad ? NAN : denominator;
            else m = fmin(m, cellStep(v, c, denominator, bad, cfl, maximumStep));
        }
        if (edge) {
#pragma unroll
            for (int kk = 0; kk < NQ; ++kk) {
                partial[size_t(kk) * v.cells + c] = sum[kk].rate;
                if constexpr (sizeof(R) != sizeof(double)) partial[size_t(NQ + kk) * v.cells + c] = sum[kk].comp;
            }
            continue;
        }
#pragma unroll
        for (int kk = 0; kk < NQ; ++kk) {
            const double r = sum[kk].value(iv), qk = q[size_t(kk) * v.all + c];
            const size_t o = size_t(kk) * outStride + c;
            if (mode == 0) out[o] = r;
            else if (mode == 1) out[o] = qk + dt * r;
            else out[o] = .5 * out[o] + .5 * (qk + dt * r);
        }
    }
    if (cflPass) blockMinimum(m, v.faceFlux + splitStepOffset(NQ, v.cells));
}

// Cells on the box's sides: the two end planes in z, then per inner plane its
// rows j = 0 and j = ny - 1 and its columns i = 0 and i = nx - 1 between them
// (every dimension at least 3).
__device__ __forceinline__ size_t shellCells(const CartView& v) {
    return 2 * size_t(v.nx) * v.ny + size_t(v.nz - 2) * (2 * size_t(v.nx) + 2 * size_t(v.ny - 2));
}
__device__ __forceinline__ size_t shellCell(const CartView& v, size_t e) {
    const size_t nx = v.nx, ny = v.ny, plane = nx * ny;
    if (e < 2 * plane) return e < plane ? e : e - plane + (size_t(v.nz) - 1) * plane;
    e -= 2 * plane;
    const size_t ring = 2 * nx + 2 * (ny - 2), k = 1 + e / ring, r = e % ring;
    size_t i, j;
    if (r < 2 * nx) {
        j = r < nx ? 0 : ny - 1;
        i = r < nx ? r : r - nx;
    } else {
        j = 1 + (r - 2 * nx) / 2;
        i = ((r - 2 * nx) & 1) ? nx - 1 : 0;
    }
    return i + nx * (j + ny * k);
}

// The box-side faces of the own cells on the box's sides (after
// cartRatesFromFaces), in cartRates' order, and their update: over the shell
// of side cells, or over every cell when a dimension is below 3.
template <int NS, class R, bool SGS = false>
__global__ void __launch_bounds__(128) cartRatesBoxSides(CartView v, const double* __restrict__ q,
                                                         const ReactiveTransportState* __restrict__ st,
                                                         const R* __restrict__ grad, const R* __restrict__ nut,
                                                         double* out, size_t outStride, int mode, double dt,
                                                         unsigned* error, double cfl, double maximumStep,
                                                         unsigned stepBase) {
    constexpr int NQ = NS + 4;
    const bool viscous = v.viscosity > 0 || v.wale;
    const R* partial = reinterpret_cast<const R*>(v.faceFlux + size_t(3) * NQ * v.cells);
    const double* denominators = v.faceFlux + splitDenominatorOffset(NQ, v.cells);
    const bool cflPass = cfl > 0;
    double m = maximumStep;
    const bool shell = v.nx >= 3 && v.ny >= 3 && v.nz >= 3;
    const size_t items = shell ? shellCells(v) : v.cells;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < items; e += size_t(blockDim.x) * gridDim.x) {
        const size_t c = shell ? shellCell(v, e) : e;
        if (c < v.ownBegin || c >= v.ownEnd) continue;
        int i, j, k;
        cellCoords(v, c, i, j, k);
        if (!(i == 0 || i + 1 == v.nx || j == 0 || j + 1 == v.ny || k == 0 || k + 1 == v.nz)) continue;
        CellData C;
        loadCell<NS, SGS>(v, q, st, c, C, true);
        R gC[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (viscous) {
#pragma unroll
            for (int jj = 0; jj < 9; ++jj) gC[jj] = grad[size_t(jj) * v.cells + c];
        }
        const R nutC = v.wale ? nut[c] : R(0);
        const double iv = v.invV[c];
        FaceSums<R> sum[NQ];
#pragma unroll
        for (int kk = 0; kk < NQ; ++kk) {
            sum[kk].rate = partial[size_t(kk) * v.cells + c];
            sum[kk].comp = sizeof(R) == sizeof(double) ? R(0) : partial[size_t(NQ + kk) * v.cells + c];
        }
        bool bad = false, faceBad = false;
#pragma unroll
        for (int n = 6; n < 12; ++n) {
            const int s = sideOf(n);
            if (hasNeighbour(v, s, i, j, k)) continue;
            R F[NQ];
            double sign;
            sideFlux<NS, R, SGS>(v, q, st, grad, nut, c, s, false, i, j, k, C, gC, nutC, F, sign, bad, faceBad);
#pragma unroll
            for (int kk = 0; kk < NQ; ++kk) sum[kk].add(sign, F[kk], iv);
        }
        if (bad) atomicOr(error, 1u);
        if (faceBad) atomicOr(error, 2u);
        if (cflPass) {
            // the box sides' speeds after the interior faces', as cartSteps adds them
            double denominator = denominators[c];
            bool badSpeed = isnan(denominator);
#pragma unroll
            for (int n = 6; n < 12; ++n) {
                const int s = sideOf(n);
                if (hasNeighbour(v, s, i, j, k) || badSpeed) continue;
                const int axis = s >> 1;
                const ReactiveTransportFace& f = sideFace(v, s, i, j, k);
                CellData Rt;
                boundaryRight<NS, SGS>(v, nullptr, st, f, axis, C, Rt, false);
                const double sp = faceSpeedCart<SGS>(v, axis, (s & 1) ? 1.0 : -1.0, f.distance, f.ownerWeight,
                                                     f.kind, C, Rt, double(nutC), double(nutC));
                if (!isfinite(sp) || sp < 0) badSpeed = true;
                else denominator += f.area * sp;
            }
            m = fmin(m, cellStep(v, c, denominator, badSpeed, cfl, maximumStep));
        }
#pragma unroll
        for (int kk = 0; kk < NQ; ++kk) {
            const double r = sum[kk].value(iv);
            const size_t o = size_t(kk) * outStride + c;
            if (mode == 0) out[o] = r;
            else if (mode == 1) out[o] = C.q[kk] + dt * r;
            else out[o] = .5 * out[o] + .5 * (C.q[kk] + dt * r);
        }
    }
    if (cflPass) blockMinimum(m, v.faceFlux + splitStepOffset(NQ, v.cells) + stepBase);
}

// ---------------------------------------------------------------------------
// The stage kernel with its face stencils staged through shared memory.
//
// A block owns a kTileX x kTileY tile of an x-y plane and marches a chunk of
// kTileZ planes in z. Per plane, the flux inputs of the tile's cells and of a
// one-cell halo ring in x and y are loaded once into shared memory (SoA, in the
// arithmetic type R); every x and y face of the tile's cells is then evaluated
// ONCE into shared memory by one thread, instead of once by each of its two
// cells; each column's z face is evaluated by the column's thread and carried in
// registers to the next plane as that cell's lower face. Each own cell then sums
// its faces in its face-graph incidence order (-z, -y, -x, +x, +y, +z, then the
// box sides), so the stage results are bitwise those of cartRates.
#ifndef RB200_TILE_Y
#define RB200_TILE_Y 4
#endif
#ifndef RB200_TILE_MINBLOCKS
#define RB200_TILE_MINBLOCKS 3
#endif
constexpr int kTileX = 32, kTileY = RB200_TILE_Y, kTileZ = 16;

template <int NS, bool SGS> struct TileLayout {
    static constexpr int NQ = NS + 4;
    // flux inputs: q, u, p, T, rho, c, [cp, h], gradient, eddy viscosity
    static constexpr int Q = 0, U = NQ, P = U + 3, T = P + 1, RHO = T + 1, C = RHO + 1, CP = C + 1,
                         H = CP + (SGS ? 1 : 0), G = H + (SGS ? NS : 0), NUT = G + 9, FIELDS = NUT + 1;
    static constexpr int PX = kTileX + 2, PY = kTileY + 2, SLOTS = PX * PY;
    static constexpr int FX = (kTileX + 1) * kTileY, FY = kTileX * (kTileY + 1);
    template <class R> static constexpr size_t bytes() {
        return sizeof(R) * (size_t(FIELDS) * SLOTS + size_t(FX + FY) * NQ);
    }
};

// One cell's flux inputs, rounded to R once (as asCell), with its gradient and
// eddy viscosity, into shared-memory slot `slot`.
template <int NS, class R, bool SGS>
__device__ __forceinline__ void stageTileCell(const CartView& v, const double* __restrict__ q,
                                              const ReactiveTransportState* __restrict__ st,
                                              const R* __restrict__ grad, const R* __restrict__ nut, size_t c,
                                              R* plane, int slot, bool viscous) {
    using Lay = TileLayout<NS, SGS>;
    constexpr int S = Lay::SLOTS;
    CellData d;
    loadCell<NS, SGS>(v, q, st, c, d, true);
    const CellT<R> t = asCell<NS, R, SGS>(d);
#pragma unroll
    for (int k = 0; k < Lay::NQ; ++k) plane[(Lay::Q + k) * S + slot] = t.q[k];
#pragma unroll
    for (int a = 0; a < 3; ++a) plane[(Lay::U + a) * S + slot] = t.u[a];
    plane[Lay::P * S + slot] = t.p;
    plane[Lay::T * S + slot] = t.T;
    plane[Lay::RHO * S + slot] = t.rho;
    plane[Lay::C * S + slot] = t.c;
    if constexpr (SGS) {
        plane[Lay::CP * S + slot] = t.cp;
#pragma unroll
        for (int k = 0; k < NS; ++k) plane[(Lay::H + k) * S + slot] = t.h[k];
    }
#pragma unroll
    for (int j = 0; j < 9; ++j) plane[(Lay::G + j) * S + slot] = viscous ? grad[size_t(j) * v.cells + c] : R(0);
    plane[Lay::NUT * S + slot] = v.wale ? nut[c] : R(0);
}

template <int NS, class R, bool SGS>
__device__ __forceinline__ void tileCell(const R* plane, int slot, CellT<R>& t, R* g, R& nu) {
    using Lay = TileLayout<NS, SGS>;
    constexpr int S = Lay::SLOTS;
#pragma unroll
    for (int k = 0; k < Lay::NQ; ++k) t.q[k] = plane[(Lay::Q + k) * S + slot];
#pragma unroll
    for (int a = 0; a < 3; ++a) t.u[a] = plane[(Lay::U + a) * S + slot];
    t.p = plane[Lay::P * S + slot];
    t.T = plane[Lay::T * S + slot];
    t.rho = plane[Lay::RHO * S + slot];
    t.c = plane[Lay::C * S + slot];
    t.cv = R(0);
    if constexpr (SGS) {
        t.cp = plane[Lay::CP * S + slot];
#pragma unroll
        for (int k = 0; k < NS; ++k) t.h[k] = plane[(Lay::H + k) * S + slot];
    }
#pragma unroll
    for (int j = 0; j < 9; ++j) g[j] = plane[(Lay::G + j) * S + slot];
    nu = plane[Lay::NUT * S + slot];
}

// The same inputs for a cell read straight from global memory (the column's
// next plane, and the plane below a chunk's first).
template <int NS, class R, bool SGS>
__device__ __forceinline__ void globalCell(const CartView& v, const double* __restrict__ q,
                                           const ReactiveTransportState* __restrict__ st, const R* __restrict__ grad,
                                           const R* __restrict__ nut, size_t c, bool viscous, CellT<R>& t, R* g,
                                           R& nu) {
    CellData d;
    loadCell<NS, SGS>(v, q, st, c, d, true);
    t = asCell<NS, R, SGS>(d);
#pragma unroll
    for (int j = 0; j < 9; ++j) g[j] = viscous ? grad[size_t(j) * v.cells + c] : R(0);
    nu = v.wale ? nut[c] : R(0);
}

template <int NS, class R, bool SGS = false>
__global__ void __launch_bounds__(kTileX * kTileY, RB200_TILE_MINBLOCKS) cartRatesTile(CartView v, const double* __restrict__ q,
                                                                const ReactiveTransportState* __restrict__ st,
                                                                const R* __restrict__ grad,
                                                                const R* __restrict__ nut, double* out,
                                                                size_t outStride, int mode, double dt,
                                                                unsigned* error) {
    using Lay = TileLayout<NS, SGS>;
    constexpr int NQ = Lay::NQ, S = Lay::SLOTS, PX = Lay::PX;
    constexpr bool fp64 = sizeof(R) == sizeof(double);
    extern __shared__ __align__(16) unsigned char tileMemory[];
    R* plane = reinterpret_cast<R*>(tileMemory);
    R* fx = plane + size_t(Lay::FIELDS) * S;   // x faces: [ly][lx], lx = 0..kTileX (face lx-1 | lx)
    R* fy = fx + size_t(Lay::FX) * NQ;         // y faces: [ly][lx], ly = 0..kTileY (face ly-1 | ly)
    const bool viscous = v.viscosity > 0 || v.wale;
    const int tid = threadIdx.x, tx = tid % kTileX, ty = tid / kTileX;
    const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY, z0 = blockIdx.z * kTileZ;
    const int z1 = min(z0 + kTileZ, v.nz);
    const int gx = x0 + tx, gy = y0 + ty;
    const bool inside = gx < v.nx && gy < v.ny;
    auto cellAt = [&](int x, int y, int z) { return size_t(x) + size_t(v.nx) * (size_t(y) + size_t(v.ny) * z); };
    auto own = [&](int x, int y, int z) {
        if (x < 0 || y < 0 || x >= v.nx || y >= v.ny || z < 0 || z >= v.nz) return false;
        const size_t c = cellAt(x, y, z);
        return c >= v.ownBegin && c < v.ownEnd;
    };
    bool bad = false, faceBad = false;
    R down[NQ];  // the column's lower z face (the face between this plane and the one below)
#pragma unroll
    for (int kk = 0; kk < NQ; ++kk) down[kk] = R(0);
    if (inside && z0 > 0 && z0 < z1 && (own(gx, gy, z0 - 1) || own(gx, gy, z0))) {
        CellT<R> lo, hi;
        R gl[9], gh[9], nl, nh;
        globalCell<NS, R, SGS>(v, q, st, grad, nut, cellAt(gx, gy, z0 - 1), viscous, lo, gl, nl);
        globalCell<NS, R, SGS>(v, q, st, grad, nut, cellAt(gx, gy, z0), viscous, hi, gh, nh);
        faceFluxCart<NS, R, SGS>(v, 2, 1.0, v.area[2], v.dist[2], .5, 0, true, lo, hi, gl, gh, nl, nh, down, bad,
                                 faceBad);
    }
    for (int z = z0; z < z1; ++z) {
        __syncthreads();  // the previous plane's readers are done
        // stage the plane: the tile's own slots, then the halo ring
        if (inside)
            stageTileCell<NS, R, SGS>(v, q, st, grad, nut, cellAt(gx, gy, z), plane, (ty + 1) * PX + tx + 1,
                                      viscous);
        constexpr int ring = 2 * kTileX + 2 * kTileY;
        for (int h = tid; h < ring; h += kTileX * kTileY) {
            int lx, ly;
            if (h < kTileX) { lx = h; ly = -1; }
            else if (h < 2 * kTileX) { lx = h - kTileX; ly = kTileY; }
            else if (h < 2 * kTileX + kTileY) { lx = -1; ly = h - 2 * kTileX; }
            else { lx = kTileX; ly = h - 2 * kTileX - kTileY; }
            const int x = x0 + lx, y = y0 + ly;
            if (x >= 0 && y >= 0 && x < v.nx && y < v.ny)
                stageTileCell<NS, R, SGS>(v, q, st, grad, nut, cellAt(x, y, z), plane, (ly + 1) * PX + lx + 1,
                                          viscous);
        }
        __syncthreads();
        // every x and y face of the tile's own cells, once
        for (int f = tid; f < Lay::FX + Lay::FY; f += kTileX * kTileY) {
            const bool xFace = f < Lay::FX;
            const int idx = xFace ? f : f - Lay::FX;
            const int lx = xFace ? idx % (kTileX + 1) : idx % kTileX;
            const int ly = xFace ? idx / (kTileX + 1) : idx / kTileX;
            // lower cell (ax, ay) and upper cell (bx, by) in tile coordinates
            const int ax = xFace ? lx - 1 : lx, ay = xFace ? ly : ly - 1;
            const int bx = lx, by = ly;
            const bool lowerOwn = ax >= 0 && ay >= 0 && own(x0 + ax, y0 + ay, z);
            const bool upperOwn = bx < kTileX && by < kTileY && own(x0 + bx, y0 + by, z);
            const bool exists = x0 + ax >= 0 && y0 + ay >= 0 && x0 + bx < v.nx && y0 + by < v.ny;
            R* F = (xFace ? fx : fy) + size_t(idx) * NQ;
            if (!exists || !(lowerOwn || upperOwn)) continue;
            CellT<R> L, Rt;
            R gL[9], gR[9], nL, nR;
            tileCell<NS, R, SGS>(plane, (ay + 1) * PX + ax + 1, L, gL, nL);
            tileCell<NS, R, SGS>(plane, (by + 1) * PX + bx + 1, Rt, gR, nR);
            R flux[NQ];
            const int axis = xFace ? 0 : 1;
            faceFluxCart<NS, R, SGS>(v, axis, 1.0, v.area[axis], v.dist[axis], .5, 0, true, L, Rt, gL, gR, nL, nR,
                                     flux, bad, faceBad);
#pragma unroll
            for (int kk = 0; kk < NQ; ++kk) F[kk] = flux[kk];
        }
        // the column's upper z face
        const int slot = (ty + 1) * PX + tx + 1;
        R up[NQ];
#pragma unroll
        for (int kk = 0; kk < NQ; ++kk) up[kk] = R(0);
        const bool hasUp = z + 1 < v.nz;
        if (inside && hasUp && (own(gx, gy, z) || own(gx, gy, z + 1))) {
            CellT<R> lo, hi;
            R gl[9], gh[9], nl, nh;
            tileCell<NS, R, SGS>(plane, slot, lo, gl, nl);
            globalCell<NS, R, SGS>(v, q, st, grad, nut, cellAt(gx, gy, z + 1), viscous, hi, gh, nh);
            faceFluxCart<NS, R, SGS>(v, 2, 1.0, v.area[2], v.dist[2], .5, 0, true, lo, hi, gl, gh, nl, nh, up, bad,
                                     faceBad);
        }
        __syncthreads();
        if (inside && own(gx, gy, z)) {
            const size_t c = cellAt(gx, gy, z);
            const double iv = v.invV[c];
            R rate[NQ], comp[NQ];
#pragma unroll
            for (int kk = 0; kk < NQ; ++kk) rate[kk] = comp[kk] = R(0);
            auto add = [&](const R* F, double sign) {
#pragma unroll
                for (int kk = 0; kk < NQ; ++kk) {
                    if constexpr (fp64) rate[kk] += sign * F[kk] * iv;
                    else twoSum(rate[kk], comp[kk], sign > 0 ? F[kk] : -F[kk]);
                }
            };
            // internal faces in incidence order: -z, -y, -x, +x, +y, +z
            if (z > 0) add(down, 1);
            if (gy > 0) add(fy + size_t(ty * kTileX + tx) * NQ, 1);
            if (gx > 0) add(fx + size_t(ty * (kTileX + 1) + tx) * NQ, 1);
            if (gx + 1 < v.nx) add(fx + size_t(ty * (kTileX + 1) + tx + 1) * NQ, -1);
            if (gy + 1 < v.ny) add(fy + size_t((ty + 1) * kTileX + tx) * NQ, -1);
            if (hasUp) add(up, -1);
            // box sides (-x, +x, -y, +y, -z, +z)
            CellT<R> me;
            R gMe[9], nuMe;
            tileCell<NS, R, SGS>(plane, slot, me, gMe, nuMe);
            CellData C;
            const bool boundary = gx == 0 || gy == 0 || z == 0 || gx + 1 == v.nx || gy + 1 == v.ny || z + 1 == v.nz;
            if (boundary) loadCell<NS, SGS>(v, q, st, c, C, true);
#pragma unroll
            for (int side = 0; side < 6; ++side) {
                if (hasNeighbour(v, side, gx, gy, z)) continue;
                const int axis = side >> 1;
                const ReactiveTransportFace& f = sideFace(v, side, gx, gy, z);
                CellData Rd;
                boundaryRight<NS, SGS>(v, q, st, f, axis, C, Rd, true);
                R flux[NQ];
                faceFluxCart<NS, R, SGS>(v, axis, (side & 1) ? 1.0 : -1.0, f.area, f.distance, f.ownerWeight, f.kind,
                                         false, me, asCell<NS, R, SGS>(Rd), gMe, gMe, nuMe, nuMe, flux, bad, faceBad);
                add(flux, -1);
            }
            // the cell's own conserved variables in FP64 for the update
            double qc[NQ];
#pragma unroll
            for (int kk = 0; kk < NQ; ++kk) qc[kk] = q[size_t(kk) * v.all + c];
#pragma unroll
            for (int kk = 0; kk < NQ; ++kk) {
                const double r = fp64 ? double(rate[kk]) : (double(rate[kk]) + double(comp[kk])) * iv;
                const size_t o = size_t(kk) * outStride + c;
                if (mode == 0) out[o] = r;
                else if (mode == 1) out[o] = qc[kk] + dt * r;
                else out[o] = .5 * out[o] + .5 * (qc[kk] + dt * r);
            }
        }
#pragma unroll
        for (int kk = 0; kk < NQ; ++kk) down[kk] = up[kk];
    }
    if (bad) atomicOr(error, 1u);
    if (faceBad) atomicOr(error, 2u);
}

// Wave/diffusion speed of one face (faceSpeeds of the face graph); -1 when invalid.
template <bool SGS>
__device__ __forceinline__ double faceSpeedCart(const CartView& v, int axis, double sgn, double dist, double w,
                                                int kind, const CellData& L, const CellData& R, double nutL,
                                                double nutR) {
    const double unL = L.u[axis] * sgn, unR = R.u[axis] * sgn;
    const double aL = v.waveFactor * L.c, aR = v.waveFactor * R.c;
    const double left = dmin(0, dmin(unL - aL, unR - aR)), right = dmax(0, dmax(unL + aL, unR + aR));
    const double invWave = 1 / (right - left);
    const double rhoNut = v.wale ? w * L.rho * nutL + (1 - w) * R.rho * nutR : 0;
    const double mu = v.viscosity + rhoNut;
    const double D = 0.0 + dmax(dmax(4 * mu / (3 * L.rho), 4 * mu / (3 * R.rho)),
                                dmax(v.conductivity / (L.rho * L.cv), v.conductivity / (R.rho * R.cv)));
    double scalar = 0;
    if constexpr (SGS) {
        if (kind != 1) {
            if (v.pr > 0) {
                const double k = rhoNut * (w * L.cp + (1 - w) * R.cp) / v.pr;
                scalar = dmax(scalar, dmax(k / (L.rho * L.cv), k / (R.rho * R.cv)));
            }
            if (v.sc > 0) scalar = dmax(scalar, dmax(rhoNut / L.rho, rhoNut / R.rho) / v.sc);
        }
    }
    double speed = dmax(fabs(unL) + aL, fabs(unR) + aR) + 2 * (D + scalar) / dist;
    if (!isfinite(unL) || !isfinite(unR) || !isfinite(speed) || !isfinite(invWave) || right <= left) speed = -1;
    return speed;
}

// CFL step of every cell from its six face speeds (cellSteps), folded to one
// partial minimum per block with invalid steps absorbing as -1 (minimumReduce).
template <int NS, class R, bool SGS = false>
__global__ void __launch_bounds__(256) cartSteps(CartView v, const ReactiveTransportState* __restrict__ st,
                                                 const R* __restrict__ nut, double cfl, double maximumStep,
                                                 double* partial) {
    __shared__ double warpValues[32];
    // every cell's step is at most maximumStep, so starting there changes no
    // minimum and leaves a block without own cells a valid (positive) partial
    double m = maximumStep;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        if (c < v.ownBegin || c >= v.ownEnd) continue;
        int i, j, k;
        cellCoords(v, c, i, j, k);
        CellData C;
        loadCell<NS, SGS>(v, nullptr, st, c, C, false);
        const double nutC = v.wale ? double(nut[c]) : 0;
        double denominator = 0;
        bool bad = false, faceBad = false;
#pragma unroll
        for (int n = 0; n < 12; ++n) {
            const int s = sideOf(n);
            const bool interior = hasNeighbour(v, s, i, j, k);
            if (interior != (n < 6)) continue;
            const int axis = s >> 1;
            double speed, area;
            if (interior) {
                const size_t nb = neighbourOf(v, s, c);
                CellData N;
                loadCell<NS, SGS>(v, nullptr, st, nb, N, false);
                const double nutN = v.wale ? double(nut[nb]) : 0;
                speed = (s & 1) ? faceSpeedCart<SGS>(v, axis, 1.0, v.dist[axis], .5, 0, C, N, nutC, nutN)
                                : faceSpeedCart<SGS>(v, axis, 1.0, v.dist[axis], .5, 0, N, C, nutN, nutC);
                area = v.area[axis];
            } else {
                const ReactiveTransportFace& f = sideFace(v, s, i, j, k);
                CellData Rt;
                boundaryRight<NS, SGS>(v, nullptr, st, f, axis, C, Rt, false);
                speed = faceSpeedCart<SGS>(v, axis, (s & 1) ? 1.0 : -1.0, f.distance, f.ownerWeight, f.kind, C, Rt,
                                           nutC, nutC);
                area = f.area;
            }
            if (!isfinite(speed) || speed < 0) { bad = true; break; }
            denominator += area * speed;
        }
        double step = denominator > 0 ? dmin(maximumStep, cfl / (v.invV[c] * denominator)) : maximumStep;
        if (bad || !isfinite(denominator) || denominator < 0) step = -1;
        m = fmin(m, isfinite(step) && step > 0 ? step : -1.0);
    }
    m = warpMin(m);
    if ((threadIdx.x & 31) == 0) warpValues[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? warpValues[threadIdx.x] : HUGE_VAL;
        m = warpMin(m);
        if (threadIdx.x == 0) partial[blockIdx.x] = m;
    }
}

// Boundary ledger: the sum over boundary faces of each variable's face flux.
// Pass 1 (this kernel) writes one partial per (block, variable) in a fixed
// partition, pass 2 (foldPartials) adds them in block order: deterministic.
template <int NS, class R, bool SGS = false>
__global__ void __launch_bounds__(256) cartLedger(CartView v, const double* __restrict__ q,
                                                  const ReactiveTransportState* __restrict__ st,
                                                  const R* __restrict__ grad, const R* __restrict__ nut,
                                                  double* partial) {
    __shared__ double warpValues[kCartMaxNs + 4][32];
    double sum[NS + 4];
#pragma unroll
    for (int kk = 0; kk < NS + 4; ++kk) sum[kk] = 0;
    const bool viscous = v.viscosity > 0 || v.wale;
    bool bad = false, faceBad = false;
    for (size_t b = blockIdx.x * size_t(blockDim.x) + threadIdx.x; b < v.nBoundary;
         b += size_t(blockDim.x) * gridDim.x) {
        const ReactiveTransportFace f = v.face[v.boundaryBase + b];
        const size_t c = size_t(f.owner);
        if (c < v.ownBegin || c >= v.ownEnd) continue;
        const int axis = f.normal[0] != 0 ? 0 : (f.normal[1] != 0 ? 1 : 2);
        const double sgn = f.normal[axis] > 0 ? 1.0 : -1.0;
        CellData C, Rt;
        loadCell<NS, SGS>(v, q, st, c, C, true);
        boundaryRight<NS, SGS>(v, q, st, f, axis, C, Rt, true);
        R g[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (viscous) {
#pragma unroll
            for (int jj = 0; jj < 9; ++jj) g[jj] = grad[size_t(jj) * v.cells + c];
        }
        const R nutC = v.wale ? nut[c] : R(0);
        R F[NS + 4];
        faceFluxCart<NS, R, SGS>(v, axis, sgn, f.area, f.distance, f.ownerWeight, f.kind, false,
                                 asCell<NS, R, SGS>(C), asCell<NS, R, SGS>(Rt), g, g, nutC, nutC, F, bad, faceBad);
#pragma unroll
        for (int kk = 0; kk < NS + 4; ++kk) sum[kk] += double(F[kk]);
    }
#pragma unroll
    for (int kk = 0; kk < NS + 4; ++kk) {
        const double s = warpSum(sum[kk]);
        if ((threadIdx.x & 31) == 0) warpValues[kk][threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int kk = 0; kk < NS + 4; ++kk) {
            double s = threadIdx.x < (blockDim.x >> 5) ? warpValues[kk][threadIdx.x] : 0.0;
            s = warpSum(s);
            if (threadIdx.x == 0) partial[size_t(blockIdx.x) * (NS + 4) + kk] = s;
        }
    }
}

// Vector-Jacobian product of the rate operator L of the structured box. Given
// adjoint weights w (SoA nv x cells, the adjoint of each cell's rate), a cell c
// visits its six faces and evaluates each face flux in forward dual numbers
// seeded on c's own inputs, then contracts the flux derivatives with the face's
// adjoint weight sum_side sign w / V. Gather form, no atomics; the HLL
// wave-speed switches and the HLLC star-side and supersonic switches are
// differentiated piecewise, on the branch the forward takes.
//   MODE 0: seeds on c's conserved variables (and through u = m / rho on its
//           velocity), p, sound, T and the state density; writes qBar (the
//           direct part) and stateBar {p, T, rho, 0, sound, 0, 0}.
//   MODE 1: seeds on c's velocity gradient (9) and WALE eddy viscosity; writes
//           gBar (SoA 9 x cells) and nutBar. Only for the viscous operator.
// A boundary face's ghost follows its owner's duals (slip: mirrored), a fixed
// state is constant; a boundary face uses the owner's gradient and eddy
// viscosity on both sides, as the forward does.
template <int NS, int MODE>
__global__ void __launch_bounds__(128) cartRateVjp(CartView v, const double* __restrict__ q,
                                                   const ReactiveTransportState* __restrict__ st,
                                                   const double* __restrict__ grad, const double* __restrict__ nut,
                                                   const double* __restrict__ w, double* __restrict__ qBar,
                                                   ReactiveTransportState* __restrict__ stateBar,
                                                   double* __restrict__ gBar, double* __restrict__ nutBar) {
    constexpr int N = MODE == 0 ? NS + 8 : 10;
    using D = Dual<N>;
    const bool viscous = v.viscosity > 0 || v.wale;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        int i, j, k;
        cellCoords(v, c, i, j, k);
        CellData C;
        loadCell<NS>(v, q, st, c, C, true);
        CellT<D> Cd = asCell<NS, D>(C);
        D gC[9], nutC(0.0);
#pragma unroll
        for (int t = 0; t < 9; ++t) gC[t] = D(viscous ? grad[size_t(t) * v.cells + c] : 0.0);
        if (v.wale) nutC = D(nut[c]);
        if (MODE == 0) {
            D rho(0.0);
#pragma unroll
            for (int kk = 0; kk < NS + 4; ++kk) Cd.q[kk] = D::seed(C.q[kk], kk);
#pragma unroll
            for (int kk = 0; kk < NS; ++kk) rho += Cd.q[kk];
#pragma unroll
            for (int a = 0; a < 3; ++a) Cd.u[a] = Cd.q[NS + a] / rho;
            Cd.p = D::seed(C.p, NS + 4);
            Cd.c = D::seed(C.c, NS + 5);
            Cd.T = D::seed(C.T, NS + 6);
            Cd.rho = D::seed(C.rho, NS + 7);
        } else {
#pragma unroll
            for (int t = 0; t < 9; ++t) gC[t] = D::seed(grad[size_t(t) * v.cells + c], t);
            if (v.wale) nutC = D::seed(nut[c], 9);
        }
        const double ivc = v.invV[c];
        double acc[N];
#pragma unroll
        for (int t = 0; t < N; ++t) acc[t] = 0;
        bool bad = false, faceBad = false;
#pragma unroll 1
        for (int n = 0; n < 12; ++n) {
            const int s = sideOf(n);
            const bool interior = hasNeighbour(v, s, i, j, k);
            if (interior != (n < 6)) continue;
            const int axis = s >> 1;
            D F[NS + 4];
            double W[NS + 4];
            if (interior) {
                const size_t nb = neighbourOf(v, s, c);
                CellData Nc;
                loadCell<NS>(v, q, st, nb, Nc, true);
                const CellT<D> Nd = asCell<NS, D>(Nc);
                D gN[9], nutN(0.0);
#pragma unroll
                for (int t = 0; t < 9; ++t) gN[t] = D(viscous ? grad[size_t(t) * v.cells + nb] : 0.0);
                if (v.wale) nutN = D(nut[nb]);
                const double ivn = v.invV[nb];
                if (s & 1) {  // c owns the face
                    faceFluxCart<NS, D>(v, axis, 1.0, v.area[axis], v.dist[axis], .5, 0, true, Cd, Nd, gC, gN, nutC,
                                        nutN, F, bad, faceBad);
#pragma unroll
                    for (int kk = 0; kk < NS + 4; ++kk)
                        W[kk] = w[size_t(kk) * v.cells + nb] * ivn - w[size_t(kk) * v.cells + c] * ivc;
                } else {
                    faceFluxCart<NS, D>(v, axis, 1.0, v.area[axis], v.dist[axis], .5, 0, true, Nd, Cd, gN, gC, nutN,
                                        nutC, F, bad, faceBad);
#pragma unroll
                    for (int kk = 0; kk < NS + 4; ++kk)
                        W[kk] = w[size_t(kk) * v.cells + c] * ivc - w[size_t(kk) * v.cells + nb] * ivn;
                }
            } else {
                const ReactiveTransportFace& f = sideFace(v, s, i, j, k);
                CellT<D> Rt;
                if (f.kind == 3) {
                    CellData Fx;
                    loadCell<NS>(v, q, st, v.cells + size_t(f.fixed), Fx, true);
                    Rt = asCell<NS, D>(Fx);
                } else {
                    Rt = Cd;
                    if (f.kind == 1) {
                        Rt.u[axis] = Cd.u[axis] - D(2.0) * Cd.u[axis];
                        Rt.q[NS + axis] = Cd.q[NS + axis] - D(2.0) * Cd.q[NS + axis];
                    }
                }
                faceFluxCart<NS, D>(v, axis, (s & 1) ? 1.0 : -1.0, f.area, f.distance, f.ownerWeight, f.kind, false,
                                    Cd, Rt, gC, gC, nutC, nutC, F, bad, faceBad);
#pragma unroll
                for (int kk = 0; kk < NS + 4; ++kk) W[kk] = -w[size_t(kk) * v.cells + c] * ivc;
            }
#pragma unroll
            for (int kk = 0; kk < NS + 4; ++kk)
#pragma unroll
                for (int t = 0; t < N; ++t) acc[t] += W[kk] * F[kk].d[t];
        }
        if (MODE == 0) {
#pragma unroll
            for (int kk = 0; kk < NS + 4; ++kk) qBar[size_t(kk) * v.cells + c] = acc[kk];
            stateBar[c] = ReactiveTransportState{acc[NS + 4], acc[NS + 6], acc[NS + 7], 0.0, acc[NS + 5], 0.0, 0.0};
        } else {
#pragma unroll
            for (int t = 0; t < 9; ++t) gBar[size_t(t) * v.cells + c] = acc[t];
            if (nutBar) nutBar[c] = acc[9];
        }
    }
}

// Reverse-mode derivative of the inviscid HLL face flux, written out by hand.
// With Wa the face's adjoint weights times the area and J = sum_k Wa_k F_k / A:
// J = advL SL + advR SR + pM Wm + pE We (SL = Wa.qL, SR = Wa.qR, Wm the
// axis-momentum weight times the normal sign, We the energy weight), whose
// partials with respect to the normal velocities, sound speeds (through the
// wave speeds, the active branch of each min/max as the forward selects it),
// pressures and conserved variables of both sides are returned.
struct HllBar {
    double qL, qR;  // multipliers of Wa_k for d J / d qL_k, d qR_k (advL, advR)
    double unL, unR, cL, cR, pL, pR;
};
__device__ __forceinline__ HllBar hllReverse(double wf, double unL, double unR, double cL, double cR, double pL,
                                             double pR, double SL, double SR, double Wm, double We) {
    const double aL = wf * cL, aR = wf * cR;
    const double lo1 = unL - aL, lo2 = unR - aR, hi1 = unL + aL, hi2 = unR + aR;
    const bool loFirst = lo1 < lo2, hiFirst = hi1 > hi2;
    const double loIn = loFirst ? lo1 : lo2, hiIn = hiFirst ? hi1 : hi2;
    const bool leftActive = !(0.0 < loIn), rightActive = !(0.0 > hiIn);
    const double left = leftActive ? loIn : 0.0, right = rightActive ? hiIn : 0.0;
    const double inv = 1 / (right - left);
    const double advL = right * (unL - left) * inv, advR = left * (right - unR) * inv;
    const double pM = (right * pL - left * pR) * inv, pE = (right * pL * unL - left * pR * unR) * inv;
    const double J = advL * SL + advR * SR + pM * Wm + pE * We;
    HllBar b;
    b.qL = advL;
    b.qR = advR;
    b.unL = (right * SL + right * pL * We) * inv;
    b.unR = (-left * SR - left * pR * We) * inv;
    b.pL = (right * Wm + right * unL * We) * inv;
    b.pR = (-left * Wm - left * unR * We) * inv;
    const double dRight = ((unL - left) * SL + left * SR + pL * Wm + pL * unL * We - J) * inv;
    const double dLeft = (-right * SL + (right - unR) * SR - pR * Wm - pR * unR * We + J) * inv;
    double aLb = 0, aRb = 0;
    if (leftActive) {
        if (loFirst) { b.unL += dLeft; aLb -= dLeft; } else { b.unR += dLeft; aRb -= dLeft; }
    }
    if (rightActive) {
        if (hiFirst) { b.unL += dRight; aLb += dRight; } else { b.unR += dRight; aRb += dRight; }
    }
    b.cL = wf * aLb;
    b.cR = wf * aRb;
    return b;
}

// (dL/dq)^T w and (dL/dstate)^T w of the HLL operator of the structured box at
// fixed cell gradients and eddy viscosities (the part cartRateVjp<NS, 0> forms
// in dual numbers), gather form, in registers: the HLL flux by hllReverse; the
// viscous traction through the velocities (the face-gradient correction's
// target (u_R - u_L) / d and the work's u_bar) and through rho in the WALE
// viscosity; conduction through T. With dJ/dG' = mu (a n^T + n a^T - 2/3 (a.n) I)
// (a = -(W_m + W_E u_bar) A, projected on n at a slip wall): dJ/dt = dJ/dG' n,
// dJ/du_bar = -W_E A tau, dJ/dmu = a . tau / mu. The gradients' and eddy
// viscosities' own adjoints are cartViscousGradVjp's.
template <int NS>
__global__ void __launch_bounds__(128) cartRateVjpInviscid(CartView v, const double* __restrict__ q,
                                                           const ReactiveTransportState* __restrict__ st,
                                                           const double* __restrict__ grad,
                                                           const double* __restrict__ nut,
                                                           const double* __restrict__ w, double* __restrict__ qBar,
                                                           ReactiveTransportState* __restrict__ stateBar) {
    const bool viscous = v.viscosity > 0 || v.wale;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        int i, j, k;
        cellCoords(v, c, i, j, k);
        CellData C;
        loadCell<NS>(v, q, st, c, C, true);
        const double ivc = v.invV[c];
        double dq[NS + 4], du[3] = {0, 0, 0}, dp = 0, dc = 0, dT = 0, dRhoState = 0;
#pragma unroll
        for (int kk = 0; kk < NS + 4; ++kk) dq[kk] = 0;
        double gC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (viscous) {
#pragma unroll
            for (int t = 0; t < 9; ++t) gC[t] = grad[size_t(t) * v.cells + c];
        }
        const double nutC = v.wale ? nut[c] : 0.0;
#pragma unroll 1
        for (int n = 0; n < 12; ++n) {
            const int s = sideOf(n);
            const bool interior = hasNeighbour(v, s, i, j, k);
            if (interior != (n < 6)) continue;
            const int axis = s >> 1;
            CellData O;  // the other side
            double Wa[NS + 4], sgn, area, wf, dist, gO[9], nutO = nutC;
            int kind = 0;
            bool cIsLeft = true;
            if (interior) {
                const size_t nb = neighbourOf(v, s, c);
                loadCell<NS>(v, q, st, nb, O, true);
                const double ivn = v.invV[nb];
                cIsLeft = s & 1;
                sgn = 1;
                area = v.area[axis];
                wf = .5;
                dist = v.dist[axis];
                if (viscous) {
#pragma unroll
                    for (int t = 0; t < 9; ++t) gO[t] = grad[size_t(t) * v.cells + nb];
                }
                if (v.wale) nutO = nut[nb];
#pragma unroll
                for (int kk = 0; kk < NS + 4; ++kk)
                    Wa[kk] = area * (cIsLeft ? w[size_t(kk) * v.cells + nb] * ivn - w[size_t(kk) * v.cells + c] * ivc
                                             : w[size_t(kk) * v.cells + c] * ivc - w[size_t(kk) * v.cells + nb] * ivn);
            } else {
                const ReactiveTransportFace& f = sideFace(v, s, i, j, k);
                kind = f.kind;
                boundaryRight<NS>(v, q, st, f, axis, C, O, true);
                sgn = (s & 1) ? 1.0 : -1.0;
                area = f.area;
                wf = f.ownerWeight;
                dist = f.distance;
#pragma unroll
                for (int t = 0; t < 9; ++t) gO[t] = gC[t];
#pragma unroll
                for (int kk = 0; kk < NS + 4; ++kk) Wa[kk] = -area * w[size_t(kk) * v.cells + c] * ivc;
            }
            const CellData& L = cIsLeft ? C : O;
            const CellData& R = cIsLeft ? O : C;
            double SL = 0, SR = 0;
#pragma unroll
            for (int kk = 0; kk < NS + 4; ++kk) { SL += Wa[kk] * L.q[kk]; SR += Wa[kk] * R.q[kk]; }
            const HllBar b = hllReverse(v.waveFactor, L.u[axis] * sgn, R.u[axis] * sgn, L.c, R.c, L.p, R.p, SL, SR,
                                        Wa[NS + axis] * sgn, Wa[NS + 3]);
            // c's own side
            const double qMul = cIsLeft ? b.qL : b.qR;
#pragma unroll
            for (int kk = 0; kk < NS + 4; ++kk) dq[kk] += Wa[kk] * qMul;
            du[axis] += (cIsLeft ? b.unL : b.unR) * sgn;
            dp += cIsLeft ? b.pL : b.pR;
            dc += cIsLeft ? b.cL : b.cR;
            // a boundary ghost made from c (extrapolate: itself; slip: axis momentum and velocity mirrored)
            if (!interior && (kind == 1 || kind == 2)) {
                const double mirror = kind == 1 ? -1.0 : 1.0;
#pragma unroll
                for (int kk = 0; kk < NS + 4; ++kk) dq[kk] += Wa[kk] * b.qR * (kk == NS + axis ? mirror : 1.0);
                du[axis] += b.unR * sgn * mirror;
                dp += b.pR;
                dc += b.cR;
            }
            if (!viscous && !(v.conductivity > 0 && kind != 1)) continue;
            // viscous traction and conduction at fixed gradients and eddy viscosities
            double duL[3] = {0, 0, 0}, duR[3] = {0, 0, 0}, dTL = 0, dTR = 0, dRL = 0, dRR = 0;
            double nv[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) nv[d] = d == axis ? sgn : 0.0;
            if (viscous) {
                const double* gL = cIsLeft ? gC : gO;
                const double* gR = cIsLeft ? gO : gC;
                const double nutL = cIsLeft ? nutC : nutO, nutR = cIsLeft ? nutO : nutC;
                const double kd = (kind == 1 ? 2 : 1) * dist;
                double g[9];
#pragma unroll
                for (int t = 0; t < 9; ++t) g[t] = interior ? wf * gL[t] + (1 - wf) * gR[t] : gL[t];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    double normal = 0;
#pragma unroll
                    for (int d = 0; d < 3; ++d) normal += g[a * 3 + d] * nv[d];
                    const double target = (R.u[a] - L.u[a]) / kd;
#pragma unroll
                    for (int d = 0; d < 3; ++d) g[a * 3 + d] += nv[d] * (target - normal);
                }
                const double div = g[0] + g[4] + g[8];
                const double mu = v.viscosity + (v.wale ? wf * L.rho * nutL + (1 - wf) * R.rho * nutR : 0.0);
                double tau[3], tn = 0, av[3], an = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    double t = -2.0 / 3.0 * div * nv[a];
#pragma unroll
                    for (int d = 0; d < 3; ++d) t += (g[a * 3 + d] + g[d * 3 + a]) * nv[d];
                    tau[a] = mu * t;
                    tn += tau[a] * nv[a];
                    av[a] = -(Wa[NS + a] + Wa[NS + 3] * (wf * L.u[a] + (1 - wf) * R.u[a]));
                    an += av[a] * nv[a];
                }
                if (kind == 1) {
#pragma unroll
                    for (int a = 0; a < 3; ++a) { tau[a] = tn * nv[a]; av[a] = an * nv[a]; }
                }
                an = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a) an += av[a] * nv[a];
                double jmu = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    // dJ/dt_a = (dJ/dG' n)_a; dJ/du_bar_a = -W_E A tau_a
                    double rn = 0;
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        rn += mu * (av[a] * nv[d] + nv[a] * av[d] - (a == d ? 2.0 / 3.0 * an : 0.0)) * nv[d];
                    const double dbar = -Wa[NS + 3] * tau[a];
                    duL[a] = wf * dbar - rn / kd;
                    duR[a] = (1 - wf) * dbar + rn / kd;
                    double t = -2.0 / 3.0 * div * nv[a];
#pragma unroll
                    for (int d = 0; d < 3; ++d) t += (g[a * 3 + d] + g[d * 3 + a]) * nv[d];
                    jmu += av[a] * t;
                }
                if (v.wale) {
                    dRL = jmu * wf * nutL;
                    dRR = jmu * (1 - wf) * nutR;
                }
            }
            if (v.conductivity > 0 && kind != 1) {
                dTL = Wa[NS + 3] * v.conductivity / dist;
                dTR = -dTL;
            }
            if (interior) {
#pragma unroll
                for (int a = 0; a < 3; ++a) du[a] += cIsLeft ? duL[a] : duR[a];
                dT += cIsLeft ? dTL : dTR;
                dRhoState += cIsLeft ? dRL : dRR;
            } else {
                // the owner, and the ghost made from it (extrapolate: itself; slip: mirrored velocity)
#pragma unroll
                for (int a = 0; a < 3; ++a) du[a] += duL[a];
                dT += dTL;
                dRhoState += dRL;
                if (kind == 1 || kind == 2) {
                    double rn = 0;
#pragma unroll
                    for (int a = 0; a < 3; ++a) rn += duR[a] * nv[a];
#pragma unroll
                    for (int a = 0; a < 3; ++a) du[a] += kind == 1 ? duR[a] - 2 * rn * nv[a] : duR[a];
                    dT += dTR;
                    dRhoState += dRR;
                }
            }
        }
        // u = m / rho with rho the sum of the species masses
        double rho = 0;
#pragma unroll
        for (int kk = 0; kk < NS; ++kk) rho += C.q[kk];
        double dRho = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            dq[NS + a] += du[a] / rho;
            dRho -= du[a] * C.u[a] / rho;
        }
#pragma unroll
        for (int kk = 0; kk < NS; ++kk) dq[kk] += dRho;
#pragma unroll
        for (int kk = 0; kk < NS + 4; ++kk) qBar[size_t(kk) * v.cells + c] = dq[kk];
        stateBar[c] = ReactiveTransportState{dp, dT, dRhoState, 0.0, dc, 0.0, 0.0};
    }
}

// Closed-form adjoint of the viscous/WALE traction with respect to the cells'
// velocity gradients and eddy viscosities (the part cartRateVjp<NS, 1> forms in
// dual numbers). The traction is bilinear in (mu, face gradient): with the
// corrected face gradient G' = G (I - n n^T) + t n^T, tau = mu (G' n + G'^T n -
// 2/3 tr(G') n) (projected on n at a slip wall), and J = a . tau for
// a = -A (W_m + W_E u_bar) (a -> (a.n) n at a slip wall), so
// dJ/dG' = mu (a n^T + n a^T - 2/3 (a.n) I), dJ/dG = dJ/dG' (I - n n^T) and
// dJ/dmu = J / mu; G = w G_L + (1 - w) G_R (the owner's on a boundary face) and
// mu = mu_0 + w rho_L nu_L + (1 - w) rho_R nu_R. Gather form per cell over its
// faces in the forward's order.
template <int NS>
__global__ void __launch_bounds__(128) cartViscousGradVjp(CartView v, const double* __restrict__ q,
                                                          const ReactiveTransportState* __restrict__ st,
                                                          const double* __restrict__ grad,
                                                          const double* __restrict__ nut,
                                                          const double* __restrict__ w, double* __restrict__ gBar,
                                                          double* __restrict__ nutBar) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        int i, j, k;
        cellCoords(v, c, i, j, k);
        CellData C;
        loadCell<NS>(v, q, st, c, C, false);
        double gC[9];
#pragma unroll
        for (int t = 0; t < 9; ++t) gC[t] = grad[size_t(t) * v.cells + c];
        const double nutC = v.wale ? nut[c] : 0.0;
        const double ivc = v.invV[c];
        double gb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, nb = 0;
#pragma unroll 1
        for (int n = 0; n < 12; ++n) {
            const int s = sideOf(n);
            const bool interior = hasNeighbour(v, s, i, j, k);
            if (interior != (n < 6)) continue;
            const int axis = s >> 1;
            CellData O;
            double gO[9], nutO, W[4], sgn, wf, dist, area, weightC, dmu;
            int kind = 0;
            bool cLeft = true;
            if (interior) {
                const size_t nbr = neighbourOf(v, s, c);
                loadCell<NS>(v, q, st, nbr, O, false);
#pragma unroll
                for (int t = 0; t < 9; ++t) gO[t] = grad[size_t(t) * v.cells + nbr];
                nutO = v.wale ? nut[nbr] : 0.0;
                cLeft = s & 1;
                sgn = 1;
                wf = .5;
                dist = v.dist[axis];
                area = v.area[axis];
                const double ivn = v.invV[nbr];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const size_t kk = size_t(NS + t);
                    W[t] = cLeft ? w[kk * v.cells + nbr] * ivn - w[kk * v.cells + c] * ivc
                                 : w[kk * v.cells + c] * ivc - w[kk * v.cells + nbr] * ivn;
                }
                weightC = cLeft ? wf : 1 - wf;
            } else {
                const ReactiveTransportFace& f = sideFace(v, s, i, j, k);
                boundaryRight<NS>(v, q, st, f, axis, C, O, false);
#pragma unroll
                for (int t = 0; t < 9; ++t) gO[t] = gC[t];
                nutO = nutC;
                kind = f.kind;
                sgn = (s & 1) ? 1.0 : -1.0;
                wf = f.ownerWeight;
                dist = f.distance;
                area = f.area;
#pragma unroll
                for (int t = 0; t < 4; ++t) W[t] = -w[size_t(NS + t) * v.cells + c] * ivc;
                weightC = 1;
            }
            const CellData& L = cLeft ? C : O;
            const CellData& R = cLeft ? O : C;
            const double* gL = cLeft ? gC : gO;
            const double* gR = cLeft ? gO : gC;
            const double nutL = cLeft ? nutC : nutO, nutR = cLeft ? nutO : nutC;
            dmu = interior ? (cLeft ? wf * L.rho : (1 - wf) * R.rho) : wf * L.rho + (1 - wf) * R.rho;
            double nv[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) nv[d] = d == axis ? sgn : 0.0;
            // the forward's corrected face gradient and viscosity
            double g[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) g[t] = interior ? wf * gL[t] + (1 - wf) * gR[t] : gL[t];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                double normal = 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) normal += g[a * 3 + d] * nv[d];
                const double target = (R.u[a] - L.u[a]) / ((kind == 1 ? 2 : 1) * dist);
#pragma unroll
                for (int d = 0; d < 3; ++d) g[a * 3 + d] += nv[d] * (target - normal);
            }
            const double div = g[0] + g[4] + g[8];
            const double mu = v.viscosity + (v.wale ? wf * L.rho * nutL + (1 - wf) * R.rho * nutR : 0.0);
            double av[3], an = 0;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                av[a] = -area * (W[a] + W[3] * (wf * L.u[a] + (1 - wf) * R.u[a]));
                an += av[a] * nv[a];
            }
            if (kind == 1)
#pragma unroll
                for (int a = 0; a < 3; ++a) av[a] = an * nv[a];
            an = 0;
#pragma unroll
            for (int a = 0; a < 3; ++a) an += av[a] * nv[a];
            // dJ/dG' then the correction's transpose
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                double row[3], rn = 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    row[d] = mu * (av[a] * nv[d] + nv[a] * av[d] - (a == d ? 2.0 / 3.0 * an : 0.0));
                    rn += row[d] * nv[d];
                }
#pragma unroll
                for (int d = 0; d < 3; ++d) gb[a * 3 + d] += weightC * (row[d] - rn * nv[d]);
            }
            if (v.wale) {
                double jmu = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    double t = -2.0 / 3.0 * div * nv[a];
#pragma unroll
                    for (int d = 0; d < 3; ++d) t += (g[a * 3 + d] + g[d * 3 + a]) * nv[d];
                    jmu += av[a] * t;
                }
                nb += jmu * dmu;
            }
        }
#pragma unroll
        for (int t = 0; t < 9; ++t) gBar[size_t(t) * v.cells + c] = gb[t];
        if (nutBar) nutBar[c] = nb;
    }
}

// gBar += nutBar * d nu_t / d g per cell (the WALE eddy viscosity of the cell's
// gradient, the Nicoud-Ducros relation of wale.cuh:
// nu_t = (Cw Delta)^2 |g|_max (Sd:Sd)^(3/2) / ((S:S)^(5/2) + (Sd:Sd)^(5/4))
// with the invariants of g / |g|_max; zero where the forward gives zero), by a
// reverse pass derived by hand.
__global__ void cartWaleVjp(CartView v, const double* __restrict__ grad, const double* __restrict__ nutBar,
                            double* __restrict__ gBar) {
    // nu_t = (Cw Delta)^2 |g|_max ratio(g / |g|_max) and ratio is homogeneous of
    // degree one, so d nu_t / d g = (Cw Delta)^2 d ratio / d h at h = g / |g|_max
    // (the normalisation's own derivative cancels). With ratio = dd^(3/2) /
    // (ss^(5/2) + dd^(5/4)), ss = S:S (S = sym h), dd = D:D (D = dev sym(h h)):
    // d ss / d h = 2 S and d dd / d h = G h^T + h^T G with G = 2 D.
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        const double nb = nutBar[c];
        if (nb == 0) continue;
        double g[9], scale = 0;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            g[t] = grad[size_t(t) * v.cells + c];
            scale = fmax(scale, ::fabs(g[t]));
        }
        const double delta = cbrt(1 / v.invV[c]);
        if (scale == 0 || v.cw == 0 || delta == 0) continue;
        double h[9];
#pragma unroll
        for (int t = 0; t < 9; ++t) h[t] = g[t] / scale;
        double sq[9];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) sq[3 * a + b] = h[3 * a] * h[b] + h[3 * a + 1] * h[3 + b] + h[3 * a + 2] * h[6 + b];
        const double trace = sq[0] + sq[4] + sq[8];
        double S[9], G[9], ss = 0, dd = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const double sab = .5 * (h[3 * a + b] + h[3 * b + a]);
                double dab = .5 * (sq[3 * a + b] + sq[3 * b + a]);
                if (a == b) dab -= trace / 3.0;
                S[3 * a + b] = sab;
                G[3 * a + b] = 2 * dab;
                ss += sab * sab;
                dd += dab * dab;
            }
        if (!(dd > 0)) continue;
        const double rootD = sqrt(dd), quarter = sqrt(rootD), rootS = sqrt(ss);
        const double numerator = dd * rootD, denominator = ss * ss * rootS + dd * quarter;
        const double den2 = denominator * denominator;
        const double rDd = (1.5 * rootD * denominator - numerator * 1.25 * quarter) / den2;
        const double rSs = -numerator * 2.5 * ss * rootS / den2;
        const double weight = nb * (v.cw * delta * v.cw * delta);
#pragma unroll
        for (int u = 0; u < 3; ++u)
#pragma unroll
            for (int w = 0; w < 3; ++w) {
                double dDd = 0;
#pragma unroll
                for (int k = 0; k < 3; ++k) dDd += G[3 * u + k] * h[3 * w + k] + G[3 * k + w] * h[3 * k + u];
                gBar[size_t(3 * u + w) * v.cells + c] += weight * (rDd * dDd + rSs * 2 * S[3 * u + w]);
            }
    }
}

// Transpose of the Green-Gauss gradient: uBar_c from the gradient adjoints of c
// and of its neighbours (the face velocity of an internal face is the mean of
// its two cells', a boundary face's is w u_c + (1 - w) u_ghost(u_c)), then
// through u = m / rho into qBar (accumulated).
template <int NS>
__global__ void cartGradientVjp(CartView v, const double* __restrict__ q, const double* __restrict__ gBar,
                                double* __restrict__ qBar) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        int i, j, k;
        cellCoords(v, c, i, j, k);
        const double ivc = v.invV[c];
        double uBar[3] = {0, 0, 0};
#pragma unroll
        for (int n = 0; n < 12; ++n) {
            const int s = sideOf(n);
            const bool interior = hasNeighbour(v, s, i, j, k);
            if (interior != (n < 6)) continue;
            const int axis = s >> 1;
            if (interior) {
                const size_t nb = neighbourOf(v, s, c);
                // normal +e_axis; sign +1 for the face's owner (the lower cell)
                const double sc = (s & 1) ? 1.0 : -1.0, sn = -sc;
                const double area = v.area[axis];
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    uBar[a] += .5 * (gBar[size_t(3 * a + axis) * v.cells + c] * sc * area * ivc
                                     + gBar[size_t(3 * a + axis) * v.cells + nb] * sn * area * v.invV[nb]);
            } else {
                const ReactiveTransportFace& f = sideFace(v, s, i, j, k);
                const double sgn = (s & 1) ? 1.0 : -1.0, wgt = f.ownerWeight;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    double du = wgt;  // d u_face[a] / d u_c[a]
                    if (f.kind == 2) du = wgt + (1 - wgt);
                    else if (f.kind == 1) du = wgt + (1 - wgt) * (a == axis ? -1.0 : 1.0);
                    uBar[a] += gBar[size_t(3 * a + axis) * v.cells + c] * du * sgn * f.area * ivc;
                }
            }
        }
        double rho = 0;
#pragma unroll
        for (int kk = 0; kk < NS; ++kk) rho += q[size_t(kk) * v.all + c];
        double rhoBar = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double m = q[size_t(NS + a) * v.all + c];
            qBar[size_t(NS + a) * v.cells + c] += uBar[a] / rho;
            rhoBar -= uBar[a] * m / (rho * rho);
        }
#pragma unroll
        for (int kk = 0; kk < NS; ++kk) qBar[size_t(kk) * v.cells + c] += rhoBar;
    }
}

// out[k] = sum over blocks of partial[b*nv + k], one warp per variable, fixed order.
__global__ void foldPartials(const double* __restrict__ partial, int blocks, int nv, double* out) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= nv) return;
    double s = 0;
    for (int b = lane; b < blocks; b += 32) s += partial[size_t(b) * nv + k];
    s = warpSum(s);
    if (lane == 0) out[k] = s;
}

}  // namespace rb200
