// Face-graph transport kernels (any polyhedral face list), sm_100a, FP64.
//
// Operator semantics are those of the reference functors in
// src/reactiveTransport/reactiveTransportKernels.h:
//   cellPrimitives   <- Cells            :193-199
//   cellGradients    <- Gradients        :290-301
//   cellWale         <- WaleViscosities  :303-313
//   faceSpeeds       <- FaceSpeeds       :315-341
//   faceWork         <- Faces            :343-500 (HLL core, viscous/WALE traction,
//                                                  conduction, Fick diffusion, WALE
//                                                  scalar heat flux and species mixing)
//   cellRates        <- Rhs / Advance    :502-528, :551-560
//   cellSteps        <- Step             :529-549
// The data layout is this project's: conserved and gas fields are SoA with
// stride cells+fixed; face work is SoA (one array per field) so every load in
// the gather is coalesced over faces; one thread owns one cell and applies each
// face's work record to up to eight variables from registers, so a face record
// is read once per (cell, incidence, 8 variables) instead of once per variable.
#pragma once
#include "common.cuh"
#include "wale.cuh"
#include "../../include/reactive_b200_types.h"

namespace rb200 {

enum FaceWorkField {
    FW_VELOCITY = 0, FW_ADV_L, FW_ADV_R, FW_P_MOM, FW_P_ENERGY, FW_TRACTION_X, FW_TRACTION_Y,
    FW_TRACTION_Z, FW_ENERGY, FW_DIFFUSION, FW_SUM_J, FW_CARRIER_FLUX, FW_FIELDS
};

struct GraphView {
    size_t cells = 0, fixed = 0, all = 0, ns = 0, nv = 0, faces = 0, nBoundary = 0;
    size_t ownBegin = 0, ownEnd = SIZE_MAX;  // own cells: stage update, CFL minimum and ledger
    int mechanical = 0;
    double viscosity = 0, conductivity = 0, diffusivity = 0, waveFactor = 1;
    const ReactiveTransportFace* face = nullptr;
    const int64_t* row = nullptr;        // cells+1 offsets into incidence
    const int64_t* incidence = nullptr;  // -(f+1): cell owns f; +(f+1): cell is f's neighbour
    const int64_t* boundary = nullptr;   // boundary face ids
    const double* invV = nullptr;
    const ReactiveTransportState* state = nullptr;  // all
    const double* q = nullptr;                       // SoA nv x all
    ReactiveTransportPrimitive* primitive = nullptr; // all
    double* grad = nullptr;                          // SoA 9 x cells
    double* nut = nullptr;                           // cells
    bool wale = false;
    double cw = 0;
    const double* gasY = nullptr;                    // SoA ns x all
    const double* gasH = nullptr;
    double* work = nullptr;                          // SoA FW_FIELDS x faces
    int* carrier = nullptr;                          // faces
    double* faceSpeed = nullptr;                     // faces
    double* step = nullptr;                          // cells
    unsigned* waleError = nullptr;
    // WALE scalar closure (turbulent Prandtl heat flux rho nu_t cp / Pr_t grad T,
    // turbulent Schmidt species mixing rho nu_t / Sc_t grad Y); 0 disables a term
    bool sgs = false;
    double pr = 0, sc = 0;
    const double* mixCp = nullptr;                   // all, mixture cp
    const double* spH = nullptr;                     // SoA ns x all, effective species enthalpies
    double* sgsWork = nullptr;                       // SoA 3 x faces: diffusion, sumJ, carrier flux
    int* sgsCarrier = nullptr;                       // faces
    // capillary closure: a resolved material color (cells + fixed) with its
    // diffuse interface geometry and the balanced HLLC face core; the conserved
    // vector carries the liquid inventory of species capSpecies at ns + 4
    bool capillary = false;
    size_t capSpecies = 0;
    double sigma = 0, capCfl = 0, geomEps = 0;
    const double* color = nullptr;                   // all
    double* cGrad = nullptr;                         // cells x 3 (packed per cell)
    double* cNormal = nullptr;                       // cells x 3, from color 1 towards color 0
    double* cArea = nullptr;                         // cells: |grad color|
    double* cCurv = nullptr;                         // cells
    double* cEnergy = nullptr;                       // cells: sigma |grad color|
    unsigned* capError = nullptr;                    // bit kCapillaryBit on failure
};

constexpr unsigned kCapillaryBit = 8u;

// The species-mixing record of one face (zero diffusion: no mixing flux).
struct SgsFace {
    double diffusion = 0, sumJ = 0, carrierFlux = 0, rhoL = 1, rhoR = 1;
    int carrier = 0;
};

__device__ __forceinline__ size_t rightCell(const GraphView& v, const ReactiveTransportFace& f) {
    return f.neighbour >= 0 ? size_t(f.neighbour)
                            : (f.kind == 3 ? v.cells + size_t(f.fixed) : size_t(f.owner));
}

// Right-side velocities with the slip-wall mirror u - 2(u.n)n.
__device__ __forceinline__ void sideVelocities(const GraphView& v, const ReactiveTransportFace& f,
                                               double ul[3], double ur[3]) {
    const ReactiveTransportPrimitive l = v.primitive[f.owner];
    const ReactiveTransportPrimitive r = v.primitive[rightCell(v, f)];
    double dot = 0;
    for (int d = 0; d < 3; ++d) { ul[d] = l.u[d]; ur[d] = r.u[d]; dot += r.u[d] * f.normal[d]; }
    if (f.kind == 1)
        for (int d = 0; d < 3; ++d) ur[d] -= 2 * dot * f.normal[d];
}

__device__ __forceinline__ double faceNut(const GraphView& v, const ReactiveTransportFace& f, bool right) {
    if (!v.wale) return 0;
    return v.nut[right && f.neighbour >= 0 ? size_t(f.neighbour) : size_t(f.owner)];
}

__device__ __forceinline__ SgsFace loadSgs(const GraphView& v, const ReactiveTransportFace& f, size_t fi, size_t r) {
    SgsFace g;
    if (v.sgs && v.sc > 0) {
        g.diffusion = v.sgsWork[fi];
        g.sumJ = v.sgsWork[v.faces + fi];
        g.carrierFlux = v.sgsWork[2 * v.faces + fi];
        g.carrier = v.sgsCarrier[fi];
        g.rhoL = v.state[f.owner].rho;
        g.rhoR = v.state[r].rho;
    }
    return g;
}

__global__ void cellPrimitives(GraphView v, size_t begin, size_t end) {
    for (size_t c = begin + blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < end;
         c += size_t(blockDim.x) * gridDim.x) {
        ReactiveTransportPrimitive p{};
        for (size_t k = 0; k < v.ns; ++k) p.rho += v.q[k * v.all + c];
        for (int d = 0; d < 3; ++d) p.u[d] = v.q[(v.ns + d) * v.all + c] / p.rho;
        v.primitive[c] = p;
    }
}

__global__ void cellGradients(GraphView v) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells;
         c += size_t(blockDim.x) * gridDim.x) {
        double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const double iv = v.invV[c];
        for (int64_t j = v.row[c]; j < v.row[c + 1]; ++j) {
            const int64_t e = v.incidence[j];
            const ReactiveTransportFace f = v.face[e < 0 ? -e - 1 : e - 1];
            double ul[3], ur[3];
            sideVelocities(v, f, ul, ur);
            const double scale = (e < 0 ? 1.0 : -1.0) * f.area * iv;
            for (int i = 0; i < 3; ++i) {
                const double uf = f.ownerWeight * ul[i] + (1 - f.ownerWeight) * ur[i];
                for (int d = 0; d < 3; ++d) g[3 * i + d] += uf * f.normal[d] * scale;
            }
        }
        for (int j = 0; j < 9; ++j) v.grad[j * v.cells + c] = g[j];
    }
}

__global__ void cellWale(GraphView v) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells;
         c += size_t(blockDim.x) * gridDim.x) {
        double g[9];
        for (int j = 0; j < 9; ++j) g[j] = v.grad[j * v.cells + c];
        const double volume = 1 / v.invV[c];
        double delta = 0, nut = 0;
        bool ok = isfinite(volume) && volume > 0;
        if (ok) { delta = cbrt(volume); ok = isfinite(delta) && delta > 0; }
        ok = ok && waleEddyViscosity(g, delta, v.cw, nut);
        if (!ok || !isfinite(nut) || nut < 0 || !isfinite(v.state[c].rho * nut)) {
            atomicOr(v.waleError, 1u);
            continue;
        }
        v.nut[c] = nut;
    }
}

__global__ void faceSpeeds(GraphView v) {
    for (size_t fi = blockIdx.x * size_t(blockDim.x) + threadIdx.x; fi < v.faces;
         fi += size_t(blockDim.x) * gridDim.x) {
        const ReactiveTransportFace f = v.face[fi];
        const ReactiveTransportState sl = v.state[f.owner], sr = v.state[rightCell(v, f)];
        double ul[3], ur[3], unL = 0, unR = 0;
        sideVelocities(v, f, ul, ur);
        for (int d = 0; d < 3; ++d) { unL += ul[d] * f.normal[d]; unR += ur[d] * f.normal[d]; }
        const double aL = v.waveFactor * sl.sound, aR = v.waveFactor * sr.sound;
        const double left = dmin(0, dmin(unL - aL, unR - aR)), right = dmax(0, dmax(unL + aL, unR + aR));
        const double invWave = 1 / (right - left);
        const double rhoNut = v.wale ? f.ownerWeight * sl.rho * faceNut(v, f, false)
                                           + (1 - f.ownerWeight) * sr.rho * faceNut(v, f, true)
                                     : 0;
        const double mu = v.viscosity + rhoNut;
        const double D = v.diffusivity
            + dmax(dmax(4 * mu / (3 * sl.rho), 4 * mu / (3 * sr.rho)),
                   dmax(v.conductivity / (sl.rho * sl.cv), v.conductivity / (sr.rho * sr.cv)));
        double scalar = 0;
        if (v.sgs && f.kind != 1) {
            const size_t r = rightCell(v, f);
            if (v.pr > 0) {
                const double k = rhoNut * (f.ownerWeight * v.mixCp[f.owner] + (1 - f.ownerWeight) * v.mixCp[r]) / v.pr;
                scalar = dmax(scalar, dmax(k / (sl.rho * sl.cv), k / (sr.rho * sr.cv)));
            }
            if (v.sc > 0) scalar = dmax(scalar, dmax(rhoNut / sl.rho, rhoNut / sr.rho) / v.sc);
        }
        double speed = dmax(fabs(unL) + aL, fabs(unR) + aR) + 2 * (D + scalar) / f.distance;
        if (!isfinite(unL) || !isfinite(unR) || !isfinite(speed) || !isfinite(invWave) || right <= left)
            speed = -1;
        v.faceSpeed[fi] = speed;
    }
}

// ---------------------------------------------------------------------------
// Capillary closure (src/reactiveInterface/reactiveUnstructuredInterface.h and
// reactiveBalancedCapillary.h): the color's Green-Gauss gradient, interface
// normal, area density and curvature on the face graph, and the face core in
// which the pressure jump sigma kappa (c_L - c_R) enters a contact-preserving
// HLLC solver through pi = p - sigma kappa c and the shared surface stress
// sigma |grad c| (I - n n) restores the momentum and energy fluxes.
__device__ __forceinline__ bool unitColor(double c) { return isfinite(c) && c >= 0 && c <= 1; }
__device__ __forceinline__ double capOtherColor(const GraphView& v, const ReactiveTransportFace& f) {
    if (f.neighbour >= 0) return v.color[size_t(f.neighbour)];
    if (f.kind == 3) return v.color[v.cells + size_t(f.fixed)];
    return v.color[size_t(f.owner)];
}
__device__ __forceinline__ double capFaceColor(const GraphView& v, const ReactiveTransportFace& f) {
    return f.ownerWeight * v.color[size_t(f.owner)] + (1 - f.ownerWeight) * capOtherColor(v, f);
}
// The interface normal at a face: the weighted cell normals, normalised when
// nonzero (boundary faces take the owner's).
__device__ __forceinline__ void capFaceNormal(const GraphView& v, const ReactiveTransportFace& f, double out[3]) {
    const size_t l = size_t(f.owner), r = f.neighbour >= 0 ? size_t(f.neighbour) : l;
    double mag2 = 0;
    for (int d = 0; d < 3; ++d) {
        out[d] = f.ownerWeight * v.cNormal[3 * l + d] + (1 - f.ownerWeight) * v.cNormal[3 * r + d];
        mag2 += out[d] * out[d];
    }
    if (mag2 > 0) {
        const double inv = 1 / sqrt(mag2);
        for (int d = 0; d < 3; ++d) out[d] *= inv;
    }
}

// Gradient of the color (face values less the cell's, so a uniform color has
// none), its magnitude (the interface area density) and the unit normal where
// |grad c| times the cell size exceeds the geometry threshold.
__global__ void interfaceGradient(GraphView v) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        bool ok = unitColor(v.color[c]);
        double g[3] = {0, 0, 0};
        for (int64_t j = v.row[c]; ok && j < v.row[c + 1]; ++j) {
            const int64_t e = v.incidence[j];
            const ReactiveTransportFace& f = v.face[size_t(e < 0 ? -e - 1 : e - 1)];
            const double orientation = e < 0 ? 1.0 : -1.0;
            const double cf = capFaceColor(v, f);
            if (!unitColor(cf)) { ok = false; break; }
            for (int d = 0; d < 3; ++d) g[d] += (cf - v.color[c]) * orientation * f.area * f.normal[d];
        }
        double mag2 = 0;
        for (int d = 0; ok && d < 3; ++d) {
            g[d] *= v.invV[c];
            mag2 += g[d] * g[d];
            if (!isfinite(g[d])) ok = false;
            v.cGrad[3 * c + d] = g[d];
        }
        if (ok) {
            const double mag = sqrt(mag2);
            if (!isfinite(mag) || mag < 0) ok = false;
            else {
                v.cArea[c] = mag;
                const bool active = mag * cbrt(1 / v.invV[c]) > v.geomEps;
                for (int d = 0; d < 3; ++d) v.cNormal[3 * c + d] = active ? -g[d] / mag : 0;
            }
        }
        if (!ok) atomicOr(v.capError, kCapillaryBit);
    }
}

// Curvature as the divergence of the interface normal (face normals less the
// cell's) and the surface energy density sigma |grad c|.
__global__ void interfaceCurvature(GraphView v) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells; c += size_t(blockDim.x) * gridDim.x) {
        double sum = 0;
        for (int64_t j = v.row[c]; j < v.row[c + 1]; ++j) {
            const int64_t e = v.incidence[j];
            const ReactiveTransportFace& f = v.face[size_t(e < 0 ? -e - 1 : e - 1)];
            const double orientation = e < 0 ? 1.0 : -1.0;
            double nf[3];
            capFaceNormal(v, f, nf);
            for (int d = 0; d < 3; ++d) sum += (nf[d] - v.cNormal[3 * c + d]) * orientation * f.area * f.normal[d];
        }
        const double kappa = sum * v.invV[c];
        if (!isfinite(kappa)) atomicOr(v.capError, kCapillaryBit);
        else v.cCurv[c] = kappa;
        v.cEnergy[c] = v.sigma * v.cArea[c];
    }
}

struct CapSide {
    double rho, u[3], p, sound, E, color;
};
struct CapResult {
    double advL, advR, contact, pMom, pEnergy, capEnergy, capMom[3];
};

// The balanced capillary core of one face (left = owner side), false when it
// cannot be formed. curvature, colorFace and the surface stress come from the
// shared face geometry.
__device__ inline bool capillaryCore(const CapSide& L, const CapSide& R, const double n[3], double curvature,
                                     double sigma, double colorFace, const double stress[9], CapResult& o) {
    auto valid = [](const CapSide& s) {
        if (!isfinite(s.rho) || s.rho <= 0 || !isfinite(s.p) || s.p <= 0 || !isfinite(s.sound) || s.sound <= 0
            || !isfinite(s.E) || !unitColor(s.color))
            return false;
        for (int d = 0; d < 3; ++d)
            if (!isfinite(s.u[d])) return false;
        return true;
    };
    if (!valid(L) || !valid(R) || !isfinite(curvature) || !isfinite(sigma) || sigma < 0 || !unitColor(colorFace))
        return false;
    double n2 = 0, unL = 0, unR = 0;
    for (int d = 0; d < 3; ++d) {
        if (!isfinite(n[d])) return false;
        n2 += n[d] * n[d];
        unL += L.u[d] * n[d];
        unR += R.u[d] * n[d];
    }
    if (!isfinite(n2) || fabs(n2 - 1) > 1e-10) return false;
    for (int j = 0; j < 9; ++j)
        if (!isfinite(stress[j])) return false;
    const double piL = L.p - sigma * curvature * L.color, piR = R.p - sigma * curvature * R.color;
    if (!isfinite(piL) || !isfinite(piR)) return false;
    const double sl = dmin(0, dmin(unL - L.sound, unR - R.sound)), sr = dmax(0, dmax(unL + L.sound, unR + R.sound));
    const double den = L.rho * (sl - unL) - R.rho * (sr - unR);
    if (!isfinite(den) || den == 0 || !isfinite(sl) || !isfinite(sr) || sr <= sl) return false;
    const double star = (piR - piL + L.rho * unL * (sl - unL) - R.rho * unR * (sr - unR)) / den;
    o = CapResult{};
    double mass;
    if (!isfinite(star) || star <= sl || star >= sr) {
        // waves outrunning the estimated bounds: the HLL coefficients
        const double inv = 1 / (sr - sl);
        o.contact = (sr * unL - sl * unR) * inv;
        o.advL = sr * (unL - sl) * inv;
        o.advR = sl * (sr - unR) * inv;
        mass = o.advL * L.rho + o.advR * R.rho;
        o.pMom = (sr * piL - sl * piR) * inv;
        o.pEnergy = (sr * piL * unL - sl * piR * unR) * inv;
    } else {
        const bool useLeft = star >= 0;
        const CapSide& side = useLeft ? L : R;
        const double un = useLeft ? unL : unR, wave = useLeft ? sl : sr, pi = useLeft ? piL : piR;
        const bool supersonic = (useLeft && sl >= 0) || (!useLeft && sr <= 0);
        o.contact = supersonic ? un : star;
        if (supersonic) {
            mass = side.rho * un;
            o.pMom = pi;
            o.pEnergy = pi * un;
        } else {
            const double rhoStar = side.rho * (wave - un) / (wave - star);
            const double piStar = pi + side.rho * (wave - un) * (star - un);
            const double eStar = ((wave - un) * side.E - pi * un + piStar * star) / (wave - star);
            mass = rhoStar * star;
            o.pMom = piStar + mass * (star - un);
            o.pEnergy = star * (eStar + piStar) - mass * side.E / side.rho;
        }
        if (useLeft) o.advL = mass / L.rho;
        else o.advR = mass / R.rho;
    }
    // the surface traction and its work with one shared face velocity (the
    // average tangential velocity plus the contact speed along n)
    double faceVelocity[3], averageNormal = 0;
    for (int d = 0; d < 3; ++d) {
        faceVelocity[d] = 0.5 * (L.u[d] + R.u[d]);
        averageNormal += faceVelocity[d] * n[d];
    }
    for (int d = 0; d < 3; ++d) faceVelocity[d] += (o.contact - averageNormal) * n[d];
    o.capEnergy = 0;
    for (int i = 0; i < 3; ++i) {
        double traction = 0;
        for (int j = 0; j < 3; ++j) traction += stress[3 * i + j] * n[j];
        o.capMom[i] = sigma * curvature * colorFace * n[i] - traction;
        o.capEnergy += faceVelocity[i] * o.capMom[i];
    }
    const double advective = o.advL * L.E + o.advR * R.E;
    const double total = advective + o.pEnergy + o.capEnergy;
    if (!isfinite(mass) || !isfinite(o.pMom) || !isfinite(o.pEnergy) || !isfinite(o.capEnergy) || !isfinite(total))
        return false;
    for (int d = 0; d < 3; ++d) {
        const double momentum = o.advL * L.rho * L.u[d] + o.advR * R.rho * R.u[d] + o.pMom * n[d] + o.capMom[d];
        if (!isfinite(momentum) || !isfinite(o.capMom[d])) return false;
    }
    return true;
}

// The shared face geometry of face f: curvature, color and surface stress.
__device__ inline bool capillaryFaceGeometry(const GraphView& v, const ReactiveTransportFace& f, double& curvature,
                                             double& colorFace, double stress[9]) {
    const size_t l = size_t(f.owner), r = f.neighbour >= 0 ? size_t(f.neighbour) : l;
    if (!isfinite(v.sigma) || v.sigma < 0) return false;
    const double w = f.ownerWeight;
    curvature = w * v.cCurv[l] + (1 - w) * v.cCurv[r];
    colorFace = capFaceColor(v, f);
    double ni[3];
    capFaceNormal(v, f, ni);
    const double scale = v.sigma * (w * v.cArea[l] + (1 - w) * v.cArea[r]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) stress[3 * i + j] = scale * ((i == j ? 1.0 : 0.0) - ni[i] * ni[j]);
    return isfinite(curvature) && unitColor(colorFace) && isfinite(scale);
}

__global__ void faceWork(GraphView v) {
    for (size_t fi = blockIdx.x * size_t(blockDim.x) + threadIdx.x; fi < v.faces;
         fi += size_t(blockDim.x) * gridDim.x) {
        const ReactiveTransportFace f = v.face[fi];
        const size_t l = size_t(f.owner), r = rightCell(v, f);
        const ReactiveTransportState sl = v.state[l], sr = v.state[r];
        const double w = f.ownerWeight;
        double ul[3], ur[3], unL = 0, unR = 0;
        sideVelocities(v, f, ul, ur);
        for (int d = 0; d < 3; ++d) { unL += ul[d] * f.normal[d]; unR += ur[d] * f.normal[d]; }
        const double aL = v.waveFactor * sl.sound, aR = v.waveFactor * sr.sound;
        const double left = dmin(0, dmin(unL - aL, unR - aR)), right = dmax(0, dmax(unL + aL, unR + aR));
        const double invWave = 1 / (right - left);
        double out[FW_FIELDS] = {};
        out[FW_VELOCITY] = (right * unL - left * unR) * invWave;
        out[FW_ADV_L] = right * (unL - left) * invWave;
        out[FW_ADV_R] = left * (right - unR) * invWave;
        out[FW_P_MOM] = (right * sl.p - left * sr.p) * invWave;
        out[FW_P_ENERGY] = (right * sl.p * unL - left * sr.p * unR) * invWave;
        double traction[3] = {0, 0, 0}, energy = 0;
        CapResult cap{};
        if (v.capillary) {
            CapSide cl, cr;
            cl.rho = sl.rho; cr.rho = sr.rho;
            cl.p = sl.p; cr.p = sr.p;
            cl.sound = aL; cr.sound = aR;
            cl.E = v.q[(v.ns + 3) * v.all + l];
            cr.E = v.q[(v.ns + 3) * v.all + r];
            cl.color = v.color[l]; cr.color = v.color[r];
            for (int d = 0; d < 3; ++d) { cl.u[d] = ul[d]; cr.u[d] = ur[d]; }
            double curvature, colorFace, stress[9];
            if (!capillaryFaceGeometry(v, f, curvature, colorFace, stress)
                || !capillaryCore(cl, cr, f.normal, curvature, v.sigma, colorFace, stress, cap)) {
                atomicOr(v.capError, kCapillaryBit);
                cap = CapResult{};
            }
            out[FW_VELOCITY] = cap.contact;
            out[FW_ADV_L] = cap.advL;
            out[FW_ADV_R] = cap.advR;
            out[FW_P_MOM] = cap.pMom;
            out[FW_P_ENERGY] = cap.pEnergy;
            energy += cap.capEnergy;
        }
        if (v.viscosity > 0 || v.wale) {
            double g[9];
            for (int j = 0; j < 9; ++j) {
                g[j] = v.grad[j * v.cells + l];
                if (f.neighbour >= 0) g[j] = w * g[j] + (1 - w) * v.grad[j * v.cells + r];
            }
            for (int i = 0; i < 3; ++i) {
                double normal = 0;
                for (int d = 0; d < 3; ++d) normal += g[i * 3 + d] * f.normal[d];
                const double target = (ur[i] - ul[i]) / ((f.kind == 1 ? 2 : 1) * f.distance);
                for (int d = 0; d < 3; ++d) g[i * 3 + d] += f.normal[d] * (target - normal);
            }
            const double div = g[0] + g[4] + g[8];
            const double mu = v.viscosity
                + (v.wale ? w * sl.rho * faceNut(v, f, false) + (1 - w) * sr.rho * faceNut(v, f, true) : 0);
            for (int i = 0; i < 3; ++i)
                for (int d = 0; d < 3; ++d)
                    traction[i] += mu * (g[3 * i + d] + g[3 * d + i] - (i == d ? 2 * div / 3 : 0)) * f.normal[d];
            if (f.kind == 1) {
                double dot = 0;
                for (int d = 0; d < 3; ++d) dot += traction[d] * f.normal[d];
                for (int d = 0; d < 3; ++d) traction[d] = dot * f.normal[d];
            }
            for (int d = 0; d < 3; ++d) energy -= traction[d] * (w * ul[d] + (1 - w) * ur[d]);
        }
        if (v.conductivity > 0 && f.kind != 1) energy -= v.conductivity * (sr.T - sl.T) / f.distance;
        if (v.sgs && v.pr > 0 && f.kind != 1) {
            const double rhoNut = w * sl.rho * faceNut(v, f, false) + (1 - w) * sr.rho * faceNut(v, f, true);
            const double cp = w * v.mixCp[l] + (1 - w) * v.mixCp[r];
            energy -= rhoNut * cp / v.pr * (sr.T - sl.T) / f.distance;
        }
        int carrier = 0;
        if (v.diffusivity > 0 && sl.gasMass > 0 && sr.gasMass > 0 && f.kind != 1) {
            const double mass = f.neighbour >= 0
                ? sl.gasMass * sr.gasMass / ((1 - w) * sr.gasMass + w * sl.gasMass) : sl.gasMass;
            const double diffusion = -mass * v.diffusivity / f.distance;
            double sumJ = 0, largest = -1;
            for (size_t k = 0; k < v.ns; ++k) {
                const double yl = v.gasY[k * v.all + l], yr = v.gasY[k * v.all + r];
                sumJ += diffusion * (yr - yl);
                const double y = w * yl + (1 - w) * yr;
                if (y > largest) { largest = y; carrier = int(k); }
            }
            const double hc = w * v.gasH[size_t(carrier) * v.all + l] + (1 - w) * v.gasH[size_t(carrier) * v.all + r];
            double carrierFlux = 0;
            for (size_t k = 0; k < v.ns; ++k) {
                if (int(k) == carrier) continue;
                const double yl = v.gasY[k * v.all + l], yr = v.gasY[k * v.all + r];
                const double J = diffusion * (yr - yl) - (w * yl + (1 - w) * yr) * sumJ;
                carrierFlux -= J;
                const double hk = w * v.gasH[k * v.all + l] + (1 - w) * v.gasH[k * v.all + r];
                energy += J * (hk - hc);
            }
            out[FW_DIFFUSION] = diffusion;
            out[FW_SUM_J] = sumJ;
            out[FW_CARRIER_FLUX] = carrierFlux;
        }
        SgsFace sg;
        if (v.sgs && v.sc > 0 && f.kind != 1) {
            const double rhoNut = w * sl.rho * faceNut(v, f, false) + (1 - w) * sr.rho * faceNut(v, f, true);
            sg.diffusion = -rhoNut / v.sc / f.distance;
            double largest = -1;
            for (size_t k = 0; k < v.ns; ++k) {
                const double yl = v.q[k * v.all + l] / sl.rho, yr = v.q[k * v.all + r] / sr.rho;
                sg.sumJ += sg.diffusion * (yr - yl);
                const double y = w * yl + (1 - w) * yr;
                if (y > largest) { largest = y; sg.carrier = int(k); }
            }
            const size_t kc = size_t(sg.carrier);
            const double hc = w * v.spH[kc * v.all + l] + (1 - w) * v.spH[kc * v.all + r];
            for (size_t k = 0; k < v.ns; ++k) {
                if (k == kc) continue;
                const double yl = v.q[k * v.all + l] / sl.rho, yr = v.q[k * v.all + r] / sr.rho;
                const double J = sg.diffusion * (yr - yl) - (w * yl + (1 - w) * yr) * sg.sumJ;
                sg.carrierFlux -= J;
                const double hk = w * v.spH[k * v.all + l] + (1 - w) * v.spH[k * v.all + r];
                energy += J * (hk - hc);
            }
        }
        if (v.capillary) {
            // the liquid inventory of each side lies within its species' density
            const size_t sk = v.capSpecies, lk = v.ns + 4;
            const double slq = v.q[sk * v.all + l], srq = v.q[sk * v.all + r];
            const double ml = v.q[lk * v.all + l], mr = v.q[lk * v.all + r];
            if (!isfinite(slq) || !isfinite(srq) || !isfinite(ml) || !isfinite(mr) || slq < 0 || srq < 0 || ml < 0
                || mr < 0 || ml > slq || mr > srq)
                atomicOr(v.capError, kCapillaryBit);
            // the viscous work above used the viscous traction only; the shared
            // capillary momentum flux joins the face traction here
            for (int d = 0; d < 3; ++d) traction[d] -= cap.capMom[d];
        }
        if (v.sgs && v.sc > 0) {
            v.sgsWork[fi] = sg.diffusion;
            v.sgsWork[v.faces + fi] = sg.sumJ;
            v.sgsWork[2 * v.faces + fi] = sg.carrierFlux;
            v.sgsCarrier[fi] = sg.carrier;
        }
        if (v.wale) {
            bool bad = !isfinite(energy) || !isfinite(sg.diffusion) || !isfinite(sg.sumJ) || !isfinite(sg.carrierFlux);
            for (int d = 0; d < 3; ++d) bad |= !isfinite(traction[d]);
            if (bad) atomicOr(v.waleError, 1u);
        }
        out[FW_TRACTION_X] = traction[0];
        out[FW_TRACTION_Y] = traction[1];
        out[FW_TRACTION_Z] = traction[2];
        out[FW_ENERGY] = energy;
        for (int j = 0; j < FW_FIELDS; ++j) v.work[size_t(j) * v.faces + fi] = out[j];
        v.carrier[fi] = carrier;
    }
}

// Flux of variable k through face fi, times the face area (the reference's
// View::faceFlux with speciesDiffusion and sgsSpeciesFlux,
// src/reactiveTransport/reactiveTransportKernels.h:150-191).
__device__ __forceinline__ double faceFluxK(const GraphView& v, const ReactiveTransportFace& f, size_t fi,
                                            size_t r, size_t k, const double* wk, int carrier, const SgsFace& sg) {
    const size_t l = size_t(f.owner);
    const double ql = v.q[k * v.all + l];
    double qr = v.q[k * v.all + r];
    const size_t ns = v.ns;
    if (f.kind == 1 && k >= ns && k < ns + 3) {
        double normal = 0;
        for (int d = 0; d < 3; ++d) normal += v.q[(ns + d) * v.all + r] * f.normal[d];
        qr -= 2 * normal * f.normal[k - ns];
    }
    double flux = wk[FW_ADV_L] * ql + wk[FW_ADV_R] * qr;
    if (k >= ns && k < ns + 3) flux += wk[FW_P_MOM] * f.normal[k - ns];
    if (k == ns + 3) flux += wk[FW_P_ENERGY];
    if (k < ns) {
        double diffusion = 0;
        if (wk[FW_DIFFUSION] != 0) {
            if (int(k) == carrier) diffusion += wk[FW_CARRIER_FLUX];
            else {
                const double yl = v.gasY[k * v.all + l], yr = v.gasY[k * v.all + r];
                diffusion += wk[FW_DIFFUSION] * (yr - yl)
                    - (f.ownerWeight * yl + (1 - f.ownerWeight) * yr) * wk[FW_SUM_J];
            }
        }
        if (sg.diffusion != 0) {
            if (int(k) == sg.carrier) diffusion += sg.carrierFlux;
            else {
                const double yl = v.q[k * v.all + l] / sg.rhoL, yr = v.q[k * v.all + r] / sg.rhoR;
                diffusion += sg.diffusion * (yr - yl) - (f.ownerWeight * yl + (1 - f.ownerWeight) * yr) * sg.sumJ;
            }
        }
        flux += diffusion;
    } else if (v.capillary && k == ns + 4) {
        // the liquid inventory moves with its species' turbulent mixing flux
        // in proportion to its liquid fraction on each side
        if (sg.diffusion != 0) {
            const size_t sk = v.capSpecies;
            const double sl = v.q[sk * v.all + l], sr = v.q[sk * v.all + r];
            const double ml = v.q[(ns + 4) * v.all + l], mr = v.q[(ns + 4) * v.all + r];
            if (sl < 0 || sr < 0 || ml < 0 || mr < 0 || ml > sl || mr > sr) atomicOr(v.capError, kCapillaryBit);
            else {
                double species;
                if (int(sk) == sg.carrier) species = sg.carrierFlux;
                else {
                    const double yl = v.q[sk * v.all + l] / sg.rhoL, yr = v.q[sk * v.all + r] / sg.rhoR;
                    species = sg.diffusion * (yr - yl) - (f.ownerWeight * yl + (1 - f.ownerWeight) * yr) * sg.sumJ;
                }
                const double fl = sl > 0 ? ml / sl : 0, fr = sr > 0 ? mr / sr : 0;
                flux += (f.ownerWeight * fl + (1 - f.ownerWeight) * fr) * species;
            }
        }
    } else if (k < ns + 3) flux -= wk[FW_TRACTION_X + (k - ns)];
    else if (k == ns + 3) flux += wk[FW_ENERGY];
    return flux * f.area;
}

// mode 0: rate -> out (SoA nv x cells, the materialised RHS)
// mode 1: SSPRK2 stage 0, out = q + dt*rate
// mode 2: SSPRK2 stage 1, out = .5*out + .5*(q + dt*rate)   (out holds q^n)
// out has stride `outStride` (cells for the RHS, all for the RK buffers).
template <int CHUNK>
__global__ void cellRates(GraphView v, double* out, size_t outStride, int mode, double dt) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells;
         c += size_t(blockDim.x) * gridDim.x) {
        if (c < v.ownBegin || c >= v.ownEnd) continue;
        const double iv = v.invV[c];
        const int64_t begin = v.row[c], end = v.row[c + 1];
        double div = 0;
        if (v.mechanical) {
            for (int64_t j = begin; j < end; ++j) {
                const int64_t e = v.incidence[j];
                const size_t fi = size_t(e < 0 ? -e - 1 : e - 1);
                const double sign = e < 0 ? -1 : 1;
                div -= sign * v.work[FW_VELOCITY * v.faces + fi] * v.face[fi].area * iv;
            }
        }
        for (size_t k0 = 0; k0 < v.nv; k0 += CHUNK) {
            double acc[CHUNK];
#pragma unroll
            for (int kk = 0; kk < CHUNK; ++kk) acc[kk] = 0;
            for (int64_t j = begin; j < end; ++j) {
                const int64_t e = v.incidence[j];
                const size_t fi = size_t(e < 0 ? -e - 1 : e - 1);
                const double sign = e < 0 ? -1 : 1;
                const ReactiveTransportFace f = v.face[fi];
                const size_t r = rightCell(v, f);
                double wk[FW_FIELDS];
#pragma unroll
                for (int t = 0; t < FW_FIELDS; ++t) wk[t] = v.work[size_t(t) * v.faces + fi];
                const int carrier = v.carrier[fi];
                const SgsFace sg = loadSgs(v, f, fi, r);
#pragma unroll
                for (int kk = 0; kk < CHUNK; ++kk) {
                    const size_t k = k0 + kk;
                    if (k < v.nv) acc[kk] += sign * faceFluxK(v, f, fi, r, k, wk, carrier, sg) * iv;
                }
            }
#pragma unroll
            for (int kk = 0; kk < CHUNK; ++kk) {
                const size_t k = k0 + kk;
                if (k >= v.nv) break;
                double rate = acc[kk];
                if (v.mechanical && k >= v.ns + 4)
                    rate += (v.q[k * v.all + c] + (k == v.ns + 4 ? 1 : -1) * v.state[c].dilatation) * div;
                const size_t o = k * outStride + c;
                if (mode == 0) out[o] = rate;
                else if (mode == 1) out[o] = v.q[k * v.all + c] + dt * rate;
                else out[o] = .5 * out[o] + .5 * (v.q[k * v.all + c] + dt * rate);
            }
        }
    }
}

__global__ void cellSteps(GraphView v, double cfl, double maximumStep) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < v.cells;
         c += size_t(blockDim.x) * gridDim.x) {
        if (c < v.ownBegin || c >= v.ownEnd) { v.step[c] = maximumStep; continue; }  // not this handle's cell
        double denominator = 0;
        bool bad = false;
        for (int64_t j = v.row[c]; j < v.row[c + 1]; ++j) {
            const int64_t e = v.incidence[j];
            const size_t fi = size_t(e < 0 ? -e - 1 : e - 1);
            const double speed = v.faceSpeed[fi];
            if (!isfinite(speed) || speed < 0) { bad = true; break; }
            denominator += v.face[fi].area * speed;
        }
        double step = denominator > 0 ? dmin(maximumStep, cfl / (v.invV[c] * denominator)) : maximumStep;
        if (v.capillary && v.sigma > 0) {
            // capillary waves: dt <= capCfl sqrt(rho V / (pi sigma)) where the interface is resolved
            const double volume = 1 / v.invV[c];
            if (v.cArea[c] * cbrt(volume) > v.geomEps)
                step = dmin(step, v.capCfl * sqrt(v.state[c].rho * volume / (3.141592653589793238462643383279502884
                                                                              * v.sigma)));
        }
        if (bad || !isfinite(denominator) || denominator < 0) step = -1;
        v.step[c] = step;
    }
}

// Global minimum with invalid (non-finite or non-positive) entries absorbing as
// -1 (the reference's Minimum, src/reactiveTransport/reactiveTransport.cpp:222-232).
// Pass 1 writes one value per block, pass 2 (one block) folds them.
__global__ void minimumReduce(const double* in, size_t n, double* out) {
    __shared__ double warpValues[32];
    double m = HUGE_VAL;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(blockDim.x) * gridDim.x) {
        const double x = in[i];
        m = fmin(m, isfinite(x) && x > 0 ? x : -1.0);
    }
    m = warpMin(m);
    if ((threadIdx.x & 31) == 0) warpValues[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? warpValues[threadIdx.x] : HUGE_VAL;
        m = warpMin(m);
        if (threadIdx.x == 0) out[blockIdx.x] = m;
    }
}

// Boundary ledger: sum over boundary faces of faceFlux(f,k), one block per
// variable, deterministic order (block-strided accumulation then tree).
__global__ void boundaryLedger(GraphView v, double* rate) {
    __shared__ double warpValues[32];
    const size_t k = blockIdx.x;
    double s = 0;
    for (size_t j = threadIdx.x; j < v.nBoundary; j += blockDim.x) {
        const size_t fi = size_t(v.boundary[j]);
        const ReactiveTransportFace f = v.face[fi];
        if (size_t(f.owner) < v.ownBegin || size_t(f.owner) >= v.ownEnd) continue;
        double wk[FW_FIELDS];
        for (int t = 0; t < FW_FIELDS; ++t) wk[t] = v.work[size_t(t) * v.faces + fi];
        const size_t r = rightCell(v, f);
        s += faceFluxK(v, f, fi, r, k, wk, v.carrier[fi], loadSgs(v, f, fi, r));
    }
    s = warpSum(s);
    if ((threadIdx.x & 31) == 0) warpValues[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? warpValues[threadIdx.x] : 0.0;
        s = warpSum(s);
        if (threadIdx.x == 0) rate[k] = s;
    }
}

// Input validation of the host-array entries on the device, after the upload:
// the first cell whose recovered state is not admissible (p, T, rho, sound, cv
// finite and positive, gas mass finite and non-negative, dilatation finite) to
// first[0]; the first invalid primitive to first[1] as 2 c (density not finite
// and positive) or 2 c + 1 (a velocity component not finite), so the density
// of a cell is reported before its velocity.
__global__ void validateUploads(const ReactiveTransportState* __restrict__ st,
                                const ReactiveTransportPrimitive* __restrict__ prim, size_t count,
                                unsigned long long* first) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        if (st) {
            const ReactiveTransportState s = st[c];
            const bool ok = isfinite(s.p) && s.p > 0 && isfinite(s.T) && s.T > 0 && isfinite(s.rho) && s.rho > 0
                && isfinite(s.sound) && s.sound > 0 && isfinite(s.cv) && s.cv > 0 && isfinite(s.gasMass)
                && s.gasMass >= 0 && isfinite(s.dilatation);
            if (!ok) atomicMin(first, (unsigned long long)c);
        }
        if (prim) {
            const ReactiveTransportPrimitive p = prim[c];
            if (!(isfinite(p.rho) && p.rho > 0)) atomicMin(first + 1, 2ull * c);
            else if (!(isfinite(p.u[0]) && isfinite(p.u[1]) && isfinite(p.u[2])))
                atomicMin(first + 1, 2ull * c + 1);
        }
    }
}

// Strided gather of the WALE scalar fields into the handle's arrays: cp of entry
// c to mixCp[offset + c], enthalpy k to spH[k * all + offset + c]. A cp that is
// not finite and positive or a non-finite enthalpy sets bit 2 of the status.
__global__ void gatherScalarFields(const double* __restrict__ cp, const double* __restrict__ h, size_t cpStride,
                                   size_t hStride, size_t count, size_t offset, size_t ns, size_t all,
                                   double* __restrict__ mixCp, double* __restrict__ spH, unsigned* status) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        bool bad = false;
        if (cp) {
            const double x = cp[c * cpStride];
            bad |= !(isfinite(x) && x > 0);
            mixCp[offset + c] = x;
        }
        if (h) {
            for (size_t k = 0; k < ns; ++k) {
                const double y = h[c * hStride + k];
                bad |= !isfinite(y);
                spH[k * all + offset + c] = y;
            }
        }
        if (bad) atomicOr(status, 4u);
    }
}

// Cell-major (c*width + k) <-> SoA (k*stride + offset + c) transposition used at
// the host boundary; the host ABI stays cell-major.
__global__ void packSoA(const double* __restrict__ in, double* __restrict__ out, size_t count,
                        size_t width, size_t stride, size_t offset) {
    const size_t n = count * width;
    for (size_t j = blockIdx.x * size_t(blockDim.x) + threadIdx.x; j < n; j += size_t(blockDim.x) * gridDim.x) {
        const size_t c = j / width, k = j % width;
        out[k * stride + offset + c] = in[j];
    }
}
__global__ void unpackSoA(const double* __restrict__ in, double* __restrict__ out, size_t count,
                          size_t width, size_t stride, size_t offset) {
    const size_t n = count * width;
    for (size_t j = blockIdx.x * size_t(blockDim.x) + threadIdx.x; j < n; j += size_t(blockDim.x) * gridDim.x) {
        const size_t c = j / width, k = j % width;
        out[j] = in[k * stride + offset + c];
    }
}

}  // namespace rb200
