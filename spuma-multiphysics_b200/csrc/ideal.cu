// Ideal-gas mixture closure on the device and its vector-Jacobian product.
//
// Recovery per cell follows the reference's scalar closure for pr = 0
// (src/reactiveTransport/reactiveClosureScalar.cuh:9-57): e(T) = h(T) - r T,
// cv(T) = cp(T) - r and p = rho r T from NASA polynomials; starting at the seed
// temperature, a bracket widened by doubling radii (at most 24) around the
// seed, then at most 70 Newton steps T - F/cv kept inside the bracket (else
// bisection), stopping when |F| <= .25 tol max(1e5, cp T). Here the mixture's
// h, cp and r are sums over the species' own NASA regions weighted by the mass
// fractions of the cell (the reference premixes the coefficients of one NASA
// interval on the host), and the frozen sound speed is c^2 = (cp/cv) r T.
#include "pr_eos.cuh"
#include "dual.cuh"
#include "common.cuh"
#include "../../include/reactive_b200_ideal.h"

#include <cmath>
#include <cstring>
#include <memory>
#include <string>

namespace rb200 {
namespace {

constexpr int kIdealMaxSpecies = 4;

struct IdealConst {
    int ns;
    double r[kIdealMaxSpecies];  // R / W_k, J/(kg K)
    PureSpecies sp[kIdealMaxSpecies];
    double Tmin, Tmax, tol;
};

// Mixture e(T), cv(T), r and d cv / dT at mass fractions Y.
__device__ inline void mixture(const IdealConst& G, const double* Y, double T, double& e, double& cv, double& r,
                               double* cvSlope) {
    e = cv = r = 0;
    double slope = 0;
    for (int k = 0; k < G.ns; ++k) {
        double cpR, hRT, sR;
        nasaEval(G.sp[k], T, cpR, hRT, sR);
        e += Y[k] * G.r[k] * T * (hRT - 1);
        cv += Y[k] * G.r[k] * (cpR - 1);
        r += Y[k] * G.r[k];
        if (cvSlope) {
            // d cp/R / dT of the region's polynomial
            const PureSpecies& s = G.sp[k];
            const double* a = s.coeff[nasaRegion(s, T)];
            const double iT = 1 / T;
            const double d = s.polynomial[nasaRegion(s, T)] == 7
                ? a[1] + 2 * a[2] * T + 3 * a[3] * T * T + 4 * a[4] * T * T * T
                : -2 * a[0] * iT * iT * iT - a[1] * iT * iT + a[3] + 2 * a[4] * T + 3 * a[5] * T * T
                      + 4 * a[6] * T * T * T;
            slope += Y[k] * G.r[k] * d;
        }
    }
    if (cvSlope) *cvSlope = slope;
}

__device__ inline bool inRange(const IdealConst& G, double T) { return T >= G.Tmin && T <= G.Tmax && T > 0; }

__global__ void idealClosure(const IdealConst* __restrict__ Gp, const double* __restrict__ q, size_t stride,
                             size_t count, const double* Tseed, double* Tout, ReactiveTransportState* transport,
                             int* success) {
    const IdealConst& G = *Gp;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        double rho = 0, Y[kIdealMaxSpecies];
        for (int k = 0; k < G.ns; ++k) rho += q[size_t(k) * stride + c];
        for (int k = 0; k < G.ns; ++k) Y[k] = q[size_t(k) * stride + c] / rho;
        const double mx = q[size_t(G.ns) * stride + c], my = q[size_t(G.ns + 1) * stride + c],
                     mz = q[size_t(G.ns + 2) * stride + c], E = q[size_t(G.ns + 3) * stride + c];
        const double eIn = (E - .5 * (mx * mx + my * my + mz * mz) / rho) / rho;
        const double T0 = Tseed[c];
        bool ok = isfinite(rho) && rho > 0 && isfinite(eIn) && inRange(G, T0);
        double T = T0, e = 0, cv = 0, r = 0;
        if (ok) {
            mixture(G, Y, T, e, cv, r, nullptr);
            const double tolerance = .25 * G.tol * fmax(1e5, (cv + r) * T);
            double lo = T, hi = T, fl = e - eIn, fh = fl, F = fl, radius = fmax(1., .01 * T);
            for (int j = 0; j < 24 && fabs(F) > tolerance && (fl > 0 || fh < 0); ++j, radius *= 2) {
                double ee, cc, rr;
                if (fl > 0) { lo = fmax(G.Tmin, T0 - radius); mixture(G, Y, lo, ee, cc, rr, nullptr); fl = ee - eIn; }
                if (fh < 0) { hi = fmin(G.Tmax, T0 + radius); mixture(G, Y, hi, ee, cc, rr, nullptr); fh = ee - eIn; }
            }
            ok = fabs(F) <= tolerance || (fl <= 0 && fh >= 0 && hi > lo);
            for (int it = 0; ok && it < 70 && fabs(F) > tolerance; ++it) {
                if (F > 0) hi = T; else lo = T;
                const double next = T - F / cv;
                T = isfinite(next) && next > lo && next < hi ? next : .5 * (lo + hi);
                mixture(G, Y, T, e, cv, r, nullptr);
                F = e - eIn;
            }
            ok = ok && fabs(F) <= tolerance && cv > 0;
        }
        if (success) success[c] = ok ? 1 : 0;
        if (!ok) continue;
        const double p = rho * r * T;
        const double sound = sqrt((cv + r) / cv * r * T);
        Tout[c] = T;
        transport[c] = ReactiveTransportState{p, T, rho, cv, sound, rho, 0.0};
    }
}

// d(state fields)/dq by forward-mode duals seeded on the cell's conserved
// variables; T's derivative by the implicit function theorem on
// f(T, q) = e(T, Y(q)) - e(q) = 0: dT/dq = -(df/dq) / cv.
template <int NS>
__global__ void idealClosureVjp(const IdealConst* __restrict__ Gp, const double* __restrict__ q, size_t stride,
                                size_t count, const double* __restrict__ Tconv,
                                const ReactiveTransportState* __restrict__ bar, double* qBar, size_t barStride) {
    constexpr int N = NS + 4;
    using D = Dual<N>;
    const IdealConst& G = *Gp;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        D qd[N];
#pragma unroll
        for (int k = 0; k < N; ++k) qd[k] = D::seed(q[size_t(k) * stride + c], k);
        D rho(0.0);
#pragma unroll
        for (int k = 0; k < NS; ++k) rho += qd[k];
        D Y[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) Y[k] = qd[k] / rho;
        const D m2 = qd[NS] * qd[NS] + qd[NS + 1] * qd[NS + 1] + qd[NS + 2] * qd[NS + 2];
        const D eIn = (qd[NS + 3] - D(.5) * m2 / rho) / rho;
        const double T = Tconv[c];
        // species terms at the converged T (constants), mixed with dual Y
        D e(0.0), cv(0.0), r(0.0);
        double cvSlope = 0, Yv[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) Yv[k] = Y[k].v;
        double ev, cvv, rv;
        mixture(G, Yv, T, ev, cvv, rv, &cvSlope);
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            double cpR, hRT, sR;
            nasaEval(G.sp[k], T, cpR, hRT, sR);
            e += Y[k] * D(G.r[k] * T * (hRT - 1));
            cv += Y[k] * D(G.r[k] * (cpR - 1));
            r += Y[k] * D(G.r[k]);
        }
        const D f = e - eIn;
        D Td(T);
#pragma unroll
        for (int i = 0; i < N; ++i) Td.d[i] = -f.d[i] / cvv;
        // cv also moves with T
#pragma unroll
        for (int i = 0; i < N; ++i) cv.d[i] += cvSlope * Td.d[i];
        const D p = rho * r * Td;
        const D sound = sqrt((cv + r) / cv * r * Td);
        const ReactiveTransportState b = bar[c];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const double g = b.p * p.d[k] + b.T * Td.d[k] + b.rho * rho.d[k] + b.cv * cv.d[k] + b.sound * sound.d[k]
                + b.gasMass * rho.d[k];
            qBar[size_t(k) * barStride + c] += g;
        }
    }
}

struct IdealDevice {
    int device = 0;
    IdealConst host{};
    IdealConst* dev = nullptr;
    ~IdealDevice() { if (dev) cudaFree(dev); }
};

std::string speciesFromTable(const ReactiveB200Species& s, PureSpecies& sp) {
    if (!(std::isfinite(s.molecularWeight) && s.molecularWeight > 0) || s.regionCount < 1
        || s.regionCount > kMaxRegions)
        return "Invalid ideal-gas species data";
    std::memset(&sp, 0, sizeof(sp));
    sp.W = s.molecularWeight;
    sp.regionCount = s.regionCount;
    for (int r = 0; r < s.regionCount; ++r) {
        const auto& g = s.regions[r];
        if ((g.polynomial != 7 && g.polynomial != 9) || !std::isfinite(g.minimumTemperature)
            || !std::isfinite(g.maximumTemperature) || g.minimumTemperature <= 0
            || g.maximumTemperature <= g.minimumTemperature
            || (r && g.minimumTemperature < s.regions[r - 1].minimumTemperature))
            return "Invalid ideal-gas NASA region";
        for (int j = 0; j < g.polynomial; ++j)
            if (!std::isfinite(g.coefficient[j])) return "Invalid ideal-gas NASA coefficient";
        sp.polynomial[r] = g.polynomial;
        sp.regionMin[r] = g.minimumTemperature;
        for (int j = 0; j < 9; ++j) sp.coeff[r][j] = g.coefficient[j];
    }
    sp.regionMaxLast = s.regions[s.regionCount - 1].maximumTemperature;
    return "";
}

void fail(char* error, size_t size, const char* what) {
    if (error && size) std::snprintf(error, size, "%s", what);
}

}  // namespace
}  // namespace rb200

extern "C" {

void* reactive_ideal_gas_create_v3(const void* table, size_t bytes, double Tmin, double Tmax, double tolerance,
                                   char* error, size_t size) {
    using namespace rb200;
    try {
        require(table && bytes == sizeof(ReactiveB200Table), "Invalid ideal-gas table image");
        ReactiveB200Table t;
        std::memcpy(&t, table, sizeof(t));
        require(t.ns >= 1 && t.ns <= kIdealMaxSpecies, "Ideal-gas closure supports 1 to 4 species");
        require(std::isfinite(Tmin) && std::isfinite(Tmax) && Tmin > 0 && Tmax > Tmin, "Invalid temperature range");
        require(std::isfinite(tolerance) && tolerance > 0 && tolerance < 1, "Invalid closure tolerance");
        std::unique_ptr<IdealDevice> d(new IdealDevice);
        d->host.ns = t.ns;
        d->host.Tmin = Tmin;
        d->host.Tmax = Tmax;
        d->host.tol = tolerance;
        for (int k = 0; k < t.ns; ++k) {
            const std::string why = speciesFromTable(t.species[k], d->host.sp[k]);
            require(why.empty(), why.c_str());
            require(Tmin >= t.species[k].regions[0].minimumTemperature
                        && Tmax <= d->host.sp[k].regionMaxLast,
                    "Temperature range outside a species' NASA regions");
            d->host.r[k] = kGas / t.species[k].molecularWeight;
        }
        check(cudaGetDevice(&d->device), "cudaGetDevice");
        check(cudaMalloc(&d->dev, sizeof(IdealConst)), "cudaMalloc");
        check(cudaMemcpy(d->dev, &d->host, sizeof(IdealConst), cudaMemcpyHostToDevice), "H2D");
        return d.release();
    } catch (const std::exception& e) {
        fail(error, size, e.what());
        return nullptr;
    }
}

void reactive_ideal_gas_destroy_v3(void* gas) { delete static_cast<rb200::IdealDevice*>(gas); }

int reactive_ideal_gas_run_device_v3(void* gas, const double* q, size_t stride, size_t count, size_t variables,
                                     const double* Tseed, double* T, ReactiveTransportState* transport, int* success,
                                     void* stream, char* error, size_t size) {
    using namespace rb200;
    try {
        require(gas && q && Tseed && T && transport && count && stride >= count, "Invalid ideal-gas arguments");
        auto& d = *static_cast<IdealDevice*>(gas);
        require(variables == size_t(d.host.ns) + 4, "Ideal-gas closure needs variables = species + 4");
        idealClosure<<<gridFor(count, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(d.dev, q, stride, count,
                                                                                        Tseed, T, transport, success);
        check(cudaGetLastError(), "idealClosure");
        return 0;
    } catch (const std::exception& e) {
        fail(error, size, e.what());
        return 1;
    }
}

int reactive_ideal_gas_vjp_device_v3(void* gas, const double* q, size_t stride, size_t count, size_t variables,
                                     const double* T, const ReactiveTransportState* bar, double* qBar,
                                     size_t barStride, void* stream, char* error, size_t size) {
    using namespace rb200;
    try {
        require(gas && q && T && bar && qBar && count && stride >= count && barStride >= count,
                "Invalid ideal-gas VJP arguments");
        auto& d = *static_cast<IdealDevice*>(gas);
        require(variables == size_t(d.host.ns) + 4, "Ideal-gas closure needs variables = species + 4");
        auto s = static_cast<cudaStream_t>(stream);
        const unsigned grid = gridFor(count, 128);
        switch (d.host.ns) {
        case 1: idealClosureVjp<1><<<grid, 128, 0, s>>>(d.dev, q, stride, count, T, bar, qBar, barStride); break;
        case 2: idealClosureVjp<2><<<grid, 128, 0, s>>>(d.dev, q, stride, count, T, bar, qBar, barStride); break;
        case 3: idealClosureVjp<3><<<grid, 128, 0, s>>>(d.dev, q, stride, count, T, bar, qBar, barStride); break;
        default: idealClosureVjp<4><<<grid, 128, 0, s>>>(d.dev, q, stride, count, T, bar, qBar, barStride); break;
        }
        check(cudaGetLastError(), "idealClosureVjp");
        return 0;
    } catch (const std::exception& e) {
        fail(error, size, e.what());
        return 1;
    }
}

}  // extern "C"
