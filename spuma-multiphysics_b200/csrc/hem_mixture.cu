// Multi-species HEM UV flash on the device: a Peng-Robinson gas mixture of up
// to four species with up to two pure condensed liquids (the air / N2O /
// isopropanol model of the reference's production case), one thread per cell.
//
// The search restates the reference device flash
// (src/reactiveThermo/reactiveDeviceFlash.h) for models without solids, with its
// bounded finite-difference Newton Jacobian (an image's analyticJacobian flag
// selects the reference's analytic active-set Jacobian there, which is not
// restated: such images run on the finite differences and converge to the same
// solutions within the Newton tolerances), including its capillary form
// (recoverCapillary, :572-588: the phases at their own pressures across a fixed
// jump, the boundary search in every equilibrium batch, the frozen partition):
//   * phase sums of one evaluation at (p, T) with given liquid masses, the gas
//     phase from the remaining species and, on request, virtual liquids for the
//     chemical potentials (evaluate, :210-262);
//   * the all-gas partition: the scalar T-Newton at fixed density, else the
//     frozen (ln p, ln T) Newton with its halving line search (:264-326);
//   * the active-set Newton in (ln p, ln T, liquid fractions) or, in the
//     boundary recovery, (ln p, ln T, log vapour fractions), with the residual of
//     the volume, the scaled energy and each active liquid's chemical-potential
//     difference, the bounded central-difference Jacobian, the limiter, the
//     30-fraction line search with its coordinate rejection prefix, and the
//     equilibrium sound check (:327-448);
//   * the stability test: affinities against virtual liquids when gas is
//     present, the tangent plane of the liquid species otherwise (a 33-point scan
//     and 55 golden-section steps for two liquids) (:449-480);
//   * the candidate order, the seeds {previous, .5, .95, .1, .9999}, the first
//     maximum entropy among stable candidates, the restart temperatures at
//     {.02, .25, .5, .75} of the legal liquid interval, the optional
//     stableGasPrune policy, and the boundary recovery around nearly liquid cells
//     (:486-560, src/reactiveThermo/reactiveFlashSeeds.h:14-16).
// Phase properties come from the mixture evaluator of pr_mixture.cuh (pinned to
// the reference's evaluator). Every loop is bounded.
#include "hem_mixture.h"
#include "pr_mixture.cuh"
#include "common.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

namespace rb200 {
namespace {

constexpr double kRu = 8314.46261815324;
constexpr int kNs = mix::kMaxNs;
constexpr int kLiq = 2;
constexpr int kBlock = 64;

// Phase sums of one evaluation (the state plus the derivatives the Newton
// iterations and the stability test use).
struct MixEval {
    ReactiveThermoState s;
    double volume, energy, entropyD, Vp, VT, Ep, ET, cpD;
    double muGas[kLiq], muLiq[kLiq], gasCond[kLiq];
    bool explicitGas;
};

struct Tally {
    unsigned long long phases = 0, residuals = 0, candidates = 0, stable = 0, failures = 0, fd = 0;
};

// One cell's recovery: its inputs, the search mode and, for a capillary batch,
// the interface color and the pressure jump sigma*kappa held fixed during the
// solve (src/reactiveThermo/reactiveDeviceFlash.h:146-153): the gas phase is
// evaluated at p - color*jump and the liquids at p + (1 - color)*jump, p the
// volume-averaged mechanical pressure.
struct MixCell {
    const ReactiveB200HemModel& m;
    double q[kNs];
    double energy;
    ReactiveThermoState guess;
    bool adaptive;
    Tally& n;
    double color = 0, jump = 0;
};

__device__ __forceinline__ bool fin(double x) { return x == x && fabs(x) <= 1.79769313486231570815e308; }
__device__ __forceinline__ double clampd(double a, double l, double h) { return fmin(fmax(a, l), h); }
__device__ __forceinline__ double maxAbs(const double* a, int n) {
    double r = 0;
    for (int i = 0; i < n; ++i) r = fmax(r, fabs(a[i]));
    return r;
}
__device__ __forceinline__ bool unavailable(int status) { return status == mix::UNAVAILABLE || status == mix::NO_ROOT; }

__device__ __forceinline__ double density(const MixCell& c) {
    double r = 0;
    for (int k = 0; k < c.m.ns; ++k) r += c.q[k];
    return r;
}
__device__ __forceinline__ bool inBounds(const ReactiveB200HemModel& m, double p, double T) {
    return fin(p) && fin(T) && p >= m.pmin && p <= m.pmax && T >= m.Tmin && T <= m.Tmax;
}
__device__ __forceinline__ bool isCondensable(const ReactiveB200HemModel& m, int k) {
    for (int i = 0; i < m.nl; ++i)
        if (m.condensable[i] == k) return true;
    return false;
}
__device__ __forceinline__ double energyScale(const MixEval& v) { return fmax(1e5 * v.s.rho, v.cpD * v.s.T); }
__device__ __forceinline__ double gasPressure(const MixCell& c, double p) { return p - c.color * c.jump; }
__device__ __forceinline__ double liquidPressure(const MixCell& c, double p) { return p + (1 - c.color) * c.jump; }

// The gas mixture at (p, T, Y) on its gas root; species outside their NASA
// range invalidate the state when the model enforces the ranges.
__device__ __noinline__ int gasPhase(MixCell& c, double p, double T, const double* Y, bool chem, mix::Props& out) {
    ++c.n.phases;
    if (!inBounds(c.m, p, T)) return mix::BAD_INPUT;
    if (c.m.enforceSpeciesTemperatureBounds)
        for (int k = 0; k < c.m.ns; ++k)
            if (Y[k] > 0) {
                const ReactiveB200Species& sp = c.m.phase[0].species[k];
                if (T < sp.regions[0].minimumTemperature || T > sp.regions[sp.regionCount - 1].maximumTemperature)
                    return mix::BAD_INPUT;
            }
    return mix::tp(c.m.phase[0], T, p, Y, mix::GAS, chem, out);
}

// The pure liquid of condensed phase i at (p, T) on its liquid root.
__device__ __noinline__ int liquidPhase(MixCell& c, int i, double p, double T, bool chem, mix::Props& out) {
    ++c.n.phases;
    if (!inBounds(c.m, p, T)) return mix::BAD_INPUT;
    if (T < c.m.liquidTmin[i]) return mix::BAD_INPUT;
    if (T >= c.m.liquidTc[i] * (1 - 1e-10)) return mix::UNAVAILABLE;
    const double pure[kNs] = {1, 0, 0, 0};
    return mix::tp(c.m.phase[i + 1], T, p, pure, mix::LIQUID, chem, out);
}

__device__ __forceinline__ void addPhase(MixEval& v, double mass, const mix::Props& p, double pressure) {
    const double volume = mass / p.rho, vp = -volume * p.kappaT, vt = volume * p.alpha;
    v.volume += volume;
    v.energy += mass * p.e;
    v.entropyD += mass * p.s;
    v.Vp += vp;
    v.VT += vt;
    v.Ep += -v.s.T * vt - pressure * vp;
    v.ET += mass * p.cp - pressure * vt;
    v.cpD += mass * p.cp;
}

// Phase sums at (p, T) with liquid masses `mass`; `vapor` (the boundary
// recovery) gives each condensable's gas amount explicitly; `virt` also
// evaluates absent liquids for the chemical potentials.
__device__ __noinline__ bool evaluate(MixCell& c, const double* mass, double p, double T, MixEval& v, bool virt,
                                      const double* vapor) {
    const ReactiveB200HemModel& m = c.m;
    v = MixEval{};
    if (!inBounds(m, p, T)) return false;
    ReactiveThermoState& s = v.s;
    s.p = p;
    s.T = T;
    s.rho = density(c);
    if (!(s.rho > 0)) return false;
    double gas[kNs] = {0, 0, 0, 0};
    for (int k = 0; k < m.ns; ++k) {
        if (!fin(c.q[k]) || c.q[k] < 0) return false;
        gas[k] = c.q[k];
    }
    for (int i = 0; i < m.nl; ++i) {
        const int k = m.condensable[i];
        if (!fin(mass[i]) || mass[i] < 0 || mass[i] > c.q[k]) return false;
        gas[k] = vapor ? vapor[i] : gas[k] - mass[i];
        if (!fin(gas[k]) || gas[k] < 0 || gas[k] > c.q[k]) return false;
    }
    for (int i = 0; i < m.nl; ++i) v.gasCond[i] = gas[m.condensable[i]];
    v.explicitGas = vapor != nullptr;
    double mg = 0;
    for (int k = 0; k < m.ns; ++k) mg += gas[k];
    s.gasMass = mg;
    const double pg = gasPressure(c, p), pl = liquidPressure(c, p);
    if (mg > 0) {
        for (int k = 0; k < m.ns; ++k) gas[k] /= mg;
        mix::Props prop;
        if (gasPhase(c, pg, T, gas, virt, prop) != mix::OK) return false;
        addPhase(v, mg, prop, pg);
        s.alphaGas = mg / prop.rho;
        s.rhoGas = prop.rho;
        if (virt)
            for (int i = 0; i < m.nl; ++i) v.muGas[i] = prop.mu[m.condensable[i]] / (kRu * T);
    }
    for (int i = 0; i < m.nl; ++i) {
        s.liquidMass[i] = mass[i];
        if (!(mass[i] > 0 || (virt && c.q[m.condensable[i]] > 0))) continue;
        mix::Props prop;
        const int status = liquidPhase(c, i, pl, T, virt, prop);
        if (status != mix::OK) {
            if (mass[i] > 0 || !unavailable(status)) return false;
            v.muLiq[i] = HUGE_VAL;
            continue;
        }
        if (virt) v.muLiq[i] = prop.mu[0] / (kRu * T);
        if (mass[i] > 0) {
            addPhase(v, mass[i], prop, pl);
            s.rhoLiquid[i] = prop.rho;
            s.alphaLiquid[i] = mass[i] / prop.rho;
            s.activeLiquids |= 1 << i;
        }
    }
    s.e = v.energy / s.rho;
    s.entropy = v.entropyD / s.rho;
    s.cp = v.cpD / s.rho;
    s.cv = (v.cpD + T * v.VT * v.VT / v.Vp) / s.rho;
    if (!fin(s.cv) || s.cv <= 0) return false;
    const double specific = v.volume / s.rho, vp = v.Vp / s.rho, vt = v.VT / s.rho;
    const double adiabatic = vp + T * vt * vt / s.cp;
    if (!(adiabatic < 0)) return false;
    s.soundFrozen = sqrt(-specific * specific / adiabatic);
    s.soundEquilibrium = s.soundFrozen;
    return fin(s.soundFrozen) && s.soundFrozen > 0;
}

// Dense solve with full pivoting (pivot search column by column, rows inside
// each column, first strict maximum) and the rank test pivot > largest * n * eps.
__device__ bool solveDense(const double a0[4][4], const double* rhs, int n, double* x) {
    double a[4][4], b[4], largest = 0;
    int column[4] = {0, 1, 2, 3};
    for (int i = 0; i < n; ++i) {
        b[i] = rhs[i];
        if (!fin(b[i])) return false;
        for (int j = 0; j < n; ++j) {
            a[i][j] = a0[i][j];
            if (!fin(a[i][j])) return false;
        }
    }
    for (int k = 0; k < n; ++k) {
        int row = k, col = k;
        double pivot = 0;
        for (int j = k; j < n; ++j)
            for (int i = k; i < n; ++i)
                if (fabs(a[i][j]) > pivot) { pivot = fabs(a[i][j]); row = i; col = j; }
        largest = fmax(largest, pivot);
        if (!(pivot > largest * n * 2.220446049250313e-16)) return false;
        if (row != k) {
            for (int j = 0; j < n; ++j) { const double t = a[k][j]; a[k][j] = a[row][j]; a[row][j] = t; }
            const double t = b[k]; b[k] = b[row]; b[row] = t;
        }
        if (col != k) {
            for (int i = 0; i < n; ++i) { const double t = a[i][k]; a[i][k] = a[i][col]; a[i][col] = t; }
            const int t = column[k]; column[k] = column[col]; column[col] = t;
        }
        for (int i = k + 1; i < n; ++i) {
            const double f = a[i][k] / a[k][k];
            a[i][k] = f;
            for (int j = k + 1; j < n; ++j) a[i][j] -= f * a[k][j];
            b[i] -= f * b[k];
        }
    }
    double z[4] = {0, 0, 0, 0};
    for (int i = n - 1; i >= 0; --i) {
        double v = b[i];
        for (int j = i + 1; j < n; ++j) v -= a[i][j] * z[j];
        z[i] = v / a[i][i];
        if (!fin(z[i])) return false;
    }
    for (int i = 0; i < n; ++i) x[column[i]] = z[i];
    return true;
}

// The scalar all-gas energy residual at (T, rho): properties at (T, rho), then
// the gas root at the resulting pressure must be that density. p is the
// mechanical pressure, the gas's plus color*jump.
__device__ __noinline__ bool gasProbe(MixCell& c, double T, double& F, double& cv, double& p, double* cp) {
    const double rho = density(c);
    double Y[kNs] = {0, 0, 0, 0};
    for (int k = 0; k < c.m.ns; ++k) Y[k] = c.q[k] / rho;
    ++c.n.phases;
    mix::Props prop;
    if (mix::trho(c.m.phase[0], T, rho, Y, false, prop) != mix::OK) return false;
    const double gasP = prop.p;
    p = gasP + c.color * c.jump;
    if (!inBounds(c.m, p, T)) return false;
    mix::Props gas;
    if (gasPhase(c, gasP, T, Y, false, gas) != mix::OK || fabs(gas.rho - rho) > 1e-8 * rho) return false;
    F = rho * prop.e - c.energy;
    cv = rho * prop.cv;
    if (cp) *cp = prop.cp;
    return fin(F) && fin(cv) && cv > 0;
}

__device__ __noinline__ bool scalarGas(MixCell& c, MixEval& result) {
    const ReactiveB200HemModel& m = c.m;
    const double rho = density(c);
    double T = clampd(c.guess.T, m.Tmin, m.Tmax), F, cv, p, cp;
    if (!gasProbe(c, T, F, cv, p, &cp)) return false;
    const double tol = m.etol * fmax(1e5 * rho, rho * cp * T);
    double lower = T, upper = T, fl = F, fh = F;
    if (fabs(F) > tol) {
        double radius = fmax(1., .01 * T);
        for (int j = 0; j < 24 && (fl > 0 || fh < 0); ++j, radius *= 2) {
            if (fl > 0) {
                double probe = fmax(m.Tmin, T - radius), value, dCv, dP;
                bool found = false;
                for (int retry = 0; retry < 8 && !found; ++retry) {
                    if (gasProbe(c, probe, value, dCv, dP, nullptr)) { fl = value; lower = probe; found = true; }
                    else probe = .5 * (lower + probe);
                }
                if (!found) return false;
            }
            if (fh < 0) {
                double probe = fmin(m.Tmax, T + radius), value, dCv, dP;
                bool found = false;
                for (int retry = 0; retry < 8 && !found; ++retry) {
                    if (gasProbe(c, probe, value, dCv, dP, nullptr)) { fh = value; upper = probe; found = true; }
                    else probe = .5 * (upper + probe);
                }
                if (!found) return false;
            }
            if (fabs(fl) <= tol) { T = lower; if (!gasProbe(c, T, F, cv, p, nullptr)) return false; break; }
            if (fabs(fh) <= tol) { T = upper; if (!gasProbe(c, T, F, cv, p, nullptr)) return false; break; }
            if (lower == m.Tmin && upper == m.Tmax) break;
        }
        if (!(fabs(F) <= tol || (fl <= 0 && fh >= 0 && upper > lower))) return false;
    }
    int it = 0;
    for (; it < 70 && fabs(F) > tol; ++it) {
        if (F > 0) upper = T; else lower = T;
        const double next = T - F / cv;
        T = fin(next) && next > lower && next < upper ? next : .5 * (lower + upper);
        if (!gasProbe(c, T, F, cv, p, nullptr)) return false;
    }
    if (fabs(F) > tol) return false;
    const double zero[kLiq] = {0, 0};
    if (!evaluate(c, zero, p, T, result, false, nullptr)) return false;
    result.s.volumeResidual = fabs(result.volume - 1);
    result.s.energyResidual = fabs(result.energy - c.energy) / energyScale(result);
    result.s.iterations = it;
    return result.s.volumeResidual <= m.vtol && result.s.energyResidual <= m.etol;
}

// A frozen partition (fixed liquid masses): Newton in (ln p, ln T) with the
// (0.7, 0.2) limiter and a halving line search; stallLimit > 0 ends the solve as
// a failure after that many consecutive steps accepted below a fraction of 1/32.
__device__ __noinline__ bool frozen(MixCell& c, const double* mass, MixEval& value, int stallLimit) {
    const ReactiveB200HemModel& m = c.m;
    if (!fin(c.energy)) return false;
    if (m.scalarRecovery && mass[0] == 0 && mass[1] == 0 && scalarGas(c, value)) return true;
    double p = clampd(c.guess.p, m.pmin, m.pmax), T = clampd(c.guess.T, m.Tmin, m.Tmax);
    if (!evaluate(c, mass, p, T, value, false, nullptr)) return false;
    int stalled = 0;
    for (int it = 0; it < 70; ++it) {
        const double scale = energyScale(value), rv = value.volume - 1, re = (value.energy - c.energy) / scale;
        value.s.volumeResidual = fabs(rv);
        value.s.energyResidual = fabs(re);
        value.s.iterations = it;
        if (fabs(rv) <= m.vtol && fabs(re) <= m.etol) return true;
        double jac[4][4] = {}, rhs[4] = {-rv, -re, 0, 0}, step[4] = {};
        jac[0][0] = value.Vp * p; jac[0][1] = value.VT * T;
        jac[1][0] = value.Ep * p / scale; jac[1][1] = value.ET * T / scale;
        if (!solveDense(jac, rhs, 2, step)) return false;
        const double limit = fmax(1., fmax(fabs(step[0]) / .7, fabs(step[1]) / .2));
        step[0] /= limit;
        step[1] /= limit;
        const double previous = fmax(fabs(rv), fabs(re));
        bool accepted = false;
        for (double fraction = 1; fraction > 1e-9; fraction *= .5) {
            const double pp = p * exp(fraction * step[0]), tt = T * exp(fraction * step[1]);
            MixEval trial;
            if (evaluate(c, mass, pp, tt, trial, false, nullptr)) {
                const double next = fmax(fabs(trial.volume - 1), fabs(trial.energy - c.energy) / scale);
                if (next < previous * (1 - 1e-4 * fraction) || next < fmin(m.vtol, m.etol)) {
                    value = trial;
                    p = pp;
                    T = tt;
                    accepted = true;
                    stalled = fraction < 1. / 32 ? stalled + 1 : 0;
                    break;
                }
            }
        }
        if (!accepted) return false;
        if (stallLimit > 0 && stalled >= stallLimit
            && !(fabs(value.volume - 1) <= m.vtol && fabs(value.energy - c.energy) / energyScale(value) <= m.etol))
            return false;
    }
    return false;
}

// Residual of an active set at x = (ln p, ln T, fractions): liquid fractions in
// [0, 1) or, in the boundary recovery, log vapour fractions <= 0.
__device__ __noinline__ bool activeResidual(MixCell& c, const int* active, int n, const double* x, double scale,
                                            double* f, MixEval* out) {
    ++c.n.residuals;
    const ReactiveB200HemModel& m = c.m;
    double mass[kLiq] = {0, 0}, vapor[kLiq] = {0, 0};
    for (int i = 0; i < m.nl; ++i) vapor[i] = c.q[m.condensable[i]];
    for (int j = 0; j < n; ++j) {
        const int i = active[j];
        const double q = c.q[m.condensable[i]];
        if (c.adaptive) {
            if (!fin(x[j + 2]) || x[j + 2] > 0) return false;
            vapor[i] = exp(x[j + 2]) * q;
            if (!(vapor[i] > 0)) return false;
            mass[i] = -expm1(x[j + 2]) * q;
        } else {
            if (!(x[j + 2] >= 0 && x[j + 2] < 1)) return false;
            mass[i] = x[j + 2] * q;
        }
    }
    MixEval v;
    if (!evaluate(c, mass, exp(x[0]), exp(x[1]), v, true, c.adaptive ? vapor : nullptr) || !(v.s.gasMass > 0))
        return false;
    f[0] = v.volume - 1;
    f[1] = (v.energy - c.energy) / scale;
    for (int j = 0; j < n; ++j) {
        f[2 + j] = v.muLiq[active[j]] - v.muGas[active[j]];
        if (!fin(f[2 + j])) return false;
    }
    if (out) *out = v;
    return true;
}

// Bounded central differences (h = 2e-6 in ln p and ln T, 2e-5 in the
// fractions, halved up to 12 times when neither side evaluates; one-sided when
// only one does; the boundary recovery's coordinates step at least one ulp and
// weight the two sides by their actual steps).
__device__ __noinline__ bool jacobianFD(MixCell& c, const int* active, int n, const double* x, double scale,
                                        const double* f, double jac[4][4]) {
    ++c.n.fd;
    const int size = n + 2;
    for (int j = 0; j < size; ++j) {
        double h = j < 2 ? 2e-6 : 2e-5;
        bool success = false;
        for (int attempt = 0; attempt < 12 && !success; ++attempt, h *= .5) {
            double xp[4] = {}, xm[4] = {}, fp[4] = {}, fm[4] = {};
            for (int i = 0; i < size; ++i) xp[i] = xm[i] = x[i];
            xp[j] += h;
            xm[j] -= h;
            if (c.adaptive) {
                if (xp[j] == x[j]) xp[j] = nextafter(x[j], HUGE_VAL);
                if (xm[j] == x[j]) xm[j] = nextafter(x[j], -HUGE_VAL);
            }
            const bool plus = activeResidual(c, active, n, xp, scale, fp, nullptr);
            const bool minus = activeResidual(c, active, n, xm, scale, fm, nullptr);
            if (!plus && !minus) continue;
            const double hp = xp[j] - x[j], hm = x[j] - xm[j];
            double maximum = 0;
            success = true;
            for (int i = 0; i < size; ++i) {
                double d;
                if (c.adaptive)
                    d = plus && minus ? (hm / (hp + hm)) * ((fp[i] - f[i]) / hp) + (hp / (hp + hm)) * ((f[i] - fm[i]) / hm)
                                      : plus ? (fp[i] - f[i]) / hp : (f[i] - fm[i]) / hm;
                else
                    d = plus && minus ? (fp[i] - fm[i]) / (2 * h) : plus ? (fp[i] - f[i]) / h : (f[i] - fm[i]) / h;
                jac[i][j] = d;
                maximum = fmax(maximum, fabs(d));
                success = success && fin(d);
            }
            if (c.adaptive) success = success && maximum > 0;
        }
        if (!success) return false;
    }
    return true;
}

__device__ __forceinline__ bool rejectedCoordinate(bool adaptive, double y) {
    return adaptive ? (!fin(y) || y > 0) : !(y >= 0 && y < 1);
}

// Newton on an active set of liquids from a fraction seed (seed < 0: the seed
// state's liquid fraction; -3 in the boundary recovery: a vapour fraction from
// the non-condensable inventory); secondSeed (when not -2) seeds the second
// liquid; restart (optional) replaces the seed state.
__device__ __noinline__ bool activeFlash(MixCell& c, const int* active, int n, double seed, MixEval& value,
                                         double secondSeed, const ReactiveThermoState* restart) {
    ++c.n.candidates;
    const ReactiveB200HemModel& m = c.m;
    const int size = n + 2;
    const double rho = density(c);
    const ReactiveThermoState& g = restart ? *restart : c.guess;
    const double scale = fmax(1e5 * rho, fmax(fabs(c.energy), rho * 2000 * fmax(g.T, m.Tmin)));
    double x[4] = {log(clampd(g.p, m.pmin, m.pmax)), log(clampd(g.T, m.Tmin, m.Tmax)), 0, 0};
    for (int j = 0; j < n; ++j) {
        const int i = active[j];
        const double selected = j == 1 && secondSeed != -2 ? secondSeed : seed;
        const double previous = g.liquidMass[i] / c.q[m.condensable[i]];
        x[j + 2] = selected < 0 ? clampd(previous, 1e-8, 1 - 1e-8) : selected;
        if (c.adaptive) {
            double vapor = selected < 0 ? 1 - previous : 1 - selected;
            if (selected == -3 || (selected < 0 && vapor < 1e-6)) {
                double other = 0;
                for (int k = 0; k < m.ns; ++k) {
                    bool chosen = false;
                    for (int a = 0; a < n; ++a) chosen |= k == m.condensable[active[a]];
                    if (!chosen) other += c.q[k];
                }
                vapor = other > 0 ? fmin(1e-6, .01 * (other / c.q[m.condensable[i]])) : 1e-8;
            }
            if (!(vapor > 0 && fin(vapor))) return false;
            x[j + 2] = log(fmin(1., vapor));
        }
    }
    double f[4] = {};
    if (!activeResidual(c, active, n, x, scale, f, &value)) return false;
    for (int it = 0; it < 90; ++it) {
        const double chemical = maxAbs(f + 2, n);
        double jac[4][4] = {};
        if (fabs(f[0]) <= m.vtol && fabs(f[1]) <= m.etol && chemical <= m.mutol) {
            value.s.volumeResidual = fabs(f[0]);
            value.s.energyResidual = fabs(f[1]);
            value.s.chemicalResidual = chemical;
            value.s.iterations = it;
            if (!jacobianFD(c, active, n, x, scale, f, jac)) return false;
            const double rhs[4] = {-1 / rho, value.s.p / (rho * scale), 0, 0};
            double response[4] = {};
            if (!solveDense(jac, rhs, size, response)) return false;
            const double squared = value.s.p * response[0];
            if (!fin(squared) || squared <= 0) return false;
            value.s.soundEquilibrium = sqrt(squared);
            return value.s.soundEquilibrium <= value.s.soundFrozen * (1 + 2e-3);
        }
        if (!jacobianFD(c, active, n, x, scale, f, jac)) return false;
        double rhs[4] = {}, step[4] = {};
        for (int j = 0; j < size; ++j) rhs[j] = -f[j];
        if (!solveDense(jac, rhs, size, step)) return false;
        double limiter = fmax(1., fmax(fabs(step[0]) / .7, fabs(step[1]) / .18));
        for (int j = 2; j < size; ++j) limiter = fmax(limiter, fabs(step[j]) / (c.adaptive ? 2. : .3));
        for (int j = 0; j < size; ++j) step[j] /= limiter;
        bool accepted = false;
        const double previous = maxAbs(f, size);
        double fraction = 1;
        for (int k = 0; k < 30; ++k, fraction *= .5) {
            double tx[4] = {}, tf[4] = {};
            for (int j = 0; j < size; ++j) tx[j] = x[j] + fraction * step[j];
            bool rejected = false;
            for (int j = 0; j < n; ++j) rejected |= rejectedCoordinate(c.adaptive, tx[j + 2]);
            if (rejected) {
                // the rejected fractions form a prefix (each coordinate moves back
                // toward the valid x as the fraction halves): its end by bisection
                // on the same expression and predicate, 30 standing for none
                int lower = k, upper = 30;
                while (upper - lower > 1) {
                    const int mid = (lower + upper) / 2;
                    const double fm = ldexp(1.0, -mid);
                    bool bad = false;
                    for (int j = 0; j < n; ++j) bad |= rejectedCoordinate(c.adaptive, x[j + 2] + fm * step[j + 2]);
                    if (bad) lower = mid; else upper = mid;
                }
                c.n.residuals += unsigned(upper - k);
                if (upper == 30) break;
                k = upper;
                fraction = ldexp(1.0, -upper);
                for (int j = 0; j < size; ++j) tx[j] = x[j] + fraction * step[j];
            }
            MixEval trial;
            if (activeResidual(c, active, n, tx, scale, tf, &trial) && maxAbs(tf, size) < previous * (1 - 1e-4 * fraction)) {
                for (int j = 0; j < size; ++j) { x[j] = tx[j]; f[j] = tf[j]; }
                value = trial;
                accepted = true;
                break;
            }
        }
        if (!accepted) return false;
    }
    return false;
}

// Gibbs energy of the gas mixture of the present liquids' species at mole
// fractions (fraction, 1 - fraction), less the liquids' chemical potentials:
// the tangent-plane distance (HUGE_VAL where the gas phase does not exist).
__device__ __noinline__ double tangent(MixCell& c, double p, double T, const int* present, int n, const double* mu,
                                       double fraction) {
    const ReactiveB200HemModel& m = c.m;
    double mole[kNs] = {0, 0, 0, 0}, Y[kNs] = {0, 0, 0, 0}, sum = 0;
    mole[m.condensable[present[0]]] = n == 1 ? 1 : fraction;
    if (n == 2) mole[m.condensable[present[1]]] = 1 - fraction;
    for (int k = 0; k < m.ns; ++k) { Y[k] = mole[k] * m.weights[k]; sum += Y[k]; }
    for (int k = 0; k < m.ns; ++k) Y[k] /= sum;
    mix::Props prop;
    const int status = gasPhase(c, gasPressure(c, p), T, Y, false, prop);
    if (status != mix::OK) return unavailable(status) ? HUGE_VAL : nan("");
    double reference = 0, W = 0;
    for (int i = 0; i < n; ++i) reference += mole[m.condensable[present[i]]] * mu[present[i]];
    for (int k = 0; k < m.ns; ++k) W += mole[k] * m.weights[k];
    return (prop.h - T * prop.s) * W / (kRu * T) - reference;
}

__device__ __noinline__ bool stableCandidate(MixCell& c, const MixEval& v) {
    const ReactiveB200HemModel& m = c.m;
    const double p = v.s.p, T = v.s.T;
    if (v.s.gasMass > 0) {
        const double mass[kLiq] = {v.s.liquidMass[0], v.s.liquidMass[1]};
        MixEval cmp;
        if (!evaluate(c, mass, p, T, cmp, true, v.explicitGas ? v.gasCond : nullptr)) return false;
        for (int i = 0; i < m.nl; ++i) {
            if (c.q[m.condensable[i]] == 0) continue;
            const double affinity = cmp.muLiq[i] - cmp.muGas[i];
            if (mass[i] > 0) {
                if (!fin(affinity) || fabs(affinity) > m.mutol * 2) return false;
            } else if (affinity < -m.mutol) return false;
        }
        return true;
    }
    int present[kLiq] = {0, 0}, np = 0;
    double mu[kLiq] = {0, 0};
    for (int i = 0; i < m.nl; ++i)
        if (v.s.liquidMass[i] > 0) {
            present[np++] = i;
            mix::Props prop;
            if (liquidPhase(c, i, liquidPressure(c, p), T, true, prop) != mix::OK) return false;
            mu[i] = prop.mu[0] / (kRu * T);
        }
    if (!np) return false;
    if (np == 1) return tangent(c, p, T, present, 1, mu, 1) >= -m.mutol;
    double best = HUGE_VAL;
    int location = 0;
    for (int j = 0; j <= 32; ++j) {
        const double t = tangent(c, p, T, present, np, mu, double(j) / 32);
        if (t != t) return false;
        if (t < best) { best = t; location = j; }
    }
    double left = fmax(0., double(location - 1) / 32), right = fmin(1., double(location + 1) / 32);
    for (int j = 0; j < 55; ++j) {
        const double a = left + (right - left) * .38196601125, b = left + (right - left) * .61803398875;
        const double ta = tangent(c, p, T, present, np, mu, a), tb = tangent(c, p, T, present, np, mu, b);
        if (ta != ta || tb != tb) return false;
        best = fmin(best, fmin(ta, tb));
        if (ta < tb) right = b; else left = a;
    }
    return best >= -m.mutol;
}

// A converged candidate enters the selection when stable; the first maximum of
// the entropy density wins. Returns whether it was stable.
__device__ bool consider(MixCell& c, const MixEval& cand, MixEval& best, bool& have) {
    if (!stableCandidate(c, cand)) { ++c.n.failures; return false; }
    ++c.n.stable;
    if (!have || cand.entropyD > best.entropyD) { best = cand; have = true; }
    return true;
}

__device__ __noinline__ bool temperatureSearch(MixCell& c, MixEval& best) {
    const ReactiveB200HemModel& m = c.m;
    constexpr double seeds[5] = {-1, .5, .95, .1, .9999};
    constexpr double fractions[4] = {.02, .25, .5, .75};
    bool have = false;
    MixEval cand;
    for (int mask = 1; mask < (1 << m.nl); ++mask) {
        int active[kLiq] = {0, 0}, n = 0;
        bool possible = true;
        double lower = m.Tmin, upper = m.Tmax;
        for (int i = 0; i < m.nl; ++i)
            if (mask & (1 << i)) {
                if (c.q[m.condensable[i]] <= 0) possible = false;
                else {
                    active[n++] = i;
                    lower = fmax(lower, m.liquidTmin[i]);
                    upper = fmin(upper, m.liquidTc[i] * (1 - 1e-10));
                }
            }
        if (!possible || !(upper > lower)) continue;
        for (int t = 0; t < 4; ++t) {
            ReactiveThermoState restart = c.guess;
            restart.T = lower + (upper - lower) * fractions[t];
            for (int j = 0; j < 5; ++j) {
                if (activeFlash(c, active, n, seeds[j], cand, -2, &restart)) consider(c, cand, best, have);
                else ++c.n.failures;
            }
        }
    }
    return have;
}

__device__ __forceinline__ bool prunable(const ReactiveB200HemModel& m) {
    return m.nl == 1 && m.condensedKind[0] == 0 && m.condensedKind[1] == 0;
}

__device__ __noinline__ bool searchCandidates(MixCell& c, MixEval& best) {
    const ReactiveB200HemModel& m = c.m;
    constexpr double seeds[5] = {-1, .5, .95, .1, .9999};
    constexpr double pairs[4] = {.1, .5, .95, .9999};
    bool have = false, gasStable = false;
    MixEval cand;
    double mass[kLiq] = {0, 0};
    const bool fastGas = m.stableGasPrune && prunable(m) && !c.adaptive;
    if (frozen(c, mass, cand, fastGas ? 4 : 0)) gasStable = consider(c, cand, best, have) && cand.s.gasMass > 0;
    else ++c.n.failures;
    const bool prune = m.stableGasPrune && prunable(m) && gasStable && !c.adaptive;
    double other = 0;
    for (int k = 0; k < m.ns; ++k)
        if (!isCondensable(m, k)) other += c.q[k];
    if (other == 0 && m.nl) {
        for (int i = 0; i < m.nl; ++i) mass[i] = c.q[m.condensable[i]];
        if (frozen(c, mass, cand, 0)) consider(c, cand, best, have);
        else ++c.n.failures;
    }
    for (int mask = 1; !prune && mask < (1 << m.nl); ++mask) {
        int active[kLiq] = {0, 0}, n = 0;
        bool possible = true;
        for (int i = 0; i < m.nl; ++i)
            if (mask & (1 << i)) {
                if (c.q[m.condensable[i]] <= 0) possible = false;
                else active[n++] = i;
            }
        if (!possible) continue;
        for (int j = 0; j < 5; ++j) {
            if (activeFlash(c, active, n, seeds[j], cand, -2, nullptr)) consider(c, cand, best, have);
            else ++c.n.failures;
        }
        if (c.adaptive) {
            if (activeFlash(c, active, n, -3, cand, -2, nullptr)) consider(c, cand, best, have);
            else ++c.n.failures;
        }
        if (c.adaptive && n == 2)
            for (int first = 1; first < 5; ++first)
                for (int second = 1; second < 5; ++second) {
                    if (first == second) continue;
                    if (activeFlash(c, active, n, pairs[first - 1], cand, pairs[second - 1], nullptr))
                        consider(c, cand, best, have);
                    else ++c.n.failures;
                }
    }
    // restart temperatures only when the search found no stable candidate
    if (!have) have = temperatureSearch(c, best);
    return have;
}

// The recovery of one cell: the candidate search; with the boundary recovery (or
// in a capillary batch, whose transported trace inventories can defeat the
// reference seeds) a second search in log vapour fractions when the first found
// nothing or left a condensable almost entirely liquid beside a gas phase, the
// larger entropy (the first search on a tie) kept.
__device__ bool recoverCell(MixCell& c, MixEval& result, bool capillaryBoundary) {
    const ReactiveB200HemModel& m = c.m;
    if (m.ns <= 0 || m.ns > kNs || m.nl < 0 || m.nl > kLiq || !fin(c.energy) || !(density(c) > 0)) return false;
    for (int k = 0; k < m.ns; ++k)
        if (!fin(c.q[k]) || c.q[k] < 0) return false;
    MixEval reference;
    const bool have = searchCandidates(c, reference);
    if (!m.boundaryRecovery && !capillaryBoundary) {
        if (have) result = reference;
        return have;
    }
    if (have) {
        bool boundary = false;
        for (int i = 0; i < m.nl; ++i) {
            const double q = c.q[m.condensable[i]];
            if (q > 0 && reference.s.gasMass > 0) boundary |= reference.s.liquidMass[i] / q > 1 - 1e-4;
        }
        if (!boundary) { result = reference; return true; }
    }
    c.adaptive = true;
    MixEval recovered;
    const bool found = searchCandidates(c, recovered);
    c.adaptive = false;
    if (!found && !have) return false;
    result = have && (!found || reference.entropyD >= recovered.entropyD) ? reference : recovered;
    return true;
}

enum : int { M_PHASES, M_RESIDUALS, M_CANDIDATES, M_STABLE, M_FD, M_SUCCEEDED, M_COUNT };

// A capillary cell input the reference's recoverCapillary accepts
// (src/reactiveThermo/reactiveDeviceFlash.h:572-588): a color in [0, 1], a
// finite jump, and a nonzero jump only with one pure liquid.
__device__ __forceinline__ bool capillaryAccepted(const ReactiveB200HemModel& m, double color, double jump) {
    return fin(color) && color >= 0 && color <= 1 && fin(jump) && (jump == 0 || (m.nl == 1 && m.condensedKind[0] == 0));
}

// One thread per cell. `order` (optional) names the cells: thread item i works on
// cell order[i], and every per-cell array is indexed by that cell. With
// `capillary` each cell is the reference's capillary recovery: UV equilibrium
// with the boundary search, or (equilibrium = 0) the frozen partition at the
// seed's liquid masses. Results go to out/success, or to outputs[cell] for the
// resident form; a failed cell gets its seed.
__global__ void __launch_bounds__(kBlock) mixtureFlashKernel(const ReactiveB200HemModel* __restrict__ model,
                                                            const double* __restrict__ q,
                                                            const double* __restrict__ energy, size_t count,
                                                            const ReactiveThermoState* __restrict__ seed,
                                                            const ReactiveGpuHemCapillaryInputV2* capillary,
                                                            const uint32_t* order, ReactiveThermoState* out,
                                                            int* success, ReactiveGpuHemOutputV1* outputs,
                                                            unsigned long long* totals) {
    const ReactiveB200HemModel& m = *model;
    Tally n;
    unsigned long long succeeded = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(blockDim.x) * gridDim.x) {
        const size_t cell = order ? size_t(order[i]) : i;
        MixCell c{m, {0, 0, 0, 0}, energy[cell], seed[cell], false, n};
        for (int k = 0; k < m.ns && k < kNs; ++k) c.q[k] = q[cell * size_t(m.ns) + k];
        MixEval result;
        bool ok;
        if (capillary) {
            const ReactiveGpuHemCapillaryInputV2 in = capillary[cell];
            c.color = in.color;
            c.jump = in.pressureJump;
            if (!capillaryAccepted(m, c.color, c.jump)) ok = false;
            else if (in.equilibrium) ok = recoverCell(c, result, true);
            else {
                const double mass[kLiq] = {c.guess.liquidMass[0], c.guess.liquidMass[1]};
                ok = frozen(c, mass, result, 0);
            }
        } else ok = recoverCell(c, result, false);
        const ReactiveThermoState& st = ok ? result.s : c.guess;
        if (out) out[cell] = st;
        if (success) success[cell] = ok ? 1 : 0;
        if (outputs) {
            outputs[cell].state = st;
            outputs[cell].success = ok ? 1 : 0;
        }
        succeeded += ok ? 1 : 0;
    }
    atomicAdd(totals + M_PHASES, n.phases);
    atomicAdd(totals + M_RESIDUALS, n.residuals);
    atomicAdd(totals + M_CANDIDATES, n.candidates);
    atomicAdd(totals + M_STABLE, n.stable);
    atomicAdd(totals + M_FD, n.fd);
    atomicAdd(totals + M_SUCCEEDED, succeeded);
}

// The capillary primitive initialisation (initializeCapillaryTP,
// src/reactiveThermo/reactiveDeviceFlash.h:589-613), one thread per cell: at the
// seed's (p, T) and liquid mass, with the gas at p - color*jump and the liquid
// at p + (1 - color)*jump, scale the densities so the phase volumes fill the
// cell; q and energy become the normalised densities and their energy where a
// cell succeeds.
__global__ void __launch_bounds__(kBlock) mixtureInitializeKernel(const ReactiveB200HemModel* __restrict__ model,
                                                                 double* q, double* energy, size_t count,
                                                                 const ReactiveThermoState* __restrict__ seed,
                                                                 const ReactiveGpuHemCapillaryInputV2* capillary,
                                                                 ReactiveThermoState* out, int* success,
                                                                 unsigned long long* totals) {
    const ReactiveB200HemModel& m = *model;
    Tally n;
    unsigned long long succeeded = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(blockDim.x) * gridDim.x) {
        MixCell c{m, {0, 0, 0, 0}, energy[i], seed[i], false, n};
        for (int k = 0; k < m.ns && k < kNs; ++k) c.q[k] = q[i * size_t(m.ns) + k];
        c.color = capillary[i].color;
        c.jump = capillary[i].pressureJump;
        bool ok = m.nl == 1 && m.condensedKind[0] == 0 && fin(c.color) && c.color >= 0 && c.color <= 1 && fin(c.jump);
        double liquid[kLiq] = {c.guess.liquidMass[0], 0};
        MixEval unit, value;
        if (ok) ok = evaluate(c, liquid, c.guess.p, c.guess.T, unit, false, nullptr) && fin(unit.volume)
                     && unit.volume > 0;
        if (ok) {
            for (int k = 0; k < m.ns; ++k) c.q[k] /= unit.volume;
            liquid[0] /= unit.volume;
            ok = evaluate(c, liquid, c.guess.p, c.guess.T, value, false, nullptr) && fin(value.energy)
                 && fabs(value.volume - 1) <= m.vtol;
        }
        if (ok) {
            value.s.volumeResidual = fabs(value.volume - 1);
            for (int k = 0; k < m.ns; ++k) q[i * size_t(m.ns) + k] = c.q[k];
            energy[i] = value.energy;
            out[i] = value.s;
        } else out[i] = c.guess;
        success[i] = ok ? 1 : 0;
        succeeded += ok ? 1 : 0;
    }
    atomicAdd(totals + M_PHASES, n.phases);
    atomicAdd(totals + M_SUCCEEDED, succeeded);
}

bool finiteHost(double x) { return x == x && std::fabs(x) <= 1.79769313486231570815e308; }

// The scope this build's mixture flash covers, on top of the reference's model
// validation (src/reactiveThermo/reactiveDeviceFlash.h:80-108).
std::string mixtureScope(const ReactiveB200HemModel& m) {
    if (m.ns < 1 || m.ns > kNs || m.nl < 0 || m.nl > kLiq)
        return "HEM model outside the mixture flash's scope: 1 to 4 gas species and 0 to 2 pure liquids";
    if (m.condensedKind[0] != 0 || m.condensedKind[1] != 0) return "Solid condensed phases are not part of this build";
    if ((m.boundaryRecovery != 0 && m.boundaryRecovery != 1) || (m.scalarRecovery != 0 && m.scalarRecovery != 1)
        || (m.stableGasPrune != 0 && m.stableGasPrune != 1)
        || (m.stableGasPrune && m.nl != 1)
        || (m.enforceSpeciesTemperatureBounds != 0 && m.enforceSpeciesTemperatureBounds != 1))
        return "Invalid CUDA HEM model flags";
    if (!finiteHost(m.Tmin) || !finiteHost(m.Tmax) || !(m.Tmin > 0 && m.Tmax > m.Tmin) || !finiteHost(m.pmin)
        || !finiteHost(m.pmax) || !(m.pmin > 0 && m.pmax > m.pmin) || !finiteHost(m.vtol) || !finiteHost(m.etol)
        || !finiteHost(m.mutol) || !(m.vtol > 0 && m.etol > 0 && m.mutol > 0))
        return "Invalid CUDA HEM model tables or domain";
    if (m.phase[0].ns != m.ns) return "Invalid CUDA HEM gas table";
    for (int k = 0; k < m.ns; ++k) {
        const ReactiveB200Species& sp = m.phase[0].species[k];
        if (!finiteHost(m.weights[k]) || m.weights[k] != sp.molecularWeight || !(sp.a > 0) || !(sp.b > 0)
            || sp.regionCount < 1 || sp.regionCount > REACTIVE_B200_MAX_REGIONS)
            return "Invalid CUDA HEM gas table";
    }
    for (int i = 0; i < m.nl; ++i) {
        const ReactiveB200Table& t = m.phase[i + 1];
        if (m.condensable[i] < 0 || m.condensable[i] >= m.ns || t.ns != 1
            || t.species[0].molecularWeight != m.weights[m.condensable[i]] || !(t.species[0].a > 0)
            || !(t.species[0].b > 0) || t.species[0].regionCount < 1
            || t.species[0].regionCount > REACTIVE_B200_MAX_REGIONS || !finiteHost(m.liquidTmin[i])
            || !finiteHost(m.liquidTc[i]) || !(m.liquidTmin[i] > 0 && m.liquidTc[i] > m.liquidTmin[i]))
            return "Invalid CUDA HEM liquid table or range";
        for (int j = 0; j < i; ++j)
            if (m.condensable[j] == m.condensable[i]) return "Invalid CUDA HEM liquid table or range";
    }
    return "";
}

}  // namespace

struct MixtureFlash {
    int device = 0;
    size_t capacity = 0;
    size_t bytes = 0;
    int ns = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> blocks;
    ReactiveB200HemModel* model = nullptr;
    double* q = nullptr;
    double* energy = nullptr;
    ReactiveThermoState* seed = nullptr;
    ReactiveThermoState* out = nullptr;
    int* success = nullptr;
    ReactiveGpuHemCapillaryInputV2* capillary = nullptr;  // allocated by the first capillary batch
    unsigned long long* totals = nullptr;
    template <class T> T* alloc(size_t n) {
        void* p = nullptr;
        check(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
        blocks.push_back(p);
        bytes += n * sizeof(T);
        return static_cast<T*>(p);
    }
    ~MixtureFlash() {
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : blocks) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
};

MixtureFlash* mixtureCreate(const ReactiveB200HemModel& m, size_t capacity, int device, std::string& why) {
    why = mixtureScope(m);
    if (!why.empty()) return nullptr;
    std::unique_ptr<MixtureFlash> f(new MixtureFlash);
    f->device = device;
    f->capacity = capacity;
    f->ns = m.ns;
    check(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    f->model = f->alloc<ReactiveB200HemModel>(1);
    f->q = f->alloc<double>(capacity * size_t(m.ns));
    f->energy = f->alloc<double>(capacity);
    f->seed = f->alloc<ReactiveThermoState>(capacity);
    f->out = f->alloc<ReactiveThermoState>(capacity);
    f->success = f->alloc<int>(capacity);
    f->totals = f->alloc<unsigned long long>(M_COUNT);
    check(cudaMemcpyAsync(f->model, &m, sizeof(m), cudaMemcpyHostToDevice, f->stream), "H2D model");
    check(cudaStreamSynchronize(f->stream), "sync");
    return f.release();
}

void mixtureDestroy(MixtureFlash* f) { delete f; }
size_t mixtureDeviceBytes(const MixtureFlash* f) { return f ? f->bytes : 0; }

void mixtureRun(MixtureFlash* f, const double* q, const double* energy, size_t count,
                const ReactiveGpuHemCapillaryInputV2* capillary, ReactiveThermoState* states, int* success,
                ReactiveGpuHemProfileV1& p) {
    require(count && count <= f->capacity, "CUDA HEM batch exceeds capacity");
    check(cudaSetDevice(f->device), "cudaSetDevice");
    const auto begin = std::chrono::steady_clock::now();
    cudaStream_t s = f->stream;
    if (capillary && !f->capillary) f->capillary = f->alloc<ReactiveGpuHemCapillaryInputV2>(f->capacity);
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "event");
    check(cudaEventCreate(&b), "event");
    check(cudaMemcpyAsync(f->q, q, count * size_t(f->ns) * sizeof(double), cudaMemcpyHostToDevice, s), "H2D q");
    check(cudaMemcpyAsync(f->energy, energy, count * sizeof(double), cudaMemcpyHostToDevice, s), "H2D e");
    check(cudaMemcpyAsync(f->seed, states, count * sizeof(ReactiveThermoState), cudaMemcpyHostToDevice, s), "H2D seed");
    if (capillary)
        check(cudaMemcpyAsync(f->capillary, capillary, count * sizeof(ReactiveGpuHemCapillaryInputV2),
                              cudaMemcpyHostToDevice, s),
              "H2D capillary");
    check(cudaMemsetAsync(f->totals, 0, M_COUNT * sizeof(unsigned long long), s), "memset");
    check(cudaEventRecord(a, s), "event");
    mixtureFlashKernel<<<gridFor(count, kBlock), kBlock, 0, s>>>(f->model, f->q, f->energy, count, f->seed,
                                                                  capillary ? f->capillary : nullptr, nullptr, f->out,
                                                                  f->success, nullptr, f->totals);
    check(cudaGetLastError(), "mixture flash");
    check(cudaEventRecord(b, s), "event");
    check(cudaMemcpyAsync(states, f->out, count * sizeof(ReactiveThermoState), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(success, f->success, count * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H success");
    unsigned long long t[M_COUNT] = {};
    check(cudaMemcpyAsync(t, f->totals, sizeof(t), cudaMemcpyDeviceToHost, s), "D2H totals");
    check(cudaStreamSynchronize(s), "sync");
    float kernel = 0;
    cudaEventElapsedTime(&kernel, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    p.batches = 1;
    p.submitted = count;
    p.succeeded = t[M_SUCCEEDED];
    p.deviceFailures = count - p.succeeded;
    p.phaseEvaluations = t[M_PHASES];
    p.residualEvaluations = t[M_RESIDUALS];
    p.flashCandidates = t[M_CANDIDATES];
    p.stableCandidates = t[M_STABLE];
    p.finiteDifferenceJacobians = t[M_FD];
    p.transferBytes = count * ((f->ns + 1) * sizeof(double) + 2 * sizeof(ReactiveThermoState) + sizeof(int)
                               + (capillary ? sizeof(ReactiveGpuHemCapillaryInputV2) : 0));
    p.deviceBytes = f->bytes;
    p.hostBytes = count * sizeof(ReactiveThermoState);
    p.kernelSeconds = kernel / 1000.;
    p.wallSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
    p.copySeconds = std::max(0.0, p.wallSeconds - p.kernelSeconds);
}

void mixtureInitialize(MixtureFlash* f, double* q, double* energy, size_t count,
                       const ReactiveGpuHemCapillaryInputV2* capillary, ReactiveThermoState* states, int* success,
                       ReactiveGpuHemProfileV1& p) {
    require(count && count <= f->capacity, "CUDA HEM batch exceeds capacity");
    check(cudaSetDevice(f->device), "cudaSetDevice");
    const auto begin = std::chrono::steady_clock::now();
    cudaStream_t s = f->stream;
    if (!f->capillary) f->capillary = f->alloc<ReactiveGpuHemCapillaryInputV2>(f->capacity);
    const size_t qBytes = count * size_t(f->ns) * sizeof(double);
    check(cudaMemcpyAsync(f->q, q, qBytes, cudaMemcpyHostToDevice, s), "H2D q");
    check(cudaMemcpyAsync(f->energy, energy, count * sizeof(double), cudaMemcpyHostToDevice, s), "H2D e");
    check(cudaMemcpyAsync(f->seed, states, count * sizeof(ReactiveThermoState), cudaMemcpyHostToDevice, s), "H2D seed");
    check(cudaMemcpyAsync(f->capillary, capillary, count * sizeof(ReactiveGpuHemCapillaryInputV2),
                          cudaMemcpyHostToDevice, s),
          "H2D capillary");
    check(cudaMemsetAsync(f->totals, 0, M_COUNT * sizeof(unsigned long long), s), "memset");
    mixtureInitializeKernel<<<gridFor(count, kBlock), kBlock, 0, s>>>(f->model, f->q, f->energy, count, f->seed,
                                                                       f->capillary, f->out, f->success, f->totals);
    check(cudaGetLastError(), "capillary initialisation");
    std::vector<double> nq(count * size_t(f->ns)), ne(count);
    std::vector<ReactiveThermoState> out(count);
    check(cudaMemcpyAsync(nq.data(), f->q, qBytes, cudaMemcpyDeviceToHost, s), "D2H q");
    check(cudaMemcpyAsync(ne.data(), f->energy, count * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H e");
    check(cudaMemcpyAsync(out.data(), f->out, count * sizeof(ReactiveThermoState), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(success, f->success, count * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H success");
    unsigned long long t[M_COUNT] = {};
    check(cudaMemcpyAsync(t, f->totals, sizeof(t), cudaMemcpyDeviceToHost, s), "D2H totals");
    check(cudaStreamSynchronize(s), "sync");
    p.batches = 1;
    p.submitted = count;
    p.succeeded = t[M_SUCCEEDED];
    p.deviceFailures = count - p.succeeded;
    p.phaseEvaluations = t[M_PHASES];
    // the caller's arrays change only when every cell succeeded
    if (!p.deviceFailures) {
        std::memcpy(q, nq.data(), qBytes);
        std::memcpy(energy, ne.data(), count * sizeof(double));
        std::memcpy(states, out.data(), count * sizeof(ReactiveThermoState));
    }
    p.transferBytes = 2 * (qBytes + count * sizeof(double)) + count * (2 * sizeof(ReactiveThermoState) + sizeof(int)
                                                                      + sizeof(ReactiveGpuHemCapillaryInputV2));
    p.deviceBytes = f->bytes;
    p.hostBytes = qBytes + count * (sizeof(double) + sizeof(ReactiveThermoState));
    p.wallSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
}

void mixtureRunResident(MixtureFlash* f, const double* q, const double* energy, const ReactiveThermoState* seed,
                        const ReactiveGpuHemCapillaryInputV2* capillary, const uint32_t* order, size_t count,
                        ReactiveGpuHemOutputV1* output, ReactiveGpuHemProfileV1& p) {
    require(count && count <= f->capacity, "Resident CUDA HEM batch exceeds capacity");
    check(cudaSetDevice(f->device), "cudaSetDevice");
    const auto begin = std::chrono::steady_clock::now();
    cudaStream_t s = f->stream;
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "event");
    check(cudaEventCreate(&b), "event");
    check(cudaMemsetAsync(f->totals, 0, M_COUNT * sizeof(unsigned long long), s), "memset");
    check(cudaEventRecord(a, s), "event");
    mixtureFlashKernel<<<gridFor(count, kBlock), kBlock, 0, s>>>(f->model, q, energy, count, seed, capillary, order,
                                                                  nullptr, nullptr, output, f->totals);
    check(cudaGetLastError(), "mixture flash");
    check(cudaEventRecord(b, s), "event");
    unsigned long long t[M_COUNT] = {};
    check(cudaMemcpyAsync(t, f->totals, sizeof(t), cudaMemcpyDeviceToHost, s), "D2H totals");
    check(cudaStreamSynchronize(s), "sync");
    float kernel = 0;
    cudaEventElapsedTime(&kernel, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    p.batches = 1;
    p.submitted = count;
    p.succeeded = t[M_SUCCEEDED];
    p.deviceFailures = count - p.succeeded;
    p.phaseEvaluations = t[M_PHASES];
    p.residualEvaluations = t[M_RESIDUALS];
    p.flashCandidates = t[M_CANDIDATES];
    p.stableCandidates = t[M_STABLE];
    p.finiteDifferenceJacobians = t[M_FD];
    p.transferBytes = sizeof(t);
    p.deviceBytes = f->bytes;
    p.kernelSeconds = kernel / 1000.;
    p.wallSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
    p.copySeconds = std::max(0.0, p.wallSeconds - p.kernelSeconds);
}

}  // namespace rb200
