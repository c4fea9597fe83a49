// Pure-fluid HEM UV flash on the device: one candidate solve per thread.
//
// For one condensable species with its own pure liquid (the pure-N2O cases)
// the reference search (src/reactiveThermo/reactiveDeviceFlash.h:509-560) is a
// fixed list of independent candidates followed by a selection:
//   0 all-gas partition: scalar T-Newton at fixed rho (:264-299), else the
//     frozen (ln p, ln T) Newton (:302-326)
//   1 all-liquid partition: frozen (ln p, ln T) Newton
//   2..6 two-phase (ln p, ln T, beta) Newton from beta seeds
//     {previous, .5, .95, .1, .9999} (:374-448, :527)
// each checked for stability (:449-485) and ranked by entropy density, first
// maximum wins (:486-489); with no stable candidate, the same two-phase seeds
// restart from T fractions {.02, .25, .5, .75} of the legal liquid interval
// (:490-508, src/reactiveThermo/reactiveFlashSeeds.h:14-16).
//
// Because candidates only meet in the selection, each (cell, candidate) pair is
// an independent work item here: warps run one candidate kind over 32 cells, so
// control flow inside a warp differs only by iteration counts, and a persistent
// kernel pulls items from an on-device queue so uneven Newton work balances
// across SMs. The per-thread state is kept to what the Newton iteration needs
// (the line search overwrites the current evaluation in place).
#pragma once
#include "pr_eos.cuh"
#include "../../include/reactive_b200_types.h"

// Linkage of the flash-level routines (see RB200_EOS_FN).
#ifndef RB200_FLASH_FN
#define RB200_FLASH_FN static __noinline__
#endif

namespace rb200 {

struct HemConst {
    PureSpecies gas, liq;
    double Tmin, Tmax, pmin, pmax, vtol, etol, mutol;
    double liquidTmin, liquidTc;
    double gasTmin, gasTmax;  // NASA fit bounds of the gas species (enforced when requested)
    int enforceBounds, scalarRecovery, analyticJacobian, stableGasPrune;
    int samePure;  // gas and liquid tables hold the same species: one cubic serves both roots
    // Density below which the all-liquid partition provably cannot converge (0: no bound).
    // A reported liquid needs rho >= rhoMid(T) >= rho_c whenever the reported-phase line
    // falls with T and the liquid range ends at or below its Tc; the all-liquid volume
    // residual q/rho_l - 1 then stays below q/rho_c - 1 < -vtol.
    double liquidFloor;
    // Two-phase admissibility bound of a pure fluid (domeN = 0: none). A two-phase
    // candidate can only converge to a mixture of the two roots of one cubic at a
    // (p, T) where their chemical potentials agree to mutol, so the cell's specific
    // volume and internal energy must lie (within the volume and energy
    // tolerances) on a saturation tie line. domeUp[j] / domeLo[j] bound the
    // specific internal energy of every tie-line point whose specific volume lies
    // within one grid step of v_j = exp(domeLnV0 + j / domeInvStep).
    const double* domeUp;
    const double* domeLo;
    int domeN;
    double domeLnV0, domeInvStep, domeVlo, domeVhi, domeMarginU, domeMarginV;
    // Saturation pressure of the pure fluid at satN temperatures T_j = satT0 + j / satInvStep
    // (built with the bound; satP[j] = 0 where unresolved or where the coexisting phases'
    // compressibility factors lie within 0.05 of each other, near the critical end).
    const double* satP;
    int satN;
    double satT0, satInvStep;
};

struct CellInput {
    double q, e, gp, gT, gml;  // mass density, internal energy density, seed p, T, liquid mass
    int noTwoPhase;            // no two-phase candidate can converge (the dome bound)
};

// True when the cell's (1/q, e/q) lies provably outside every saturation tie
// line widened by the margins: the two-phase seeds would all fail.
__device__ inline bool twoPhaseImpossible(const HemConst& C, double q, double e) {
    if (C.domeN < 4 || !(q > 0) || !isfinite(q) || !isfinite(e)) return false;
    const double v = 1 / q, u = e / q;
    if (v < C.domeVlo * (1 - C.domeMarginV) || v > C.domeVhi * (1 + C.domeMarginV)) return true;
    int j = int(floor((log(v) - C.domeLnV0) * C.domeInvStep));
    j = j < 1 ? 1 : (j > C.domeN - 3 ? C.domeN - 3 : j);
    double up = C.domeUp[j - 1], lo = C.domeLo[j - 1];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        up = fmax(up, C.domeUp[j + k]);
        lo = fmin(lo, C.domeLo[j + k]);
    }
    const double margin = C.domeMarginU + 10 * C.etol * fabs(u);
    return u > up + margin || u < lo - margin;
}

struct Counts {
    unsigned phases = 0, residuals = 0, candidates = 0, stable = 0, failures = 0, analytic = 0, fd = 0;
};

// Phase sums of one evaluation at (p, T) with a given liquid mass (the
// reference's Evaluation, reduced to the fields the solvers and the state need).
struct Eval {
    double p, T, gasMass, liqMass;
    double volume, energy, entropyD, Vp, VT, Ep, ET, cpD;
    double muG, muL;                // chemical potential / RT
    double gRho, gE, gV, gH;        // gas phase (if gasMass > 0)
    double lRho, lE, lV, lH;        // liquid phase (if liqOk)
    double cv, soundFrozen;
    bool liqOk;
};

__device__ __forceinline__ double clampd(double a, double l, double h) { return fmin(fmax(a, l), h); }

__device__ __forceinline__ bool inBounds(const HemConst& C, double p, double T) {
    return fin(p) && fin(T) && p >= C.pmin && p <= C.pmax && T >= C.Tmin && T <= C.Tmax;
}

__device__ RB200_FLASH_FN int gasPhase(const HemConst& C, double p, double T, bool chem, PhaseProps& o, Counts& n) {
    ++n.phases;
    if (!inBounds(C, p, T)) return EOS_INVALID_INPUT;
    if (C.enforceBounds && (T < C.gasTmin || T > C.gasTmax)) return EOS_INVALID_INPUT;
    return prTP(C.gas, T, p, ROOT_GAS, chem, o);
}

__device__ RB200_FLASH_FN int liquidPhase(const HemConst& C, double p, double T, bool chem, PhaseProps& o, Counts& n) {
    ++n.phases;
    if (!inBounds(C, p, T)) return EOS_INVALID_INPUT;
    if (T < C.liquidTmin) return EOS_INVALID_INPUT;
    if (T >= C.liquidTc * (1 - 1e-10)) return EOS_UNAVAILABLE;
    return prTP(C.liq, T, p, ROOT_LIQUID, chem, o);
}

__device__ __forceinline__ bool unavailableStatus(int s) { return s == EOS_UNAVAILABLE || s == EOS_NO_ROOT; }

__device__ __forceinline__ void addPhase(Eval& v, double mass, const PhaseProps& ph, double pressure) {
    const double volume = mass / ph.rho, vp = -volume * ph.kappaT, vt = volume * ph.alpha;
    v.volume += volume;
    v.energy += mass * ph.e;
    v.entropyD += mass * ph.s;
    v.Vp += vp;
    v.VT += vt;
    v.Ep += -v.T * vt - pressure * vp;
    v.ET += mass * ph.cp - pressure * vt;
    v.cpD += mass * ph.cp;
}

// Gas-branch status at (p, T) from shared T-terms and roots (same checks and
// order as gasPhase).
__device__ __forceinline__ int gasFromShared(const HemConst& C, int shared, const TTerms& t, const Roots& r,
                                             double p, bool chem, PhaseProps& o, Counts& n) {
    ++n.phases;
    if (C.enforceBounds && (t.T < C.gasTmin || t.T > C.gasTmax)) return EOS_INVALID_INPUT;
    if (shared != EOS_OK) return shared;
    return rootProps(C.gas, t, r, p, ROOT_GAS, chem, o);
}
__device__ __forceinline__ int liquidFromShared(const HemConst& C, int shared, const TTerms& t, const Roots& r,
                                                double p, bool chem, PhaseProps& o, Counts& n) {
    ++n.phases;
    if (t.T < C.liquidTmin) return EOS_INVALID_INPUT;
    if (t.T >= C.liquidTc * (1 - 1e-10)) return EOS_UNAVAILABLE;
    if (shared != EOS_OK) return shared;
    return rootProps(C.liq, t, r, p, ROOT_LIQUID, chem, o);
}

// What an accepted gas probe at (p, T) hands to the evaluations that follow at
// the same point: the gas table's T-terms, the gas phase's properties (without
// the chemical potential) at the probe's density, which is the gas root of the
// cubic at (p, T), with their chemical-potential intermediates, and the cubic's
// roots when the probe solved it (`roots`; otherwise an evaluation that needs
// them solves the cubic itself, through the same routine). `clear` (meaningful
// without roots): the cubic has no liquid root, or one above the covolume and at
// least 1e-6 of its volume below the middle root, both by margins far above
// rounding.
struct GasPoint {
    TTerms t;
    Roots r;
    PhaseProps gas;
    ChemTerms chem;
    bool roots, clear;
};

// Phase sums at (p, T) for liquid mass `mass` out of total density q. With
// `virt` the liquid is also evaluated when absent and both chemical potentials
// are formed (two-phase residual and stability test). When both branches are
// needed and the tables hold one species, the T-terms and the cubic are formed
// once for both roots (the same arithmetic as two separate evaluations).
// `known` (optional) is an accepted gas probe's point at exactly (p, T): its
// T-terms replace the shared path's, its gas properties the gas root's, with
// `virt` its chemical potential from the kept intermediates; its roots, or the
// cubic solved here through the same routine the probe uses, serve the liquid.
__device__ RB200_FLASH_FN bool evaluate(const HemConst& C, double q, double mass, double p, double T, bool virt, Eval& v,
                                Counts& n, const GasPoint* known = nullptr) {
    v.p = p; v.T = T;
    v.volume = v.energy = v.entropyD = v.Vp = v.VT = v.Ep = v.ET = v.cpD = 0;
    v.muG = v.muL = 0;
    v.gRho = v.gE = v.gV = v.gH = 0;
    v.lRho = v.lE = v.lV = v.lH = 0;
    v.liqOk = false;
    v.liqMass = mass;
    v.gasMass = 0;
    if (!inBounds(C, p, T)) return false;
    if (!(q > 0) || !fin(q)) return false;
    if (!fin(mass) || mass < 0 || mass > q) return false;
    const double gas = q - mass;
    if (!fin(gas) || gas < 0 || gas > q) return false;
    v.gasMass = gas;
    const bool needLiquid = mass > 0 || (virt && q > 0);
    const bool shared = C.samePure && gas > 0 && needLiquid;
    TTerms t;
    Roots r;
    int sharedStatus = EOS_OK;
    if (shared && known) {
        t = known->t;
        if (known->roots) r = known->r;
        else sharedStatus = cubicRoots(C.gas, T, p, t.aa, r);
    } else if (shared) {
        sharedStatus = tTerms(C.gas, T, t);
        if (sharedStatus == EOS_OK) sharedStatus = cubicRoots(C.gas, T, p, t.aa, r);
    }
    PhaseProps ph;
    if (gas > 0) {
        int st = EOS_OK;
        if (known) {
            ph = known->gas;
            if (virt) {
                ph.mu = chemPotential(C.gas, known->t, ph.V, known->chem);
                if (!fin(ph.mu)) st = EOS_NONFINITE;
            }
        } else st = shared ? gasFromShared(C, sharedStatus, t, r, p, virt, ph, n) : gasPhase(C, p, T, virt, ph, n);
        if (st != EOS_OK) return false;
        addPhase(v, gas, ph, p);
        v.gRho = ph.rho; v.gE = ph.e; v.gV = ph.V; v.gH = ph.h;
        if (virt) v.muG = ph.mu / (kGas * T);
    }
    if (needLiquid) {
        const int status = shared ? liquidFromShared(C, sharedStatus, t, r, p, virt, ph, n)
                                  : liquidPhase(C, p, T, virt, ph, n);
        if (status != EOS_OK) {
            if (mass > 0 || !unavailableStatus(status)) return false;
            v.muL = HUGE_VAL;
        } else {
            v.liqOk = true;
            v.lRho = ph.rho; v.lE = ph.e; v.lV = ph.V; v.lH = ph.h;
            if (virt) v.muL = ph.mu / (kGas * T);
            if (mass > 0) addPhase(v, mass, ph, p);
        }
    }
    const double cp = v.cpD / q;
    v.cv = (v.cpD + T * v.VT * v.VT / v.Vp) / q;
    if (!fin(v.cv) || v.cv <= 0) return false;
    const double specific = v.volume / q, vp = v.Vp / q, vt = v.VT / q;
    const double adiabatic = vp + T * vt * vt / cp;
    if (!(adiabatic < 0)) return false;
    v.soundFrozen = sqrt(-specific * specific / adiabatic);
    return fin(v.soundFrozen) && v.soundFrozen > 0;
}

__device__ __forceinline__ double energyScale(const Eval& v, double q) { return fmax(1e5 * q, v.cpD * v.T); }

// Full-pivot elimination for n <= 3 with the rank test pivot > largest*n*eps.
__device__ RB200_FLASH_FN bool solveSmall(double a[3][3], double b[3], int n, double x[3]) {
    int column[3] = {0, 1, 2};
    double largest = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (i >= n) continue;
        if (!fin(b[i])) return false;
#pragma unroll
        for (int j = 0; j < 3; ++j) if (j < n && !fin(a[i][j])) return false;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (k >= n) break;
        int row = k, col = k;
        double pivot = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                if (j >= k && i >= k && j < n && i < n && fabs(a[i][j]) > pivot) { pivot = fabs(a[i][j]); row = i; col = j; }
        largest = fmax(largest, pivot);
        if (!(pivot > largest * n * DBL_EPSILON)) return false;
#pragma unroll
        for (int r = 0; r < 3; ++r)
            if (r == row && row != k) {
#pragma unroll
                for (int j = 0; j < 3; ++j) { const double t = a[k][j]; a[k][j] = a[r][j]; a[r][j] = t; }
                const double t = b[k]; b[k] = b[r]; b[r] = t;
            }
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (c == col && col != k) {
#pragma unroll
                for (int i = 0; i < 3; ++i) { const double t = a[i][k]; a[i][k] = a[i][c]; a[i][c] = t; }
                const int t = column[k]; column[k] = column[c]; column[c] = t;
            }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (i <= k || i >= n) continue;
            const double f = a[i][k] / a[k][k];
            a[i][k] = f;
#pragma unroll
            for (int j = 0; j < 3; ++j) if (j > k && j < n) a[i][j] -= f * a[k][j];
            b[i] -= f * b[k];
        }
    }
    double z[3] = {0, 0, 0};
#pragma unroll
    for (int i = 2; i >= 0; --i) {
        if (i >= n) continue;
        double v = b[i];
#pragma unroll
        for (int j = 0; j < 3; ++j) if (j > i && j < n) v -= a[i][j] * z[j];
        z[i] = v / a[i][i];
        if (!fin(z[i])) return false;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (i < n && column[i] == c) x[c] = z[i];
    return true;
}

// The gas-root check by the root solve: the cubic's roots at (g.t.T, p) into
// g.r (through the out-of-line cubicRoots, the routine every later evaluation
// at this point uses, so the roots carry the same bits on every path), then the
// gas root must pass the root-property checks and be the density q the
// pressure came from (to 1e-8 of q).
__device__ RB200_FLASH_FN bool gasRootAt(const HemConst& C, double q, double p, GasPoint& g) {
    if (cubicRoots(C.gas, g.t.T, p, g.t.aa, g.r) != EOS_OK) return false;
    PhaseProps root;
    return rootPropsBody(C.gas, g.t, g.r, p, ROOT_GAS, false, root, nullptr) == EOS_OK
           && !(fabs(root.rho - q) > 1e-8 * q);
}

// The outcome of gasRootAt decided without solving the cubic: p = p(T, q), so
// V0 = W/q is a root of the cubic at (T, p), which factors as
// (V - V0)(V^2 + sV + t) and leaves the other two roots to a quadratic. 1: the
// root solve would classify a gas root equal to V0 (to rounding) and accept it
// on q's side of the reported-phase line; 0: it would not (another root is the
// gas root, or the gas branch is missing there); -1: undecided, the root solve
// decides. Every decision keeps margins orders of magnitude above rounding from
// the root solve's own thresholds: its discriminant classes (|disc| >= 1e-10
// against 1e-14, ||h| - |q|| >= 1e-8 against 1e-10), the other roots at least
// 1e-6 of V0 away from V0 (so V0 is no near-double root and dp/dV stays off
// zero there), and 1e-9 of V0 (or of the line's density) from the covolume,
// the classification centre and the reported-phase line. `phase` is the
// reported phase of the (T, q) evaluation; `clear` as GasPoint::clear.
__device__ __forceinline__ int gasRootIsV0(const PureSpecies& sp, const TTerms& t, double p, double q, int phase,
                                           bool& clear) {
    const double T = t.T, V0 = sp.W / q, ip = 1.0 / p;
    const double b = sp.b, b2 = b * b, RTp = kGas * T * ip, aap = t.aa * ip, bn = b - RTp;
    const double cn = -(2.0 * RTp * b - aap + 3.0 * b2), dn = b2 * RTp + b2 * b - aap * b;
    const double center = -bn * kThird, delta2 = (bn * bn - 3.0 * cn) * (1.0 / 9.0);
    const double qc = 2.0 * bn * bn * bn * (1.0 / 27.0) - bn * cn * kThird + dn;
    const double delta = delta2 > 0 ? sqrt(delta2) : 0.0, h = 2.0 * delta * delta2;
    const double disc = qc * qc - h * h, margin = 1e-9 * V0;
    clear = false;
    if (!(fabs(fabs(h) - fabs(qc)) >= 1e-8) || !(fabs(disc) >= 1e-10) || !(V0 - b > margin)) return -1;
    bool single = disc > 0;  // one real root: V0
    clear = single;
    if (!single) {
        const double s = bn + V0, tq = cn + V0 * s, d2 = s * s - 4.0 * tq;
        if (!(d2 > 0)) return -1;
        const double r = sqrt(d2), v1 = .5 * (-s + r), v2 = .5 * (-s - r);
        if (v1 > V0 + 1e-6 * V0) return 0;  // the largest root, the gas root if any, is not V0
        if (!(v1 < V0 - 1e-6 * V0) || !(fabs(v1 - b) > margin) || !(fabs(v2 - b) > margin)) return -1;
        single = !(v1 > b);  // V0 the only root above the covolume
        // three physical roots with the liquid one off the spinodal, or V0 alone
        clear = single || (v2 > b && v1 - v2 > 1e-6 * v1);
    }
    if (single && !(T > sp.Tc)) {
        // a lone root is the gas root when it is not below the centre
        if (!(fabs(V0 - center) > margin)) return -1;
        if (V0 < center) return 0;
    }
    if (phase == -2) return 1;  // above the reported-phase line's temperature: no density test
    const double rhoMid = sp.rhoC + (T - sp.tcLine) * sp.dRho / sp.dT;
    if (q < rhoMid * (1 - 1e-9)) return phase == -1 ? 1 : -1;
    if (q > rhoMid * (1 + 1e-9)) return phase == 0 ? 0 : -1;
    return -1;
}

// Energy residual of the all-gas state at (T, rho) and the gas-root check: the
// properties at (T, rho), then the gas root of the cubic at the resulting
// pressure must be that density: decided by gasRootIsV0 where its margins
// allow, else by the root solve. `g` receives the point: the T-terms, the
// properties at rho with their chemical-potential intermediates, and the roots
// when they were solved.
__device__ RB200_FLASH_FN bool gasProbe(const HemConst& C, double q, double eIn, double T, double& F, double& cv, double& p,
                                double& cp, GasPoint& g, Counts& n) {
    int phase;
    ++n.phases;
    if (!fin(T) || !fin(q) || T <= 0 || q <= 0) return false;
    if (tTermsBody(C.gas, T, g.t) != EOS_OK || prTrhoTBody(C.gas, g.t, q, false, g.gas, phase, &g.chem) != EOS_OK)
        return false;
    p = g.gas.p;  // finite and positive
    if (!inBounds(C, p, T)) return false;
    if (C.enforceBounds && (T < C.gasTmin || T > C.gasTmax)) return false;
    const int decided = gasRootIsV0(C.gas, g.t, p, q, phase, g.clear);
    if (decided == 0) return false;
    g.roots = decided < 0;
    if (g.roots) {
        ++n.phases;
        if (!gasRootAt(C, q, p, g)) return false;
    }
    F = q * g.gas.e - eIn;
    cv = q * g.gas.cv;
    cp = g.gas.cp;
    return fin(F) && fin(cv) && cv > 0;
}

struct CandidateOut {
    double vres, eres, cres, soundEq;
    int iterations;
};

// Scalar T-Newton of the all-gas partition at fixed rho. `g` ends with the gas
// table's terms at the converged (p, T): the probe that set them is the last
// probe (a bracket search is always followed by a probe at the bracket end or
// by at least one Newton probe, which rewrite `g`). The probes' gas-root
// decisions are those of full root solves, so the iterates and the final
// point are those of probes that always solve.
__device__ RB200_FLASH_FN bool scalarGas(const HemConst& C, const CellInput& in, Eval& v, CandidateOut& o, GasPoint& g,
                                 Counts& n) {
    const double q = in.q;
    double T = clampd(in.gT, C.Tmin, C.Tmax), F, cv, p, cp;
    if (!gasProbe(C, q, in.e, T, F, cv, p, cp, g, n)) return false;
    const double scale = fmax(1e5 * q, q * cp * T);
    double lower = T, upper = T, fl = F, fh = F;
    if (fabs(F) > C.etol * scale) {
        double radius = fmax(1., .01 * T);
        for (int j = 0; j < 24 && (fl > 0 || fh < 0); ++j, radius *= 2) {
            double val, d1, d2, d3;
            if (fl > 0) {
                double cand = fmax(C.Tmin, T - radius);
                bool found = false;
                for (int r = 0; r < 8 && !found; ++r) {
                    if (gasProbe(C, q, in.e, cand, val, d1, d2, d3, g, n)) { fl = val; lower = cand; found = true; }
                    else cand = .5 * (lower + cand);
                }
                if (!found) return false;
            }
            if (fh < 0) {
                double cand = fmin(C.Tmax, T + radius);
                bool found = false;
                for (int r = 0; r < 8 && !found; ++r) {
                    if (gasProbe(C, q, in.e, cand, val, d1, d2, d3, g, n)) { fh = val; upper = cand; found = true; }
                    else cand = .5 * (upper + cand);
                }
                if (!found) return false;
            }
            if (fabs(fl) <= C.etol * scale) { T = lower; if (!gasProbe(C, q, in.e, T, F, cv, p, d3, g, n)) return false; break; }
            if (fabs(fh) <= C.etol * scale) { T = upper; if (!gasProbe(C, q, in.e, T, F, cv, p, d3, g, n)) return false; break; }
            if (lower == C.Tmin && upper == C.Tmax) break;
        }
        if (!(fabs(F) <= C.etol * scale || (fl <= 0 && fh >= 0 && upper > lower))) return false;
    }
    int it = 0;
    for (; it < 70 && fabs(F) > C.etol * scale; ++it) {
        if (F > 0) upper = T; else lower = T;
        const double next = T - F / cv;
        T = fin(next) && next > lower && next < upper ? next : .5 * (lower + upper);
        double d3;
        if (!gasProbe(C, q, in.e, T, F, cv, p, d3, g, n)) return false;
    }
    if (fabs(F) > C.etol * scale) return false;
    if (!evaluate(C, q, 0.0, p, T, false, v, n, &g)) return false;
    o.vres = fabs(v.volume - 1);
    o.eres = fabs(v.energy - in.e) / energyScale(v, q);
    o.cres = 0;
    o.iterations = it;
    o.soundEq = v.soundFrozen;
    return o.vres <= C.vtol && o.eres <= C.etol;
}

// Newton on (ln p, ln T) with the liquid partition held fixed. A converged
// scalar all-gas solve leaves the gas table's terms at its (p, T) in `g` and
// sets `known`.
__device__ RB200_FLASH_FN bool frozenSolve(const HemConst& C, const CellInput& in, double mass, int stallLimit, Eval& v,
                                   CandidateOut& o, Counts& n, GasPoint& g, bool& known) {
    known = false;
    if (!fin(in.e)) return false;
    if (C.scalarRecovery && mass == 0 && scalarGas(C, in, v, o, g, n)) {
        known = true;
        return true;
    }
    double p = clampd(in.gp, C.pmin, C.pmax), T = clampd(in.gT, C.Tmin, C.Tmax);
    if (!evaluate(C, in.q, mass, p, T, false, v, n)) return false;
    int stalled = 0;
    for (int it = 0; it < 70; ++it) {
        const double scale = energyScale(v, in.q), rv = v.volume - 1, re = (v.energy - in.e) / scale;
        o.vres = fabs(rv); o.eres = fabs(re); o.cres = 0; o.iterations = it; o.soundEq = v.soundFrozen;
        if (fabs(rv) <= C.vtol && fabs(re) <= C.etol) return true;
        double a[3][3] = {{v.Vp * p, v.VT * T, 0}, {v.Ep * p / scale, v.ET * T / scale, 0}, {0, 0, 0}};
        double b[3] = {-rv, -re, 0}, step[3] = {0, 0, 0};
        if (!solveSmall(a, b, 2, step)) return false;
        const double limit = fmax(1., fmax(fabs(step[0]) / .7, fabs(step[1]) / .2));
        step[0] /= limit;
        step[1] /= limit;
        const double previous = fmax(fabs(rv), fabs(re));
        bool accepted = false;
        double fraction = 1;
        for (int k = 0; k < 30; ++k, fraction *= .5) {
            const double pp = p * exp(fraction * step[0]), tt = T * exp(fraction * step[1]);
            if (evaluate(C, in.q, mass, pp, tt, false, v, n)) {
                const double next = fmax(fabs(v.volume - 1), fabs(v.energy - in.e) / scale);
                if (next < previous * (1 - 1e-4 * fraction) || next < fmin(C.vtol, C.etol)) {
                    p = pp; T = tt; accepted = true;
                    stalled = fraction < 1. / 32 ? stalled + 1 : 0;
                    break;
                }
            }
        }
        if (!accepted) return false;
        if (stallLimit > 0 && stalled >= stallLimit
            && !(fabs(v.volume - 1) <= C.vtol && fabs(v.energy - in.e) / energyScale(v, in.q) <= C.etol))
            return false;
    }
    return false;
}

__device__ RB200_FLASH_FN bool twoPhaseResidual(const HemConst& C, const CellInput& in, double lp, double lT, double beta,
                                        double scale, double f[3], Eval& v, Counts& n) {
    ++n.residuals;
    if (!(beta >= 0 && beta < 1)) return false;
    if (!evaluate(C, in.q, beta * in.q, exp(lp), exp(lT), true, v, n) || !(v.gasMass > 0)) return false;
    f[0] = v.volume - 1;
    f[1] = (v.energy - in.e) / scale;
    f[2] = v.muL - v.muG;
    return fin(f[2]);
}

// d f / d(ln p, ln T, beta): the volume and energy rows from the phase sums,
// dV/dbeta = q(1/rho_l - 1/rho_g), dE/dbeta = q(e_l - e_g); the chemical row from
// d(mu/RT)/d ln p = p V/RT and d(mu/RT)/d ln T = -H/RT of each pure phase.
__device__ inline bool analyticJacobian(const Eval& v, double q, double W, double scale, double J[3][3]) {
    if (!v.liqOk || !(v.gasMass > 0)) return false;
    const double RT = kGas * v.T;
    J[0][0] = v.Vp * v.p; J[0][1] = v.VT * v.T; J[0][2] = q * (1 / v.lRho - 1 / v.gRho);
    J[1][0] = v.Ep * v.p / scale; J[1][1] = v.ET * v.T / scale; J[1][2] = q * (v.lE - v.gE) / scale;
    J[2][0] = v.p * (v.lV - v.gV) / RT;
    J[2][1] = -(v.lH - v.gH) * W / RT;
    J[2][2] = 0;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) if (!fin(J[i][j])) return false;
    return true;
}

__device__ RB200_FLASH_FN bool jacobian(const HemConst& C, const CellInput& in, const double x[3], double scale,
                                const double f[3], const Eval& v, double J[3][3], Counts& n) {
    if (C.analyticJacobian && analyticJacobian(v, in.q, C.liq.W, scale, J)) { ++n.analytic; return true; }
    ++n.fd;
    Eval w;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        double h = j < 2 ? 2e-6 : 2e-5;
        bool success = false;
        for (int attempt = 0; attempt < 12 && !success; ++attempt, h *= .5) {
            double xp[3] = {x[0], x[1], x[2]}, xm[3] = {x[0], x[1], x[2]}, fp[3], fm[3];
            xp[j] += h;
            xm[j] -= h;
            const bool plus = twoPhaseResidual(C, in, xp[0], xp[1], xp[2], scale, fp, w, n);
            const bool minus = twoPhaseResidual(C, in, xm[0], xm[1], xm[2], scale, fm, w, n);
            if (!plus && !minus) continue;
            success = true;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double val = plus && minus ? (fp[i] - fm[i]) / (2 * h) : plus ? (fp[i] - f[i]) / h
                                                                                     : (f[i] - fm[i]) / h;
                J[i][j] = val;
                success = success && fin(val);
            }
        }
        if (!success) return false;
    }
    return true;
}

// Two-phase Newton from a beta seed (seed < 0: the previous state's liquid
// fraction clamped to [1e-8, 1-1e-8]); restartT >= 0 replaces the seed T.
__device__ RB200_FLASH_FN bool twoPhaseSolve(const HemConst& C, const CellInput& in, double seed, double restartT, Eval& v,
                                     CandidateOut& o, Counts& n) {
    ++n.candidates;
    const double q = in.q;
    const double gT = restartT >= 0 ? restartT : in.gT;
    const double scale = fmax(1e5 * q, fmax(fabs(in.e), q * 2000 * fmax(gT, C.Tmin)));
    double x[3] = {log(clampd(in.gp, C.pmin, C.pmax)), log(clampd(gT, C.Tmin, C.Tmax)),
                   seed < 0 ? clampd(in.gml / q, 1e-8, 1 - 1e-8) : seed};
    double f[3];
    if (!twoPhaseResidual(C, in, x[0], x[1], x[2], scale, f, v, n)) return false;
    for (int it = 0; it < 90; ++it) {
        double J[3][3];
        const double chemical = fabs(f[2]);
        if (fabs(f[0]) <= C.vtol && fabs(f[1]) <= C.etol && chemical <= C.mutol) {
            o.vres = fabs(f[0]); o.eres = fabs(f[1]); o.cres = chemical; o.iterations = it;
            if (!jacobian(C, in, x, scale, f, v, J, n)) return false;
            double rhs[3] = {-1 / q, v.p / (q * scale), 0}, response[3] = {0, 0, 0};
            if (!solveSmall(J, rhs, 3, response)) return false;
            const double squared = v.p * response[0];
            if (!fin(squared) || squared <= 0) return false;
            o.soundEq = sqrt(squared);
            return o.soundEq <= v.soundFrozen * (1 + 2e-3);
        }
        if (!jacobian(C, in, x, scale, f, v, J, n)) return false;
        double rhs[3] = {-f[0], -f[1], -f[2]}, step[3] = {0, 0, 0};
        if (!solveSmall(J, rhs, 3, step)) return false;
        const double limiter = fmax(fmax(1., fmax(fabs(step[0]) / .7, fabs(step[1]) / .18)), fabs(step[2]) / .3);
        for (int j = 0; j < 3; ++j) step[j] /= limiter;
        const double previous = fmax(fabs(f[0]), fmax(fabs(f[1]), fabs(f[2])));
        bool accepted = false;
        double fraction = 1;
        for (int k = 0; k < 30; ++k, fraction *= .5) {
            const double tb = x[2] + fraction * step[2];
            if (!(tb >= 0 && tb < 1)) { ++n.residuals; continue; }
            const double tp = x[0] + fraction * step[0], tt = x[1] + fraction * step[1];
            double tf[3];
            if (twoPhaseResidual(C, in, tp, tt, tb, scale, tf, v, n)
                && fmax(fabs(tf[0]), fmax(fabs(tf[1]), fabs(tf[2]))) < previous * (1 - 1e-4 * fraction)) {
                x[0] = tp; x[1] = tt; x[2] = tb;
                f[0] = tf[0]; f[1] = tf[1]; f[2] = tf[2];
                accepted = true;
                break;
            }
        }
        if (!accepted) return false;
    }
    return false;
}

// Stability of a converged candidate at (p, T) with liquid mass `mass`
// (`known`: the gas table's terms at exactly (p, T), if the caller has them).
// The stability test of an all-gas state at (p, T) with its gas point `g`
// decided without evaluating the liquid root, where the outcome is provably
// "stable": p lies 1e-6 of it below the saturation pressure tabulated at the
// table temperature one below T's cell (the saturation pressure rises with T,
// and the table's pressures, from a 160-step bisection to |mu_l - mu_g| <=
// 1e-9 RT, are off by less than 1e-7 where the phases' Z differ by 0.05 or
// more), so a liquid root has the larger chemical potential by far more than
// rounding (the affinity is positive, above -mutol); and the liquid root, when
// the cubic has one, lies at least 1e-6 of its volume below the middle root,
// so its evaluation succeeds (dp/dV < 0 off the spinodal, cv > 0 with the PR
// attraction term) or the root is not a liquid by the reported-phase line
// (unavailable, also stable). T at or above the table's start is at or above
// the liquid range's lower end, where the full test would fail the candidate.
__device__ __forceinline__ bool gasStableBelowSaturation(const HemConst& C, double p, double T, const GasPoint& g) {
    if (!C.domeN || C.satN < 2 || !(T >= C.satT0)) return false;
    const double cell = floor((T - C.satT0) * C.satInvStep) - 1;
    if (!(cell >= 0) || !(cell < C.satN)) return false;
    const double ps = C.satP[int(cell)];
    if (!(p < ps * (1 - 1e-6))) return false;
    if (!g.roots) return g.clear;
    if (!g.r.liquid) return true;  // no liquid root: unavailable, stable
    if (g.r.count != 3) return false;
    const double mid = -(C.gas.b - kGas * T / p) - g.r.lo - g.r.hi;  // the roots sum to -bn
    return mid - g.r.lo > 1e-6 * mid;
}

__device__ RB200_FLASH_FN bool stableAt(const HemConst& C, double q, double mass, double p, double T, Counts& n,
                                const GasPoint* known = nullptr) {
    if (q - mass > 0) {
        if (mass == 0 && known && gasStableBelowSaturation(C, p, T, *known)) return true;
        Eval cmp;
        if (!evaluate(C, q, mass, p, T, true, cmp, n, known)) return false;
        const double affinity = cmp.muL - cmp.muG;
        if (mass > 0) return fin(affinity) && fabs(affinity) <= C.mutol * 2;
        return !(affinity < -C.mutol);
    }
    if (!(mass > 0)) return false;
    PhaseProps liq, gas;
    if (liquidPhase(C, p, T, true, liq, n) != EOS_OK) return false;
    const double muL = liq.mu / (kGas * T);
    const int status = gasPhase(C, p, T, false, gas, n);
    if (status != EOS_OK) return unavailableStatus(status);  // no gas branch: +inf tangent, stable
    const double tangent = (gas.h - T * gas.s) * C.gas.W / (kGas * T) - muL;
    return tangent >= -C.mutol;
}

// Final state of a converged candidate (the reference's ReactiveThermoState
// fields, src/reactiveThermo/reactiveThermo.h:11-19).
__device__ inline void stateFromEval(const Eval& v, double q, const CandidateOut& o, ReactiveThermoState& s) {
    s.p = v.p;
    s.T = v.T;
    s.rho = q;
    s.e = v.energy / q;
    s.entropy = v.entropyD / q;
    s.soundFrozen = v.soundFrozen;
    s.soundEquilibrium = o.soundEq;
    s.volumeResidual = o.vres;
    s.energyResidual = o.eres;
    s.chemicalResidual = o.cres;
    s.alphaGas = v.gasMass > 0 ? v.gasMass / v.gRho : 0;
    s.alphaLiquid[0] = v.liqMass > 0 ? v.liqMass / v.lRho : 0;
    s.alphaLiquid[1] = 0;
    s.rhoGas = v.gasMass > 0 ? v.gRho : 0;
    s.rhoLiquid[0] = v.liqMass > 0 ? v.lRho : 0;
    s.rhoLiquid[1] = 0;
    s.liquidMass[0] = v.liqMass;
    s.liquidMass[1] = 0;
    s.gasMass = v.gasMass;
    s.cp = v.cpD / q;
    s.cv = v.cv;
    s.activeLiquids = v.liqMass > 0 ? 1 : 0;
    s.iterations = o.iterations;
}

}  // namespace rb200
