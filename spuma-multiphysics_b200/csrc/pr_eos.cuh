// Peng-Robinson equation of state of one pure species on the device (FP64).
//
// Thermodynamic relations (Cantera 3.2 conventions, as restated by the
// reference in src/reactiveThermo/reactiveDevicePR.h): NASA7/9 ideal-gas part
// (:127-155, region choice :198-212), alpha(T) and its T-derivatives (:214-247),
// cubic Z roots with the absolute near-repeated-root band and the isolated third
// root (:280-307, :333-422), residual (T, rho) properties and chemical potential
// (:474-562), root choice at (T, p) and the pressure postcondition (:575-609),
// and the reported-phase line through (Tc, rho_c) (:429-471) precomputed once
// per table (src/reactiveThermo/reactiveDevicePRPurePhaseCache.h:29-85).
//
// The root solve and root selection stay FP64: the discriminant thresholds are
// absolute and the near-repeated band decides phase availability.
#pragma once
#include <cuda_runtime.h>
#include <cfloat>

// Linkage of the large EOS routines. Out of line (one copy each in the binary)
// keeps the instruction footprint of the flash kernels small: their warps run
// different solver states side by side, and with every call site expanded the
// code no longer fits the instruction cache.
#ifndef RB200_EOS_FN
#define RB200_EOS_FN static __noinline__
#endif

namespace rb200 {

constexpr double kGas = 8314.46261815324;  // J/(kmol K)
constexpr double kSqrt2 = 1.41421356237309504880168872420969808;
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kOmegaA = 4.5723552892138218e-1;
constexpr double kOmegaB = 7.77960739038885e-2;
constexpr double kOmegaVc = 3.07401308698703833e-1;

enum EosStatus : int {
    EOS_OK = 0, EOS_INVALID_TABLE, EOS_INVALID_INPUT, EOS_INVALID_COMPOSITION, EOS_NO_ROOT,
    EOS_UNAVAILABLE, EOS_UNSTABLE, EOS_NONFINITE
};
enum RootChoice : int { ROOT_AUTO = 0, ROOT_GAS = 1, ROOT_LIQUID = 2 };

constexpr int kMaxRegions = 8;

// Immutable per-species constants, derived on the host from the model image.
struct PureSpecies {
    double a, b, kappa, W, Tc, refP;
    double tcLine, rhoC, dRho, dT;  // reported-phase line
    double invW, invL, invL2;       // 1/W, 1/(2 sqrt2 b), 1/(2 sqrt2 b^2)
    double invTc, vc;               // 1/Tc; critical molar volume of the cubic (single-root side test)
    double invRefP;                 // 1/reference pressure
    int regionCount;
    int polynomial[kMaxRegions];
    double regionMin[kMaxRegions];
    double regionMaxLast;
    double coeff[kMaxRegions][9];
};

struct PhaseProps {
    double p, rho, e, s, cp, cv, alpha, kappaT, V, h, mu;  // per mass except V (molar), mu (molar)
};

__device__ __forceinline__ bool fin(double x) { return isfinite(x); }

__device__ __forceinline__ int nasaRegion(const PureSpecies& sp, double T) {
    int r = 0;
    for (int j = 1; j < sp.regionCount; ++j) {
        const double b = sp.regionMin[j];
        const bool high = sp.polynomial[j] == 9 ? T >= b : T > b;
        if (!high) break;
        r = j;
    }
    return r;
}

constexpr double kThird = 1.0 / 3.0;

// NASA7/9 cp/R, h/RT, s/R at T (iT = 1/T), thirds as products (the PR T-terms).
__device__ __forceinline__ void nasaEvalT(const PureSpecies& sp, double T, double iT, double& cpR, double& hRT,
                                          double& sR) {
    const int r = nasaRegion(sp, T);
    const double* a = sp.coeff[r];
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, lT = log(T);
    if (sp.polynomial[r] == 7) {
        cpR = a[0] + a[1] * T + a[2] * T2 + a[3] * T3 + a[4] * T4;
        hRT = a[0] + .5 * a[1] * T + a[2] * T2 * kThird + .25 * a[3] * T3 + .2 * a[4] * T4 + a[5] * iT;
        sR = a[0] * lT + a[1] * T + .5 * a[2] * T2 + a[3] * T3 * kThird + .25 * a[4] * T4 + a[6];
    } else {
        const double c0 = a[0] * iT * iT, c1 = a[1] * iT, c2 = a[2], c3 = a[3] * T, c4 = a[4] * T2,
                     c5 = a[5] * T3, c6 = a[6] * T4;
        cpR = c0 + c1 + c2 + c3 + c4 + c5 + c6;
        hRT = -c0 + lT * c1 + c2 + .5 * c3 + c4 * kThird + .25 * c5 + .2 * c6 + a[7] * iT;
        sR = -.5 * c0 - c1 + lT * c2 + c3 + .5 * c4 + c5 * kThird + .25 * c6 + a[8];
    }
}
// NASA7/9 cp/R, h/RT, s/R at T (the ideal-gas closure's form).
__device__ __forceinline__ void nasaEval(const PureSpecies& sp, double T, double& cpR, double& hRT, double& sR) {
    const int r = nasaRegion(sp, T);
    const double* a = sp.coeff[r];
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, iT = 1.0 / T, lT = log(T);
    if (sp.polynomial[r] == 7) {
        cpR = a[0] + a[1] * T + a[2] * T2 + a[3] * T3 + a[4] * T4;
        hRT = a[0] + .5 * a[1] * T + a[2] * T2 / 3.0 + .25 * a[3] * T3 + .2 * a[4] * T4 + a[5] * iT;
        sR = a[0] * lT + a[1] * T + .5 * a[2] * T2 + a[3] * T3 / 3.0 + .25 * a[4] * T4 + a[6];
    } else {
        const double c0 = a[0] * iT * iT, c1 = a[1] * iT, c2 = a[2], c3 = a[3] * T, c4 = a[4] * T2,
                     c5 = a[5] * T3, c6 = a[6] * T4;
        cpR = c0 + c1 + c2 + c3 + c4 + c5 + c6;
        hRT = -c0 + lT * c1 + c2 + .5 * c3 + c4 / 3.0 + .25 * c5 + .2 * c6 + a[7] * iT;
        sR = -.5 * c0 - c1 + lT * c2 + c3 + .5 * c4 + c5 / 3.0 + .25 * c6 + a[8];
    }
}

__device__ __forceinline__ double cubicAt(double V, double bn, double cn, double dn) {
    return ((V + bn) * V + cn) * V + dn;
}

// Physical roots (finite, above the covolume), smallest and largest.
struct Roots {
    double lo, hi;
    int count;
    bool gas, liquid;
};

__device__ inline bool isolatedRoot(double center, double delta, double delta2, double q, double bn, double cn,
                                    double dn, double b, double RTp, double aap, double& root, bool& gasSide) {
    if (!(delta2 > 0) || !fin(delta) || !fin(q) || q == 0) return false;
    gasSide = q < 0;
    const double pair = center + (gasSide ? -1.0 : 1.0) * delta;
    double x = center + (gasSide ? 2.0 : -2.0) * delta;
    bool converged = false;
    for (int n = 0; n < 24; ++n) {
        const double f = cubicAt(x, bn, cn, dn), df = (3.0 * x + 2.0 * bn) * x + cn;
        if (!fin(f) || !fin(df) || fabs(df) <= 1e-300) return false;
        const double step = f / df;
        x -= step;
        if (fabs(step) <= 4e-15 * fmax(1.0, fabs(x))) { converged = true; break; }
    }
    if (!converged || !fin(x) || !(x > b)) return false;
    const double f = cubicAt(x, bn, cn, dn);
    const double scale = fabs(x * x * x) + fabs(bn * x * x) + fabs(cn * x) + fabs(dn);
    if (!(fabs(f) <= 64.0 * DBL_EPSILON * scale)) return false;
    if (!(fabs(x - pair) > 1e-3 * fmax(fabs(x), fabs(pair)))) return false;
    if (gasSide ? !(x > pair) : !(x < pair)) return false;
    const double vb = x - b, den = x * x + 2.0 * b * x - b * b;
    if (!(vb > 0) || !(den > 0)) return false;
    if (!(-RTp / (vb * vb) + 2.0 * aap * (x + b) / (den * den) < 0)) return false;
    root = x;
    return true;
}

__device__ __forceinline__ double signedCbrt(double x) { return cbrt(x); }

// Twelve Newton polishing steps on the cubic (stops early on a tiny step).
__device__ __forceinline__ double polishRoot(double x, double bn, double cn, double dn) {
    for (int n = 0; n < 12; ++n) {
        const double res = cubicAt(x, bn, cn, dn), d = (3.0 * x + 2.0 * bn) * x + cn;
        if (fabs(d) <= 1e-300) break;
        const double step = res / d;
        x -= step;
        if (fabs(step) <= 4e-15 * fmax(1.0, fabs(x))) break;
    }
    return x;
}

__device__ __forceinline__ int cubicRootsBody(const PureSpecies& sp, double T, double p, double aa, Roots& r) {
    const double ip = 1.0 / p;
    const double b = sp.b, b2 = b * b, RTp = kGas * T * ip, aap = aa * ip, bn = b - RTp;
    const double cn = -(2.0 * RTp * b - aap + 3.0 * b2), dn = b2 * RTp + b2 * b - aap * b;
    const double center = -bn * kThird, delta2 = (bn * bn - 3.0 * cn) * (1.0 / 9.0);
    const double q = 2.0 * bn * bn * bn * (1.0 / 27.0) - bn * cn * kThird + dn;
    const double delta = delta2 > 0 ? sqrt(delta2) : 0.0, h = 2.0 * delta * delta2;
    double disc = q * q - h * h;
    if (fabs(fabs(h) - fabs(q)) < 1e-10) {
        if (disc > 1e-10) return EOS_NONFINITE;
        disc = 0;
    }
    double raw0 = 0, raw1 = 0, raw2 = 0;
    int rawCount;
    int side = 0;
    if (fabs(disc) < 1e-14) {
        bool gasSide = false;
        if (!isolatedRoot(center, delta, delta2, q, bn, cn, dn, b, RTp, aap, raw0, gasSide)) return EOS_NO_ROOT;
        rawCount = 1;
        side = gasSide ? 1 : -1;
    } else if (disc > 1e-14 || !(delta2 > 0)) {
        const double sd = .5 * sqrt(fmax(0.0, disc));
        raw0 = center + signedCbrt(-.5 * q + sd) + signedCbrt(-.5 * q - sd);
        rawCount = 1;
    } else if (disc < -1e-14) {
        const double arg = fmin(1.0, fmax(-1.0, -.5 * q / (delta * delta * delta)));
        // 2 delta cos(theta + 2 pi k / 3), k = 0, 1, 2, from one sine and cosine:
        // cos(theta +- 2 pi / 3) = -cos(theta) / 2 -+ sqrt3 / 2 sin(theta)
        double sn, cs;
        sincos(acos(arg) * kThird, &sn, &cs);
        const double dc = delta * cs, ds = 1.7320508075688772 * delta * sn;
        raw0 = center + 2.0 * dc;
        raw1 = center - dc - ds;
        raw2 = center - dc + ds;
        rawCount = 3;
    } else return EOS_NO_ROOT;
    if (!side) {
        raw0 = polishRoot(raw0, bn, cn, dn);
        if (rawCount == 3) {
            raw1 = polishRoot(raw1, bn, cn, dn);
            raw2 = polishRoot(raw2, bn, cn, dn);
            double t;
            if (raw0 > raw1) { t = raw0; raw0 = raw1; raw1 = t; }
            if (raw1 > raw2) { t = raw1; raw1 = raw2; raw2 = t; }
            if (raw0 > raw1) { t = raw0; raw0 = raw1; raw1 = t; }
        }
    }
    const bool ok0 = fin(raw0) && raw0 > b;
    const bool ok1 = rawCount == 3 && fin(raw1) && raw1 > b;
    const bool ok2 = rawCount == 3 && fin(raw2) && raw2 > b;
    const int n = int(ok0) + int(ok1) + int(ok2);
    if (!n) return EOS_NO_ROOT;
    r.count = n;
    r.lo = ok0 ? raw0 : (ok1 ? raw1 : raw2);
    r.hi = ok2 ? raw2 : (ok1 ? raw1 : raw0);
    if (side) {
        r.gas = side > 0;
        r.liquid = side < 0;
    } else if (n >= 2) {
        r.gas = r.liquid = true;
    } else {
        const bool liquidSign = T > sp.Tc ? r.lo < sp.vc : r.lo < center;
        r.liquid = liquidSign;
        r.gas = !liquidSign || T > sp.Tc;
    }
    return EOS_OK;
}
__device__ RB200_EOS_FN int cubicRoots(const PureSpecies& sp, double T, double p, double aa, Roots& r) {
    return cubicRootsBody(sp, T, p, aa, r);
}

// Temperature-only terms shared by every evaluation at one T: a*alpha and its
// T-derivatives, |1 + kappa(1 - sqrt(T/Tc))|, and the NASA cp/R, h/RT, s/R.
struct TTerms {
    double T, aa, da, d2a, q, cpR, hRT, sR;
};

__device__ __forceinline__ int tTermsBody(const PureSpecies& sp, double T, TTerms& t) {
    if (!fin(T) || T <= 0) return EOS_INVALID_INPUT;
    const double iT = 1.0 / T;
    const double sq = sqrt(T * sp.invTc), f = 1.0 + sp.kappa * (1.0 - sq);
    if (fabs(f) <= 1e-14) return EOS_NONFINITE;
    const double sign = f > 0 ? 1.0 : -1.0, q = fabs(f);
    // dq/dT = -kappa / (2 Tc sqrt(T/Tc)) and d2q/dT2 = -dq/dT / (2 T) (Tc sq^2 = T)
    const double dq = -sign * sp.kappa * (.5 * sp.invTc) / sq;
    const double d2q = -.5 * dq * iT;
    t.T = T;
    t.q = q;
    t.aa = sp.a * q * q;
    t.da = sp.a * (dq * q + q * dq);
    t.d2a = sp.a * (d2q * q + 2.0 * dq * dq + q * d2q);
    if (!(fin(t.aa) && fin(t.da) && fin(t.d2a) && t.aa > 0)) return EOS_NONFINITE;
    nasaEvalT(sp, T, iT, t.cpR, t.hRT, t.sR);
    return EOS_OK;
}
__device__ RB200_EOS_FN int tTerms(const PureSpecies& sp, double T, TTerms& t) {
    return tTermsBody(sp, T, t);
}

// The intermediates of a (T, rho) evaluation that its chemical potential reads:
// 1/(V - b), 1/den, ln(RT / (pref (V - b))) and the attraction logarithm.
struct ChemTerms {
    double iv, id, lg, logRatio;
};

// Molar chemical potential at molar volume V from the T-terms and the
// evaluation's intermediates (one routine, so every caller forms the same bits).
__device__ __forceinline__ double chemPotential(const PureSpecies& sp, const TTerms& t, double V, const ChemTerms& c) {
    const double RT = kGas * t.T, b = sp.b, aa = t.aa;
    const double pp = sp.a * (t.q * t.q), num = 2.0 * b * pp - aa * b;
    return RT * (t.hRT - t.sR) + RT * c.lg + RT * b * c.iv - num * sp.invL2 * c.logRatio - aa * V * c.id;
}

// Properties at (T, rho) from the T-only terms. chem: also the molar chemical
// potential. phaseOut: -2 supercritical, -1 gas, 0 liquid by the reported-phase line.
// keep (optional): the chemical potential's intermediates, on success.
__device__ __forceinline__ int prTrhoTBody(const PureSpecies& sp, const TTerms& t, double rho, bool chem, PhaseProps& s,
                              int& phaseOut, ChemTerms* keep) {
    const double T = t.T, aa = t.aa, da = t.da, d2a = t.d2a;
    if (!fin(rho) || rho <= 0) return EOS_INVALID_INPUT;
    const double b = sp.b, W = sp.W, V = W / rho;
    if (!(V > b)) return EOS_NO_ROOT;
    const double den = V * V + 2.0 * V * b - b * b, vmb = V - b;
    if (!(den > 0) || !(vmb > 0)) return EOS_NO_ROOT;
    // one reciprocal per repeated denominator (1/(V-b), 1/den, 1/W, 1/V, 1/dp/dV)
    const double RT = kGas * T, iv = 1.0 / vmb, id = 1.0 / den, iW = sp.invW, iV = rho * iW;
    const double p = RT * iv - aa * id;
    if (!fin(p) || p <= 0) return EOS_NO_ROOT;
    const double dpdV = -RT * (iv * iv) + 2.0 * aa * (V + b) * (id * id);
    const double dpdT = kGas * iv - da * id;
    if (!fin(dpdV) || !fin(dpdT) || dpdV >= 0) return EOS_UNSTABLE;
    const double idp = 1.0 / dpdV;
    const double logRatio = log((V + (1.0 + kSqrt2) * b) / (V + (1.0 - kSqrt2) * b));
    const double L = logRatio * sp.invL;
    const double z = p * V / RT;
    // ln(p/pref) - ln z(1 - b/V) = ln(RT / (pref (V - b))): the ideal-gas and residual
    // logarithms of the entropy (and of the chemical potential) as one
    const double lg = log(RT * iv * sp.invRefP);
    const double hM = RT * t.hRT + (RT * (z - 1.0) + L * (T * da - aa));
    const double sM = kGas * (t.sR - lg) + L * da;
    const double dHdT = kGas * t.cpR + V * dpdT - kGas + L * T * d2a;
    const double cpM = dHdT - (V + T * dpdT * idp) * dpdT;
    const double cvM = cpM + T * dpdT * dpdT * idp;
    s.p = p;
    s.rho = rho;
    s.V = V;
    s.h = hM * iW;
    s.e = (hM - p * V) * iW;
    s.s = sM * iW;
    s.cp = cpM * iW;
    s.cv = cvM * iW;
    s.alpha = -dpdT * idp * iV;
    s.kappaT = -idp * iV;
    const double sound2 = V * V * (-cpM / cvM * dpdV * iW);
    if (!(s.cp > 0) || !(s.cv > 0) || !(s.kappaT > 0) || !(sound2 > 0)) return EOS_UNSTABLE;
    const ChemTerms ct{iv, id, lg, logRatio};
    if (chem) {
        s.mu = chemPotential(sp, t, V, ct);
        if (!fin(s.mu)) return EOS_NONFINITE;
    }
    if (T >= sp.tcLine) phaseOut = -2;
    else {
        const double rhoMid = sp.rhoC + (T - sp.tcLine) * sp.dRho / sp.dT;
        if (!fin(rhoMid)) return EOS_NONFINITE;
        phaseOut = rho < rhoMid ? -1 : 0;
    }
    // (sound2 > 0 here, so its square root is finite exactly when sound2 is)
    if (!fin(s.e) || !fin(s.h) || !fin(s.s) || !fin(s.cp) || !fin(s.cv) || !fin(s.alpha) || !fin(s.kappaT)
        || !fin(sound2) || !fin(dpdT) || !fin(dpdV))
        return EOS_NONFINITE;
    if (keep) *keep = ct;
    return EOS_OK;
}
__device__ RB200_EOS_FN int prTrhoT(const PureSpecies& sp, const TTerms& t, double rho, bool chem, PhaseProps& s,
                              int& phaseOut, ChemTerms* keep = nullptr) {
    return prTrhoTBody(sp, t, rho, chem, s, phaseOut, keep);
}

__device__ RB200_EOS_FN int prTrho(const PureSpecies& sp, double T, double rho, bool chem, PhaseProps& s, int& phaseOut) {
    if (!fin(T) || !fin(rho) || T <= 0 || rho <= 0) return EOS_INVALID_INPUT;
    TTerms t;
    const int st = tTerms(sp, T, t);
    if (st != EOS_OK) return st;
    return prTrhoT(sp, t, rho, chem, s, phaseOut);
}

// Root choice at (T, p) with the host postcondition |p(T, rho) - p| <= 1e-7 max(1, p)
// and the reported-phase consistency of the chosen branch.
__device__ __forceinline__ int rootPropsBody(const PureSpecies& sp, const TTerms& t, const Roots& r, double p, int choice,
                                bool chem, PhaseProps& s, ChemTerms* keep) {
    int sel = r.count - 1;
    if (choice == ROOT_LIQUID) {
        if (!r.liquid) return EOS_UNAVAILABLE;
        sel = 0;
    } else if (choice == ROOT_GAS && !r.gas) return EOS_UNAVAILABLE;
    const double V = sel == 0 ? r.lo : r.hi;
    int phase = 0;
    const int st = prTrhoTBody(sp, t, sp.W / V, chem, s, phase, keep);
    if (st != EOS_OK) return st;
    if (fabs(s.p - p) > 1e-7 * fmax(1.0, p)) return EOS_NONFINITE;
    s.p = p;
    if (choice == ROOT_GAS && phase >= 0) return EOS_UNAVAILABLE;
    if (choice == ROOT_LIQUID && phase < 0) return EOS_UNAVAILABLE;
    return EOS_OK;
}
__device__ RB200_EOS_FN int rootProps(const PureSpecies& sp, const TTerms& t, const Roots& r, double p, int choice,
                                bool chem, PhaseProps& s, ChemTerms* keep = nullptr) {
    return rootPropsBody(sp, t, r, p, choice, chem, s, keep);
}

__device__ RB200_EOS_FN int prTP(const PureSpecies& sp, double T, double p, int choice, bool chem, PhaseProps& s) {
    if (!fin(T) || !fin(p) || T <= 0 || p <= 0) return EOS_INVALID_INPUT;
    TTerms t;
    int st = tTerms(sp, T, t);
    if (st != EOS_OK) return st;
    Roots r;
    st = cubicRoots(sp, T, p, t.aa, r);
    if (st != EOS_OK) return st;
    return rootProps(sp, t, r, p, choice, chem, s);
}

}  // namespace rb200
