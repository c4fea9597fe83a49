// Peng-Robinson mixture properties at (T, rho, Y) and (T, p, Y): the building
// block of the multi-species (air / N2O / isopropanol) flash. Host and device
// code from one source.
//
// Relations restated from the reference's mixture evaluator
// (src/reactiveThermo/reactiveDevicePR.h): mass to mole fractions (:313-330),
// the van der Waals one-fluid mixing of a*alpha with its T-derivatives and
// b = sum x_i b_i (:214-247), NASA7/9 ideal-gas terms with the region choice
// (:127-155, :197-212), the cubic's roots with the absolute near-repeated band and
// the isolated third root (:280-307, :333-422), residual properties, the ideal
// mixing entropy and the species chemical potentials (:474-562), the
// composition-dependent reported-phase line (:429-471), and the root choice at
// (T, p) with its pressure postcondition (:575-609).
#pragma once
#include <cfloat>
#include <cmath>
#include "../../include/reactive_b200_types.h"

#ifdef __CUDACC__
#define RB200_HD __host__ __device__
#else
#define RB200_HD
#endif

namespace rb200 {
namespace mix {

constexpr int kMaxNs = 4;  // species of one mixture evaluation (the air / N2O / isopropanol case)
constexpr double kR = 8314.46261815324;
constexpr double kRt2 = 1.41421356237309504880168872420969808;
constexpr double kOmA = 4.5723552892138218e-1;
constexpr double kOmB = 7.77960739038885e-2;
constexpr double kOmVc = 3.07401308698703833e-1;

enum Status : int { OK = 0, BAD_TABLE, BAD_INPUT, BAD_COMPOSITION, NO_ROOT, UNAVAILABLE, UNSTABLE, NONFINITE };
enum Choice : int { AUTO = 0, GAS = 1, LIQUID = 2 };
enum Label : int { SUPERCRITICAL = -2, GASLIKE = -1, LIQUIDLIKE = 0 };

struct Props {
    double T, p, W, V, rho, e, h, s, cp, cv, alpha, kappaT, sound, dpdT, dpdV;
    double mu[kMaxNs];  // J/kmol
    int phase;          // Label
};

RB200_HD inline bool finiteD(double x) { return x == x && fabs(x) <= DBL_MAX; }

// Mole fractions and molar mass of the mass fractions Y (sum within 1e-12 of 1).
RB200_HD inline int moles(const ReactiveB200Table& t, const double* Y, double* x, double& W) {
    if (t.ns < 1 || t.ns > kMaxNs) return BAD_TABLE;
    double sumY = 0, perW = 0;
    for (int k = 0; k < t.ns; ++k) {
        if (!finiteD(Y[k]) || Y[k] < 0) return BAD_COMPOSITION;
        sumY += Y[k];
        perW += Y[k] / t.species[k].molecularWeight;
    }
    if (!(perW > 0) || fabs(sumY - 1.0) > 1e-12) return BAD_COMPOSITION;
    W = 1.0 / perW;
    for (int k = 0; k < t.ns; ++k) x[k] = Y[k] * W / t.species[k].molecularWeight;
    return OK;
}

// NASA7/9 cp/R, h/RT, s/R of species k at T.
RB200_HD inline void nasa(const ReactiveB200Species& sp, double T, double& cpR, double& hRT, double& sR) {
    int r = 0;
    for (int j = 1; j < sp.regionCount; ++j) {
        const double edge = sp.regions[j].minimumTemperature;
        if (!(sp.regions[j].polynomial == 9 ? T >= edge : T > edge)) break;
        r = j;
    }
    const double* a = sp.regions[r].coefficient;
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, iT = 1.0 / T, lT = log(T);
    if (sp.regions[r].polynomial == 7) {
        cpR = a[0] + a[1] * T + a[2] * T2 + a[3] * T3 + a[4] * T4;
        hRT = a[0] + .5 * a[1] * T + a[2] * T2 / 3.0 + .25 * a[3] * T3 + .2 * a[4] * T4 + a[5] * iT;
        sR = a[0] * lT + a[1] * T + .5 * a[2] * T2 + a[3] * T3 / 3.0 + .25 * a[4] * T4 + a[6];
    } else {
        const double c0 = a[0] * iT * iT, c1 = a[1] * iT, c3 = a[3] * T, c4 = a[4] * T2, c5 = a[5] * T3,
                     c6 = a[6] * T4;
        cpR = c0 + c1 + a[2] + c3 + c4 + c5 + c6;
        hRT = -c0 + lT * c1 + a[2] + .5 * c3 + c4 / 3.0 + .25 * c5 + .2 * c6 + a[7] * iT;
        sR = -.5 * c0 - c1 + lT * a[2] + c3 + .5 * c4 + c5 / 3.0 + .25 * c6 + a[8];
    }
}

// One-fluid mixing at T: a = sum x_i x_j a_ij, b = sum x_i b_i, a*alpha and its
// T-derivatives, and each species' |1 + kappa (1 - sqrt(T/Tc))| for the chemical
// potentials.
struct Mixing {
    double a, b, aa, da, d2a;
    double q[kMaxNs];
};

RB200_HD inline int mixing(const ReactiveB200Table& t, double T, const double* x, Mixing& m) {
    double dq[kMaxNs], d2q[kMaxNs];
    m.a = m.b = m.aa = m.da = m.d2a = 0;
    for (int i = 0; i < t.ns; ++i) {
        const ReactiveB200Species& sp = t.species[i];
        const double Tc = sp.a * kOmB / (sp.b * kOmA * kR);
        if (!(Tc > 0) || !finiteD(Tc)) return BAD_TABLE;
        const double root = sqrt(T / Tc), f = 1.0 + sp.kappa * (1.0 - root);
        if (fabs(f) <= 1e-14) return NONFINITE;  // the cusp of |f|: no T-derivatives
        const double sign = f > 0 ? 1.0 : -1.0;
        m.q[i] = fabs(f);
        dq[i] = -sign * sp.kappa / (2.0 * Tc * root);
        d2q[i] = sign * sp.kappa / (4.0 * Tc * Tc * root * root * root);
        m.b += x[i] * sp.b;
    }
    for (int i = 0; i < t.ns; ++i)
        for (int j = 0; j < t.ns; ++j) {
            const double w = x[i] * x[j] * t.aBinary[i][j];
            m.a += w;
            m.aa += w * m.q[i] * m.q[j];
            m.da += w * (dq[i] * m.q[j] + m.q[i] * dq[j]);
            m.d2a += w * (d2q[i] * m.q[j] + 2.0 * dq[i] * dq[j] + m.q[i] * d2q[j]);
        }
    const bool good = finiteD(m.a) && finiteD(m.b) && finiteD(m.aa) && finiteD(m.da) && finiteD(m.d2a);
    return good && m.a > 0 && m.b > 0 && m.aa > 0 ? OK : NONFINITE;
}

struct Roots {
    double V[3];  // ascending physical molar volumes (> b)
    int count, signedCount;
    bool gas, liquid;
};

RB200_HD inline double cubic(double V, double bn, double cn, double dn) { return ((V + bn) * V + cn) * V + dn; }

// Roots of the PR cubic in V at (T, p) for mixture terms m (Cantera's signed root
// count: 3, 2, +1 gas side, -1 liquid side).
RB200_HD inline int roots(const Mixing& m, double T, double p, Roots& r) {
    const double b = m.b, b2 = b * b, RTp = kR * T / p, aap = m.aa / p, bn = b - RTp;
    const double cn = -(2.0 * RTp * b - aap + 3.0 * b2), dn = b2 * RTp + b2 * b - aap * b;
    const double center = -bn / 3.0, delta2 = (bn * bn - 3.0 * cn) / 9.0;
    const double q = 2.0 * bn * bn * bn / 27.0 - bn * cn / 3.0 + dn;
    const double delta = delta2 > 0 ? sqrt(delta2) : 0.0, h = 2.0 * delta * delta2;
    double disc = q * q - h * h;
    if (fabs(fabs(h) - fabs(q)) < 1e-10) {
        if (disc > 1e-10) return NONFINITE;
        disc = 0;
    }
    double v[3] = {0, 0, 0};
    int raw = 0, side = 0;
    if (fabs(disc) < 1e-14) {
        // near-repeated pair: only a separated, refined, stable third root
        if (!(delta2 > 0) || !finiteD(delta) || !finiteD(q) || q == 0) return NO_ROOT;
        const bool gasSide = q < 0;
        const double pair = center + (gasSide ? -1.0 : 1.0) * delta;
        double x = center + (gasSide ? 2.0 : -2.0) * delta;
        bool done = false;
        for (int it = 0; it < 24 && !done; ++it) {
            const double f = cubic(x, bn, cn, dn), d = (3.0 * x + 2.0 * bn) * x + cn;
            if (!finiteD(f) || !finiteD(d) || fabs(d) <= 1e-300) return NO_ROOT;
            const double step = f / d;
            x -= step;
            done = fabs(step) <= 4e-15 * fmax(1.0, fabs(x));
        }
        const double vb = x - b, den = x * x + 2.0 * b * x - b * b;
        const double scale = fabs(x * x * x) + fabs(bn * x * x) + fabs(cn * x) + fabs(dn);
        if (!done || !finiteD(x) || !(x > b) || !(fabs(cubic(x, bn, cn, dn)) <= 64.0 * DBL_EPSILON * scale)
            || !(fabs(x - pair) > 1e-3 * fmax(fabs(x), fabs(pair))) || (gasSide ? !(x > pair) : !(x < pair))
            || !(vb > 0) || !(den > 0) || !(-RTp / (vb * vb) + 2.0 * aap * (x + b) / (den * den) < 0))
            return NO_ROOT;
        v[0] = x;
        raw = 1;
        side = gasSide ? 1 : -1;
    } else if (disc > 1e-14 || !(delta2 > 0)) {
        const double sd = .5 * sqrt(fmax(0.0, disc));
        v[0] = center + cbrt(-.5 * q + sd) + cbrt(-.5 * q - sd);
        raw = 1;
    } else if (disc < -1e-14) {
        const double theta = acos(fmin(1.0, fmax(-1.0, -.5 * q / (delta * delta * delta)))) / 3.0;
        const double c = cos(theta), s = sin(theta);
        v[0] = center + 2.0 * delta * c;
        v[1] = center - delta * c - 1.7320508075688772 * delta * s;  // cos(theta + 2 pi / 3)
        v[2] = center - delta * c + 1.7320508075688772 * delta * s;  // cos(theta + 4 pi / 3)
        raw = 3;
    } else return NO_ROOT;
    if (!side)
        for (int i = 0; i < raw; ++i)
            for (int it = 0; it < 12; ++it) {
                const double d = (3.0 * v[i] + 2.0 * bn) * v[i] + cn;
                if (fabs(d) <= 1e-300) break;
                const double step = cubic(v[i], bn, cn, dn) / d;
                v[i] -= step;
                if (fabs(step) <= 4e-15 * fmax(1.0, fabs(v[i]))) break;
            }
    for (int i = 1; i < raw; ++i)  // ascending
        for (int j = i; j > 0 && v[j - 1] > v[j]; --j) {
            const double tmp = v[j];
            v[j] = v[j - 1];
            v[j - 1] = tmp;
        }
    r.count = 0;
    for (int i = 0; i < raw; ++i)
        if (finiteD(v[i]) && v[i] > b) r.V[r.count++] = v[i];
    if (!r.count) return NO_ROOT;
    const double Tcm = m.a * kOmB / (b * kOmA * kR);
    const double pc = kOmB * kR * Tcm / b, vc = kOmVc * kR * Tcm / pc;
    if (side) {
        r.signedCount = side;
        r.gas = side > 0;
        r.liquid = side < 0;
    } else if (r.count >= 2) {
        r.signedCount = r.count;
        r.gas = r.liquid = true;
    } else {
        const bool liquidSide = T > Tcm ? r.V[0] < vc : r.V[0] < center;
        r.signedCount = liquidSide ? -1 : 1;
        r.liquid = liquidSide;
        r.gas = !liquidSide || T > Tcm;
    }
    return OK;
}

// The reported phase of a mixture state (Cantera's density heuristic): above the
// mixture's pseudo-critical T supercritical; below it, gas-like when rho is under
// the line from the critical density to the mid density of the two roots at
// T_mid = Tc - 100 K (or Tc / 2), the pressure there raised by 4% until the cubic
// has both roots above pc or three roots (at most 100 cubic solves).
RB200_HD inline int reportedPhase(const ReactiveB200Table& t, double T, const double* x, double W, double rho,
                                  const Mixing& atT, int& phase) {
    const double tc = atT.a * kOmB / (atT.b * kOmA * kR), pc = kOmB * kR * tc / atT.b, vc = kOmVc * kR * tc / pc;
    if (T >= tc) {
        phase = SUPERCRITICAL;
        return OK;
    }
    const double tmid = tc - 100.0 < 0 ? .5 * tc : tc - 100.0, ratio = tc / tmid;
    double pp = pc * exp(-.8734 * ratio * ratio - 3.4522 * ratio + 4.2918), liquidV = -1;
    bool found = false;
    Mixing m;
    if (const int st = mixing(t, tmid, x, m)) return st;
    for (int it = 0; it < 100 && !found; ++it) {
        Roots r;
        if (const int st = roots(m, tmid, pp, r)) return st;
        liquidV = r.V[0];
        if (r.signedCount == 1 || r.signedCount == 2) {
            found = pp > pc;
            pp *= 1.04;
        } else found = true;
    }
    if (!found || !(liquidV > 0) || !finiteD(liquidV)) return NONFINITE;
    const double rhoC = W / vc, midT = .5 * (W / liquidV + W / (kR * tmid / pp));
    const double rhoMid = rhoC + (T - tc) * (rhoC - midT) / (tc - tmid);
    phase = rho < rhoMid ? GASLIKE : LIQUIDLIKE;
    return finiteD(rhoMid) ? OK : NONFINITE;
}

// Properties at (T, rho) and mass fractions Y; chem: the species chemical potentials.
RB200_HD inline int trho(const ReactiveB200Table& t, double T, double rho, const double* Y, bool chem, Props& s) {
    if (!finiteD(T) || !finiteD(rho) || T <= 0 || rho <= 0) return BAD_INPUT;
    double x[kMaxNs] = {}, W = 0;
    if (const int st = moles(t, Y, x, W)) return st;
    Mixing m;
    if (const int st = mixing(t, T, x, m)) return st;
    const double b = m.b, V = W / rho;
    if (!(V > b)) return NO_ROOT;
    const double den = V * V + 2.0 * V * b - b * b, vmb = V - b;
    if (!(den > 0) || !(vmb > 0)) return NO_ROOT;
    const double RT = kR * T;
    const double p = RT / vmb - m.aa / den;
    if (!finiteD(p) || p <= 0) return NO_ROOT;
    const double dpdV = -RT / (vmb * vmb) + 2.0 * m.aa * (V + b) / (den * den);
    const double dpdT = kR / vmb - m.da / den;
    if (!finiteD(dpdV) || !finiteD(dpdT) || dpdV >= 0) return UNSTABLE;
    const double logRatio = log((V + (1.0 + kRt2) * b) / (V + (1.0 - kRt2) * b));
    const double L = logRatio / (2.0 * kRt2 * b);
    double h0 = 0, s0 = 0, cp0 = 0, xlx = 0, hk[kMaxNs], sk[kMaxNs];
    for (int k = 0; k < t.ns; ++k) {
        double cpR, hRT, sR;
        nasa(t.species[k], T, cpR, hRT, sR);
        hk[k] = hRT;
        sk[k] = sR;
        cp0 += x[k] * kR * cpR;
        h0 += x[k] * RT * hRT;
        s0 += x[k] * kR * sR;
        if (x[k] > 0) xlx += x[k] * log(x[k]);
    }
    const double z = p * V / RT;
    const double hM = h0 + (RT * (z - 1.0) + L * (T * m.da - m.aa));
    const double sM = s0 - kR * xlx - kR * log(p / t.refPressure) + (kR * log(z * (1.0 - b / V)) + L * m.da);
    const double cvV = cp0 + V * dpdT - kR + L * T * m.d2a;  // dH/dT at constant V
    const double cpM = cvV - (V + T * dpdT / dpdV) * dpdT;
    const double cvM = cpM + T * dpdT * dpdT / dpdV;
    s.T = T; s.p = p; s.W = W; s.V = V; s.rho = rho;
    s.h = hM / W; s.e = (hM - p * V) / W; s.s = sM / W; s.cp = cpM / W; s.cv = cvM / W;
    s.alpha = -dpdT / (V * dpdV);
    s.kappaT = -1.0 / (V * dpdV);
    s.dpdT = dpdT;
    s.dpdV = dpdV;
    const double sound2 = V * V * (-cpM / cvM * dpdV / W);
    if (!(s.cp > 0) || !(s.cv > 0) || !(s.kappaT > 0) || !(sound2 > 0)) return UNSTABLE;
    s.sound = sqrt(sound2);
    if (chem) {
        for (int k = 0; k < t.ns; ++k) {
            double pp = 0;
            for (int i = 0; i < t.ns; ++i) pp += x[i] * t.aBinary[k][i] * (m.q[i] * m.q[k]);
            const double bk = t.species[k].b, num = 2.0 * b * pp - m.aa * bk;
            s.mu[k] = RT * (hk[k] - sk[k]) + RT * log(fmax(1e-300, x[k])) + RT * log(p / t.refPressure)
                    - RT * log(z) + RT * log(V / vmb) + RT * bk / vmb - num / (2.0 * kRt2 * b * b) * logRatio
                    - m.aa * bk * V / (b * den);
            if (!finiteD(s.mu[k])) return NONFINITE;
        }
    }
    if (const int st = reportedPhase(t, T, x, W, rho, m, s.phase)) return st;
    const double check[] = {s.e, s.h, s.s, s.cp, s.cv, s.alpha, s.kappaT, s.sound};
    for (double c : check)
        if (!finiteD(c)) return NONFINITE;
    return OK;
}

// Partial molar enthalpies [J/kmol] of the mixture of mass fractions Y at the
// state s (from trho / tp on the chosen root): the ideal-gas reference h_k(T)
// plus the Peng-Robinson departure at constant (T, p), h_k - T ds/dn_k terms
// through dp/dn_k at constant (T, V), the a*alpha composition derivative
// sum_i x_i a_ki sqrt(alpha_k alpha_i) and its T-derivative (the relations of
// Cantera 3.2's PengRobinsonPhase::getPartialMolarEnthalpies, which the
// reference's phasePartials restates, src/reactiveThermo/reactiveDeviceFlashJacobian.h:69-127).
RB200_HD inline int partialEnthalpies(const ReactiveB200Table& t, double T, const double* Y, const Props& s,
                                      double* hbar) {
    double x[kMaxNs] = {}, W = 0;
    if (const int st = moles(t, Y, x, W)) return st;
    Mixing m;
    if (const int st = mixing(t, T, x, m)) return st;
    const double V = s.V, RT = kR * T, b = m.b;
    const double vmb = V - b, den = V * V + 2.0 * V * b - b * b;
    if (!(vmb > 0) || !(den > 0) || !(s.dpdV < 0)) return NONFINITE;
    const double logRatio = log((V + (1.0 + kRt2) * b) / (V + (1.0 - kRt2) * b));
    const double L = logRatio / (2.0 * kRt2 * b);
    const double fac = T * m.da - m.aa, fac2 = V + T * s.dpdT / s.dpdV;
    double dq[kMaxNs];
    for (int i = 0; i < t.ns; ++i) {
        const ReactiveB200Species& sp = t.species[i];
        const double Tc = sp.a * kOmB / (sp.b * kOmA * kR), root = sqrt(T / Tc);
        const double f = 1.0 + sp.kappa * (1.0 - root);
        dq[i] = -(f > 0 ? 1.0 : -1.0) * sp.kappa / (2.0 * Tc * root);
    }
    for (int k = 0; k < t.ns; ++k) {
        // a*alpha's composition derivative and its temperature derivative
        double pp = 0, dpp = 0;
        for (int i = 0; i < t.ns; ++i) {
            const double pair = t.aBinary[k][i] * m.q[k] * m.q[i];
            pp += x[i] * pair;
            dpp += x[i] * pair * (2.0 * dq[i] / m.q[i] + 2.0 * dq[k] / m.q[k]);
        }
        double cpR, hRT, sR;
        nasa(t.species[k], T, cpR, hRT, sR);
        const double bk = t.species[k].b;
        const double dpdn = RT / vmb + RT * bk / (vmb * vmb) - 2.0 * pp / den + 2.0 * vmb * m.aa * bk / (den * den);
        const double departure = V * dpdn - RT - bk / (2.0 * kRt2 * b * b) * logRatio * fac
                               + V * bk / (b * den) * fac + L * (T * dpp - 2.0 * pp);
        hbar[k] = RT * hRT + departure - fac2 * dpdn;
        if (!finiteD(hbar[k])) return NONFINITE;
    }
    return OK;
}

// Properties at (T, p, Y) on the chosen root (AUTO: the largest, as Cantera starts
// gas-side), with the pressure postcondition |p(T, rho) - p| <= 1e-7 max(1, p)
// and the reported phase consistent with a GAS / LIQUID choice.
RB200_HD inline int tp(const ReactiveB200Table& t, double T, double p, const double* Y, int choice, bool chem,
                       Props& s) {
    if (!finiteD(T) || !finiteD(p) || T <= 0 || p <= 0) return BAD_INPUT;
    double x[kMaxNs] = {}, W = 0;
    if (const int st = moles(t, Y, x, W)) return st;
    Mixing m;
    if (const int st = mixing(t, T, x, m)) return st;
    Roots r;
    if (const int st = roots(m, T, p, r)) return st;
    int sel = r.count - 1;
    if (choice == LIQUID) {
        if (!r.liquid) return UNAVAILABLE;
        sel = 0;
    } else if (choice == GAS && !r.gas) return UNAVAILABLE;
    if (const int st = trho(t, T, W / r.V[sel], Y, chem, s)) return st;
    if (fabs(s.p - p) > 1e-7 * fmax(1.0, p)) return NONFINITE;
    s.p = p;
    if (choice == GAS && s.phase >= 0) return UNAVAILABLE;
    if (choice == LIQUID && s.phase < 0) return UNAVAILABLE;
    return OK;
}

}  // namespace mix
}  // namespace rb200
