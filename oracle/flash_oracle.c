/* TEST INFRASTRUCTURE ONLY (see oracle.h): serial CPU restatement of the
 * reference HEM UV flash for one condensable species with its own pure liquid
 * (ns = 1, nl = 1, no solid, no capillary), the configuration of the pure-N2O
 * cases. Algorithm steps, constants and candidate order follow
 * src/reactiveThermo/reactiveDeviceFlash.h and src/reactiveThermo/reactiveDevicePR.h:
 *   NASA7/9 cp/h/s                          reactiveDevicePR.h:127-155, region :198-212
 *   alpha(T) mixing terms                   :214-247
 *   cubic roots, near-repeated band          :280-307, :333-422
 *   reported-phase classification (cached)  :429-471, reactiveDevicePRPurePhaseCache.h:29-85
 *   (T, rho) properties and chemical potential :474-562; (T, p) root choice :575-609
 *   phase evaluation and phase sums          reactiveDeviceFlash.h:157-262
 *   all-gas scalar recovery                  :264-299
 *   frozen-partition Newton                  :302-326
 *   two-phase residual / active Newton       :327-337, :374-448
 *   stability and tangent-plane test         :449-485
 *   candidate selection and search           :486-560
 * The two-phase Jacobian is analytic (d/d ln p, d/d ln T, d/d beta of the volume,
 * energy and chemical-potential residuals), with the reference's bounded
 * finite-difference fallback when it is not finite. */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "oracle.h"

#define R_GAS 8314.46261815324
#define SQRT2 1.41421356237309504880168872420969808
#define PI_ 3.14159265358979323846264338327950288
#define OMEGA_A 4.5723552892138218e-1
#define OMEGA_B 7.77960739038885e-2
#define OMEGA_VC 3.07401308698703833e-1

enum { OK = 0, INVALID_TABLE, INVALID_INPUT, INVALID_COMPOSITION, NO_ROOT, UNAVAILABLE, UNSTABLE, NONFINITE };
enum { ROOT_AUTO = 0, ROOT_GAS = 1, ROOT_LIQUID = 2 };

typedef struct {
    const ReactiveB200Species* sp;
    double refP, Tc;
    /* reported-phase constants: rhoMid(T) = rc + (T - tc) * dRho / dT */
    double tc, rc, dRho, dT;
    int phaseCacheOk;
} Pure;

typedef struct {
    double T, p, W, V, rho, e, h, s, cp, cv, alpha, kappaT, sound, dpdT, dpdV, mu;
    int phase;
} Prop;

static int fin(double x) { return x == x && fabs(x) <= DBL_MAX; }
static double lo(double a, double b) { return a < b ? a : b; }
static double hi(double a, double b) { return a > b ? a : b; }
static double clampd(double a, double l, double h) { return lo(hi(a, l), h); }

static const ReactiveB200NasaRegion* region(const ReactiveB200Species* sp, double T) {
    int r = 0;
    for (int j = 1; j < sp->regionCount; ++j) {
        const double b = sp->regions[j].minimumTemperature;
        const int high = sp->regions[j].polynomial == 9 ? T >= b : T > b;
        if (!high) break;
        r = j;
    }
    return sp->regions + r;
}

static void nasa(const ReactiveB200NasaRegion* g, double T, double* cp, double* h, double* s) {
    const double* a = g->coefficient;
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, iT = 1.0 / T, lT = log(T);
    if (g->polynomial == 7) {
        *cp = a[0] + a[1] * T + a[2] * T2 + a[3] * T3 + a[4] * T4;
        *h = a[0] + .5 * a[1] * T + a[2] * T2 / 3.0 + .25 * a[3] * T3 + .2 * a[4] * T4 + a[5] * iT;
        *s = a[0] * lT + a[1] * T + .5 * a[2] * T2 + a[3] * T3 / 3.0 + .25 * a[4] * T4 + a[6];
    } else {
        const double c0 = a[0] * iT * iT, c1 = a[1] * iT, c2 = a[2], c3 = a[3] * T, c4 = a[4] * T2,
                     c5 = a[5] * T3, c6 = a[6] * T4;
        *cp = c0 + c1 + c2 + c3 + c4 + c5 + c6;
        *h = -c0 + lT * c1 + c2 + .5 * c3 + c4 / 3.0 + .25 * c5 + .2 * c6 + a[7] * iT;
        *s = -.5 * c0 - c1 + lT * c2 + c3 + .5 * c4 + c5 / 3.0 + .25 * c6 + a[8];
    }
}

/* a, b, a*alpha and its first two temperature derivatives for one species. */
static int alpha_terms(const Pure* P, double T, double* a, double* b, double* aa, double* da, double* d2a) {
    const ReactiveB200Species* sp = P->sp;
    const double Tc = P->Tc, sq = sqrt(T / Tc), f = 1.0 + sp->kappa * (1.0 - sq);
    double q, dq, d2q, sign;
    if (!(Tc > 0) || !fin(Tc)) return INVALID_TABLE;
    if (fabs(f) <= 1e-14) return NONFINITE;
    sign = f > 0 ? 1.0 : -1.0;
    q = fabs(f);
    dq = -sign * sp->kappa / (2.0 * Tc * sq);
    d2q = sign * sp->kappa / (4.0 * Tc * Tc * sq * sq * sq);
    *a = sp->a;
    *b = sp->b;
    *aa = sp->a * q * q;
    *da = sp->a * (dq * q + q * dq);
    *d2a = sp->a * (d2q * q + 2.0 * dq * dq + q * d2q);
    return fin(*aa) && fin(*da) && fin(*d2a) && *aa > 0 ? OK : NONFINITE;
}

static double cubic(double V, double bn, double cn, double dn) { return ((V + bn) * V + cn) * V + dn; }

typedef struct { double V[3]; int count, signedCount, gas, liquid; } Roots;

static int isolated(double center, double delta, double delta2, double q, double bn, double cn, double dn, double b,
                    double RTp, double aap, double* root, int* gasSide) {
    double pair, x, f, scale, vb, den;
    int converged = 0;
    if (!(delta2 > 0) || !fin(delta) || !fin(q) || q == 0) return 0;
    *gasSide = q < 0;
    pair = center + (*gasSide ? -1.0 : 1.0) * delta;
    x = center + (*gasSide ? 2.0 : -2.0) * delta;
    for (int n = 0; n < 24; ++n) {
        const double fx = cubic(x, bn, cn, dn), dfx = (3.0 * x + 2.0 * bn) * x + cn, step = fx / dfx;
        if (!fin(fx) || !fin(dfx) || fabs(dfx) <= 1e-300) return 0;
        x -= step;
        if (fabs(step) <= 4e-15 * hi(1.0, fabs(x))) { converged = 1; break; }
    }
    if (!converged || !fin(x) || !(x > b)) return 0;
    f = cubic(x, bn, cn, dn);
    scale = fabs(x * x * x) + fabs(bn * x * x) + fabs(cn * x) + fabs(dn);
    if (!(fabs(f) <= 64.0 * DBL_EPSILON * scale)) return 0;
    if (!(fabs(x - pair) > 1e-3 * hi(fabs(x), fabs(pair)))) return 0;
    if (*gasSide ? !(x > pair) : !(x < pair)) return 0;
    vb = x - b;
    den = x * x + 2.0 * b * x - b * b;
    if (!(vb > 0) || !(den > 0)) return 0;
    if (!(-RTp / (vb * vb) + 2.0 * aap * (x + b) / (den * den) < 0)) return 0;
    *root = x;
    return 1;
}

static double cube_root(double x) { return x < 0 ? -pow(-x, 1.0 / 3.0) : pow(x, 1.0 / 3.0); }

static int roots_tp(double T, double p, double a, double b, double aa, Roots* out) {
    const double b2 = b * b, RTp = R_GAS * T / p, aap = aa / p, bn = b - RTp;
    const double cn = -(2.0 * RTp * b - aap + 3.0 * b2), dn = b2 * RTp + b2 * b - aap * b;
    const double center = -bn / 3.0, delta2 = (bn * bn - 3.0 * cn) / 9.0;
    const double q = 2.0 * bn * bn * bn / 27.0 - bn * cn / 3.0 + dn;
    const double delta = delta2 > 0 ? sqrt(delta2) : 0, h = 2.0 * delta * delta2;
    double disc = q * q - h * h, raw[3] = {0, 0, 0}, Tcm, pc, vc;
    int rawCount = 0, side = 0, n = 0;
    if (fabs(fabs(h) - fabs(q)) < 1e-10) {
        if (disc > 1e-10) return NONFINITE;
        disc = 0;
    }
    if (fabs(disc) < 1e-14) {
        int gasSide = 0;
        if (!isolated(center, delta, delta2, q, bn, cn, dn, b, RTp, aap, raw, &gasSide)) return NO_ROOT;
        rawCount = 1;
        side = gasSide ? 1 : -1;
    } else if (disc > 1e-14 || !(delta2 > 0)) {
        const double sd = .5 * sqrt(hi(0.0, disc));
        raw[0] = center + cube_root(-.5 * q + sd) + cube_root(-.5 * q - sd);
        rawCount = 1;
    } else if (disc < -1e-14) {
        double arg = clampd(-.5 * q / (delta * delta * delta), -1.0, 1.0);
        const double theta = acos(arg) / 3.0;
        raw[0] = center + 2.0 * delta * cos(theta);
        raw[1] = center + 2.0 * delta * cos(theta + 2.0 * PI_ / 3.0);
        raw[2] = center + 2.0 * delta * cos(theta + 4.0 * PI_ / 3.0);
        rawCount = 3;
    } else return NO_ROOT;
    for (int i = 0; !side && i < rawCount; ++i)
        for (int it = 0; it < 12; ++it) {
            const double r = cubic(raw[i], bn, cn, dn), d = (3.0 * raw[i] + 2.0 * bn) * raw[i] + cn;
            double step;
            if (fabs(d) <= 1e-300) break;
            step = r / d;
            raw[i] -= step;
            if (fabs(step) <= 4e-15 * hi(1.0, fabs(raw[i]))) break;
        }
    for (int i = 1; i < rawCount; ++i) { /* insertion sort */
        const double key = raw[i];
        int j = i - 1;
        while (j >= 0 && raw[j] > key) { raw[j + 1] = raw[j]; --j; }
        raw[j + 1] = key;
    }
    for (int i = 0; i < rawCount; ++i)
        if (fin(raw[i]) && raw[i] > b) out->V[n++] = raw[i];
    if (!n) return NO_ROOT;
    out->count = n;
    Tcm = a * OMEGA_B / (b * OMEGA_A * R_GAS);
    pc = OMEGA_B * R_GAS * Tcm / b;
    vc = OMEGA_VC * R_GAS * Tcm / pc;
    if (side) { out->signedCount = side; out->gas = side > 0; out->liquid = side < 0; }
    else if (n >= 2) { out->signedCount = n; out->gas = out->liquid = 1; }
    else {
        const int liquidSign = T > Tcm ? out->V[0] < vc : out->V[0] < center;
        out->signedCount = liquidSign ? -1 : 1;
        out->liquid = liquidSign;
        out->gas = !liquidSign || T > Tcm;
    }
    return OK;
}

/* Reported-phase constants of a pure table: the classification line through
 * (Tc, rho_c) and the mid-density at Tc-100 K (Cantera's phaseState heuristic). */
static void build_phase_cache(Pure* P) {
    const double a = P->sp->a, b = P->sp->b, W = P->sp->molecularWeight;
    const double tc = a * OMEGA_B / (b * OMEGA_A * R_GAS), pc = OMEGA_B * R_GAS * tc / b;
    const double vc = OMEGA_VC * R_GAS * tc / pc;
    double tmid = tc - 100.0, ratio, pp, liquidVolume = -1, aa, da, d2a, am, bm;
    int found = 0;
    if (tmid < 0) tmid = .5 * tc;
    ratio = tc / tmid;
    pp = pc * exp(-.8734 * ratio * ratio - 3.4522 * ratio + 4.2918);
    P->phaseCacheOk = 0;
    if (alpha_terms(P, tmid, &am, &bm, &aa, &da, &d2a) != OK) return;
    for (int it = 0; it < 100; ++it) {
        Roots r = {{0, 0, 0}, 0, 0, 0, 0};
        const int st = roots_tp(tmid, pp, am, bm, aa, &r);
        if (st != OK) return;
        if (r.signedCount == 1 || r.signedCount == 2) {
            found = pp > pc;
            liquidVolume = r.V[0];
            pp *= 1.04;
            if (found) break;
        } else {
            liquidVolume = r.V[0];
            found = 1;
            break;
        }
    }
    if (!found || !(liquidVolume > 0) || !fin(liquidVolume)) return;
    {
        const double rc = W / vc, rl = W / liquidVolume, rg = W / (R_GAS * tmid / pp);
        P->tc = tc;
        P->rc = rc;
        P->dRho = rc - .5 * (rl + rg);
        P->dT = tc - tmid;
        P->phaseCacheOk = fin(P->dRho) && fin(P->dT) && P->dT > 0;
    }
}

static int evaluate_trho(const Pure* P, double T, double rho, int chem, Prop* o) {
    const double W = P->sp->molecularWeight;
    double a, b, aa, da, d2a, den, vmb, logRatio, L, cp0, h0, s0, z, hM, sM, dHdT, cpM, cvM, sound2;
    double cpR, hRT, sR;
    Prop s;
    int st;
    memset(&s, 0, sizeof(s));
    if (!fin(T) || !fin(rho) || T <= 0 || rho <= 0) return INVALID_INPUT;
    if ((st = alpha_terms(P, T, &a, &b, &aa, &da, &d2a)) != OK) return st;
    s.T = T; s.W = W; s.rho = rho; s.V = W / rho;
    if (!(s.V > b)) return NO_ROOT;
    den = s.V * s.V + 2.0 * s.V * b - b * b;
    vmb = s.V - b;
    if (!(den > 0) || !(vmb > 0)) return NO_ROOT;
    s.p = R_GAS * T / vmb - aa / den;
    if (!fin(s.p) || s.p <= 0) return NO_ROOT;
    s.dpdV = -R_GAS * T / (vmb * vmb) + 2.0 * aa * (s.V + b) / (den * den);
    s.dpdT = R_GAS / vmb - da / den;
    if (!fin(s.dpdV) || !fin(s.dpdT) || s.dpdV >= 0) return UNSTABLE;
    logRatio = log((s.V + (1.0 + SQRT2) * b) / (s.V + (1.0 - SQRT2) * b));
    L = logRatio / (2.0 * SQRT2 * b);
    nasa(region(P->sp, T), T, &cpR, &hRT, &sR);
    cp0 = R_GAS * cpR;
    h0 = R_GAS * T * hRT;
    s0 = R_GAS * sR;
    z = s.p * s.V / (R_GAS * T);
    hM = h0 + (R_GAS * T * (z - 1.0) + L * (T * da - aa));
    sM = (s0 - R_GAS * log(s.p / P->refP)) + (R_GAS * log(z * (1.0 - b / s.V)) + L * da);
    dHdT = cp0 + s.V * s.dpdT - R_GAS + L * T * d2a;
    cpM = dHdT - (s.V + T * s.dpdT / s.dpdV) * s.dpdT;
    cvM = cpM + T * s.dpdT * s.dpdT / s.dpdV;
    s.h = hM / W; s.e = (hM - s.p * s.V) / W; s.s = sM / W; s.cp = cpM / W; s.cv = cvM / W;
    s.alpha = -s.dpdT / (s.V * s.dpdV);
    s.kappaT = -1.0 / (s.V * s.dpdV);
    sound2 = s.V * s.V * (-cpM / cvM * s.dpdV / W);
    if (!(s.cp > 0) || !(s.cv > 0) || !(s.kappaT > 0) || !(sound2 > 0)) return UNSTABLE;
    s.sound = sqrt(sound2);
    if (chem) {
        const double RT = R_GAS * T, f = 1.0 + P->sp->kappa * (1.0 - sqrt(T / P->Tc));
        const double pp = P->sp->a * fabs(f * f), num = 2.0 * b * pp - aa * b;
        s.mu = RT * (hRT - sR) + RT * log(1.0) + RT * log(s.p / P->refP) - RT * log(s.p * s.V / RT)
             + RT * log(s.V / vmb) + RT * b / vmb - num / (2.0 * SQRT2 * b * b) * logRatio - aa * b * s.V / (b * den);
    }
    if (!P->phaseCacheOk) return NONFINITE;
    if (T >= P->tc) s.phase = -2;
    else {
        const double rhoMid = P->rc + (T - P->tc) * P->dRho / P->dT;
        if (!fin(rhoMid)) return NONFINITE;
        s.phase = rho < rhoMid ? -1 : 0;
    }
    {
        const double v[12] = {s.rho, s.e, s.h, s.s, s.cp, s.cv, s.alpha, s.kappaT, s.sound, s.p, s.dpdT, s.dpdV};
        for (int i = 0; i < 12; ++i) if (!fin(v[i])) return NONFINITE;
        if (chem && !fin(s.mu)) return NONFINITE;
    }
    *o = s;
    return OK;
}

static int evaluate_tp(const Pure* P, double T, double p, int choice, int chem, Prop* o) {
    double a, b, aa, da, d2a;
    Roots r = {{0, 0, 0}, 0, 0, 0, 0};
    int st, sel;
    Prop s;
    if (!fin(T) || !fin(p) || T <= 0 || p <= 0) return INVALID_INPUT;
    if ((st = alpha_terms(P, T, &a, &b, &aa, &da, &d2a)) != OK) return st;
    if ((st = roots_tp(T, p, a, b, aa, &r)) != OK) return st;
    sel = r.count - 1;
    if (choice == ROOT_LIQUID) {
        if (!r.liquid) return UNAVAILABLE;
        sel = 0;
    } else if (choice == ROOT_GAS && !r.gas) return UNAVAILABLE;
    if ((st = evaluate_trho(P, T, P->sp->molecularWeight / r.V[sel], chem, &s)) != OK) return st;
    if (fabs(s.p - p) > 1e-7 * hi(1.0, p)) return NONFINITE;
    s.p = p;
    if (choice == ROOT_GAS && s.phase >= 0) return UNAVAILABLE;
    if (choice == ROOT_LIQUID && s.phase < 0) return UNAVAILABLE;
    *o = s;
    return OK;
}

/* ------------------------------------------------------------------ flash */
typedef struct {
    ReactiveThermoState st;
    double volume, energy, entropyDensity, Vp, VT, Ep, ET, cpDensity;
    double muGas, muLiquid;
    int liquidOk; /* liquid properties at this point exist */
    Prop gas, liq;
} Eval;

typedef struct {
    const ReactiveB200HemModel* m;
    Pure gasT, liqT;
    double q, e;
    ReactiveThermoState guess;
    uint64_t phases, residuals, candidates, stable, failures, analytic, fd;
} Flash;

static int bounds(const Flash* F, double p, double T) {
    const ReactiveB200HemModel* m = F->m;
    return fin(p) && fin(T) && p >= m->pmin && p <= m->pmax && T >= m->Tmin && T <= m->Tmax;
}

static int phase_status(Flash* F, int index, double p, double T, Prop* out, int chem) {
    const ReactiveB200HemModel* m = F->m;
    ++F->phases;
    if (!bounds(F, p, T)) return INVALID_INPUT;
    if (index >= 0 && T < m->liquidTmin[index]) return INVALID_INPUT;
    if (index >= 0 && T >= m->liquidTc[index] * (1 - 1e-10)) return UNAVAILABLE;
    if (index < 0 && m->enforceSpeciesTemperatureBounds) {
        const ReactiveB200Species* sp = F->gasT.sp;
        if (T < sp->regions[0].minimumTemperature || T > sp->regions[sp->regionCount - 1].maximumTemperature)
            return INVALID_INPUT;
    }
    return index < 0 ? evaluate_tp(&F->gasT, T, p, ROOT_GAS, chem, out)
                     : evaluate_tp(&F->liqT, T, p, ROOT_LIQUID, chem, out);
}

static int unavailable(int s) { return s == UNAVAILABLE || s == NO_ROOT; }

static void accumulate(Eval* v, double mass, const Prop* p, double pressure) {
    const double volume = mass / p->rho, vp = -volume * p->kappaT, vt = volume * p->alpha;
    v->volume += volume; v->energy += mass * p->e; v->entropyDensity += mass * p->s;
    v->Vp += vp; v->VT += vt;
    v->Ep += -v->st.T * vt - pressure * vp;
    v->ET += mass * p->cp - pressure * vt;
    v->cpDensity += mass * p->cp;
}

static int evaluate(Flash* F, double mass, double p, double T, Eval* v, int virt) {
    ReactiveThermoState* s = &v->st;
    double gas, specific, vp, vt, adiabatic;
    memset(v, 0, sizeof(*v));
    if (!bounds(F, p, T)) return 0;
    s->p = p; s->T = T; s->rho = F->q;
    if (!(s->rho > 0)) return 0;
    if (!fin(F->q) || F->q < 0) return 0;
    if (!fin(mass) || mass < 0 || mass > F->q) return 0;
    gas = F->q - mass;
    if (!fin(gas) || gas < 0 || gas > F->q) return 0;
    s->gasMass = gas;
    if (gas > 0) {
        if (phase_status(F, -1, p, T, &v->gas, virt) != OK) return 0;
        accumulate(v, gas, &v->gas, p);
        s->alphaGas = gas / v->gas.rho;
        s->rhoGas = v->gas.rho;
        if (virt) v->muGas = v->gas.mu / (R_GAS * T);
    }
    s->liquidMass[0] = mass;
    if (mass > 0 || (virt && F->q > 0)) {
        const int status = phase_status(F, 0, p, T, &v->liq, virt);
        if (status != OK) {
            if (mass > 0 || !unavailable(status)) return 0;
            v->muLiquid = HUGE_VAL;
        } else {
            v->liquidOk = 1;
            if (virt) v->muLiquid = v->liq.mu / (R_GAS * T);
            if (mass > 0) {
                accumulate(v, mass, &v->liq, p);
                s->rhoLiquid[0] = v->liq.rho;
                s->alphaLiquid[0] = mass / v->liq.rho;
                s->activeLiquids |= 1;
            }
        }
    }
    s->e = v->energy / s->rho;
    s->entropy = v->entropyDensity / s->rho;
    s->cp = v->cpDensity / s->rho;
    s->cv = (v->cpDensity + T * v->VT * v->VT / v->Vp) / s->rho;
    if (!fin(s->cv) || s->cv <= 0) return 0;
    specific = v->volume / s->rho; vp = v->Vp / s->rho; vt = v->VT / s->rho;
    adiabatic = vp + T * vt * vt / s->cp;
    if (!(adiabatic < 0)) return 0;
    s->soundFrozen = sqrt(-specific * specific / adiabatic);
    s->soundEquilibrium = s->soundFrozen;
    return fin(s->soundFrozen) && s->soundFrozen > 0;
}

static double energy_scale(const Eval* v) { return hi(1e5 * v->st.rho, v->cpDensity * v->st.T); }

/* Full-pivot elimination with a rank test (pivot > largest * n * eps). */
static int solve(double A[4][4], const double* rhs, int n, double* x) {
    double a[4][4], b[4], largest = 0, z[4] = {0, 0, 0, 0};
    int column[4] = {0, 1, 2, 3};
    for (int i = 0; i < n; ++i) {
        b[i] = rhs[i];
        if (!fin(b[i])) return 0;
        for (int j = 0; j < n; ++j) { a[i][j] = A[i][j]; if (!fin(a[i][j])) return 0; }
    }
    for (int k = 0; k < n; ++k) {
        int row = k, col = k;
        double pivot = 0;
        for (int j = k; j < n; ++j)
            for (int i = k; i < n; ++i)
                if (fabs(a[i][j]) > pivot) { pivot = fabs(a[i][j]); row = i; col = j; }
        largest = hi(largest, pivot);
        if (!(pivot > largest * n * DBL_EPSILON)) return 0;
        if (row != k) {
            for (int j = 0; j < n; ++j) { const double t = a[k][j]; a[k][j] = a[row][j]; a[row][j] = t; }
            { const double t = b[k]; b[k] = b[row]; b[row] = t; }
        }
        if (col != k) {
            for (int i = 0; i < n; ++i) { const double t = a[i][k]; a[i][k] = a[i][col]; a[i][col] = t; }
            { const int t = column[k]; column[k] = column[col]; column[col] = t; }
        }
        for (int i = k + 1; i < n; ++i) {
            const double f = a[i][k] / a[k][k];
            a[i][k] = f;
            for (int j = k + 1; j < n; ++j) a[i][j] -= f * a[k][j];
            b[i] -= f * b[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double v = b[i];
        for (int j = i + 1; j < n; ++j) v -= a[i][j] * z[j];
        z[i] = v / a[i][i];
        if (!fin(z[i])) return 0;
    }
    for (int i = 0; i < n; ++i) x[column[i]] = z[i];
    return 1;
}

static int gas_probe(Flash* F, double T, double* Fv, double* cv, double* p, double* cp) {
    Prop prop, gas;
    ++F->phases;
    if (evaluate_trho(&F->gasT, T, F->q, 0, &prop) != OK) return 0;
    *p = prop.p;
    if (!bounds(F, *p, T)) return 0;
    if (phase_status(F, -1, prop.p, T, &gas, 0) != OK || fabs(gas.rho - F->q) > 1e-8 * F->q) return 0;
    *Fv = F->q * prop.e - F->e;
    *cv = F->q * prop.cv;
    if (cp) *cp = prop.cp;
    return fin(*Fv) && fin(*cv) && *cv > 0;
}

static int scalar_gas(Flash* F, Eval* result) {
    const ReactiveB200HemModel* m = F->m;
    const double rho = F->q;
    double T = clampd(F->guess.T, m->Tmin, m->Tmax), Fv, cv, p, cp, scale, lower, upper, fl, fh;
    int it = 0;
    if (!gas_probe(F, T, &Fv, &cv, &p, &cp)) return 0;
    scale = hi(1e5 * rho, rho * cp * T);
    lower = upper = T;
    fl = fh = Fv;
    if (fabs(Fv) > m->etol * scale) {
        double radius = hi(1., .01 * T);
        for (int j = 0; j < 24 && (fl > 0 || fh < 0); ++j, radius *= 2) {
            if (fl > 0) {
                double cand = hi(m->Tmin, T - radius), val, d1, d2;
                int found = 0;
                for (int r = 0; r < 8 && !found; ++r) {
                    if (gas_probe(F, cand, &val, &d1, &d2, 0)) { fl = val; lower = cand; found = 1; }
                    else cand = .5 * (lower + cand);
                }
                if (!found) return 0;
            }
            if (fh < 0) {
                double cand = lo(m->Tmax, T + radius), val, d1, d2;
                int found = 0;
                for (int r = 0; r < 8 && !found; ++r) {
                    if (gas_probe(F, cand, &val, &d1, &d2, 0)) { fh = val; upper = cand; found = 1; }
                    else cand = .5 * (upper + cand);
                }
                if (!found) return 0;
            }
            if (fabs(fl) <= m->etol * scale) { T = lower; if (!gas_probe(F, T, &Fv, &cv, &p, 0)) return 0; break; }
            if (fabs(fh) <= m->etol * scale) { T = upper; if (!gas_probe(F, T, &Fv, &cv, &p, 0)) return 0; break; }
            if (lower == m->Tmin && upper == m->Tmax) break;
        }
        if (!(fabs(Fv) <= m->etol * scale || (fl <= 0 && fh >= 0 && upper > lower))) return 0;
    }
    for (; it < 70 && fabs(Fv) > m->etol * scale; ++it) {
        double next;
        if (Fv > 0) upper = T; else lower = T;
        next = T - Fv / cv;
        T = fin(next) && next > lower && next < upper ? next : .5 * (lower + upper);
        if (!gas_probe(F, T, &Fv, &cv, &p, 0)) return 0;
    }
    if (fabs(Fv) > m->etol * scale) return 0;
    if (!evaluate(F, 0.0, p, T, result, 0)) return 0;
    result->st.volumeResidual = fabs(result->volume - 1);
    result->st.energyResidual = fabs(result->energy - F->e) / energy_scale(result);
    result->st.iterations = it;
    return result->st.volumeResidual <= m->vtol && result->st.energyResidual <= m->etol;
}

static int frozen(Flash* F, double mass, Eval* value, int stallLimit) {
    const ReactiveB200HemModel* m = F->m;
    double p, T;
    int stalled = 0;
    if (!fin(F->e)) return 0;
    if (m->scalarRecovery && mass == 0 && scalar_gas(F, value)) return 1;
    p = clampd(F->guess.p, m->pmin, m->pmax);
    T = clampd(F->guess.T, m->Tmin, m->Tmax);
    if (!evaluate(F, mass, p, T, value, 0)) return 0;
    for (int it = 0; it < 70; ++it) {
        const double scale = energy_scale(value), rv = value->volume - 1, re = (value->energy - F->e) / scale;
        double jac[4][4] = {{0}}, rhs[4] = {-rv, -re, 0, 0}, step[4] = {0, 0, 0, 0}, limit, previous;
        int accepted = 0;
        value->st.volumeResidual = fabs(rv);
        value->st.energyResidual = fabs(re);
        value->st.iterations = it;
        if (fabs(rv) <= m->vtol && fabs(re) <= m->etol) return 1;
        jac[0][0] = value->Vp * p; jac[0][1] = value->VT * T;
        jac[1][0] = value->Ep * p / scale; jac[1][1] = value->ET * T / scale;
        if (!solve(jac, rhs, 2, step)) return 0;
        limit = hi(1., hi(fabs(step[0]) / .7, fabs(step[1]) / .2));
        step[0] /= limit; step[1] /= limit;
        previous = hi(fabs(rv), fabs(re));
        for (double fraction = 1; fraction > 1e-9; fraction *= .5) {
            Eval trial;
            const double pp = p * exp(fraction * step[0]), tt = T * exp(fraction * step[1]);
            if (evaluate(F, mass, pp, tt, &trial, 0)) {
                const double next = hi(fabs(trial.volume - 1), fabs(trial.energy - F->e) / scale);
                if (next < previous * (1 - 1e-4 * fraction) || next < lo(m->vtol, m->etol)) {
                    *value = trial; p = pp; T = tt; accepted = 1;
                    stalled = fraction < 1. / 32 ? stalled + 1 : 0;
                    break;
                }
            }
        }
        if (!accepted) return 0;
        if (stallLimit > 0 && stalled >= stallLimit
            && !(fabs(value->volume - 1) <= m->vtol && fabs(value->energy - F->e) / energy_scale(value) <= m->etol))
            return 0;
    }
    return 0;
}

static int residual(Flash* F, const double* x, double scale, double* f, Eval* out) {
    Eval v;
    ++F->residuals;
    if (!(x[2] >= 0 && x[2] < 1)) return 0;
    if (!evaluate(F, x[2] * F->q, exp(x[0]), exp(x[1]), &v, 1) || !(v.st.gasMass > 0)) return 0;
    f[0] = v.volume - 1;
    f[1] = (v.energy - F->e) / scale;
    f[2] = v.muLiquid - v.muGas;
    if (!fin(f[2])) return 0;
    if (out) *out = v;
    return 1;
}

/* d(f)/d(ln p, ln T, beta) at an evaluated two-phase point. */
static int analytic_jacobian(const Flash* F, const Eval* v, double scale, double J[4][4]) {
    const double p = v->st.p, T = v->st.T, RT = R_GAS * T, q = F->q;
    const Prop* g = &v->gas;
    const Prop* l = &v->liq;
    if (!v->liquidOk || !(v->st.gasMass > 0)) return 0;
    J[0][0] = v->Vp * p; J[0][1] = v->VT * T; J[0][2] = q * (1 / l->rho - 1 / g->rho);
    J[1][0] = v->Ep * p / scale; J[1][1] = v->ET * T / scale; J[1][2] = q * (l->e - g->e) / scale;
    J[2][0] = p * (l->V - g->V) / RT;
    J[2][1] = -(l->h - g->h) * l->W / RT;
    J[2][2] = 0;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) if (!fin(J[i][j])) return 0;
    return 1;
}

static int jacobian(Flash* F, const double* x, double scale, const double* f, const Eval* point, double J[4][4]) {
    if (F->m->analyticJacobian && analytic_jacobian(F, point, scale, J)) { ++F->analytic; return 1; }
    ++F->fd;
    for (int j = 0; j < 3; ++j) {
        double h = j < 2 ? 2e-6 : 2e-5;
        int success = 0;
        for (int attempt = 0; attempt < 12 && !success; ++attempt, h *= .5) {
            double xp[4], xm[4], fp[4], fm[4];
            int plus, minus;
            for (int i = 0; i < 3; ++i) xp[i] = xm[i] = x[i];
            xp[j] += h; xm[j] -= h;
            plus = residual(F, xp, scale, fp, 0);
            minus = residual(F, xm, scale, fm, 0);
            if (!plus && !minus) continue;
            success = 1;
            for (int i = 0; i < 3; ++i) {
                const double val = plus && minus ? (fp[i] - fm[i]) / (2 * h) : plus ? (fp[i] - f[i]) / h : (f[i] - fm[i]) / h;
                J[i][j] = val;
                success = success && fin(val);
            }
        }
        if (!success) return 0;
    }
    return 1;
}

static int active_flash(Flash* F, double seed, Eval* value, const ReactiveThermoState* restart) {
    const ReactiveB200HemModel* m = F->m;
    const ReactiveThermoState* guess = restart ? restart : &F->guess;
    const double rho = F->q;
    const double scale = hi(1e5 * rho, hi(fabs(F->e), rho * 2000 * hi(guess->T, m->Tmin)));
    double x[4] = {log(clampd(guess->p, m->pmin, m->pmax)), log(clampd(guess->T, m->Tmin, m->Tmax)), 0, 0};
    double f[4] = {0, 0, 0, 0};
    ++F->candidates;
    {
        const double previous = guess->liquidMass[0] / F->q;
        x[2] = seed < 0 ? clampd(previous, 1e-8, 1 - 1e-8) : seed;
    }
    if (!residual(F, x, scale, f, value)) return 0;
    for (int it = 0; it < 90; ++it) {
        const double chemical = fabs(f[2]);
        double jac[4][4] = {{0}}, rhs[4], step[4] = {0, 0, 0, 0}, limiter, previous, fraction = 1;
        int accepted = 0;
        if (fabs(f[0]) <= m->vtol && fabs(f[1]) <= m->etol && chemical <= m->mutol) {
            double response[4] = {0, 0, 0, 0}, squared;
            value->st.volumeResidual = fabs(f[0]);
            value->st.energyResidual = fabs(f[1]);
            value->st.chemicalResidual = chemical;
            value->st.iterations = it;
            if (!jacobian(F, x, scale, f, value, jac)) return 0;
            rhs[0] = -1 / rho; rhs[1] = value->st.p / (rho * scale); rhs[2] = 0;
            if (!solve(jac, rhs, 3, response)) return 0;
            squared = value->st.p * response[0];
            if (!fin(squared) || squared <= 0) return 0;
            value->st.soundEquilibrium = sqrt(squared);
            return value->st.soundEquilibrium <= value->st.soundFrozen * (1 + 2e-3);
        }
        if (!jacobian(F, x, scale, f, value, jac)) return 0;
        for (int j = 0; j < 3; ++j) rhs[j] = -f[j];
        if (!solve(jac, rhs, 3, step)) return 0;
        limiter = hi(1., hi(fabs(step[0]) / .7, fabs(step[1]) / .18));
        limiter = hi(limiter, fabs(step[2]) / .3);
        for (int j = 0; j < 3; ++j) step[j] /= limiter;
        previous = hi(fabs(f[0]), hi(fabs(f[1]), fabs(f[2])));
        for (int k = 0; k < 30; ++k, fraction *= .5) {
            double tx[4], tf[4];
            Eval trial;
            for (int j = 0; j < 3; ++j) tx[j] = x[j] + fraction * step[j];
            if (!(tx[2] >= 0 && tx[2] < 1)) { ++F->residuals; continue; }
            if (residual(F, tx, scale, tf, &trial)
                && hi(fabs(tf[0]), hi(fabs(tf[1]), fabs(tf[2]))) < previous * (1 - 1e-4 * fraction)) {
                for (int j = 0; j < 3; ++j) { x[j] = tx[j]; f[j] = tf[j]; }
                *value = trial;
                accepted = 1;
                break;
            }
        }
        if (!accepted) return 0;
    }
    return 0;
}

static double tangent(Flash* F, double p, double T, double muLiquid) {
    Prop prop;
    const int status = phase_status(F, -1, p, T, &prop, 0);
    if (status != OK) return unavailable(status) ? HUGE_VAL : NAN;
    return (prop.h - T * prop.s) * prop.W / (R_GAS * T) - muLiquid;
}

static int stable(Flash* F, Eval* value) {
    const double p = value->st.p, T = value->st.T;
    if (value->st.gasMass > 0) {
        Eval cmp;
        const double mass = value->st.liquidMass[0];
        double affinity;
        if (!evaluate(F, mass, p, T, &cmp, 1)) return 0;
        if (F->q == 0) return 1;
        affinity = cmp.muLiquid - cmp.muGas;
        if (mass > 0) { if (!fin(affinity) || fabs(affinity) > F->m->mutol * 2) return 0; }
        else if (affinity < -F->m->mutol) return 0;
        return 1;
    }
    if (!(value->st.liquidMass[0] > 0)) return 0;
    {
        Prop prop;
        double mu;
        if (phase_status(F, 0, p, T, &prop, 1) != OK) return 0;
        mu = prop.mu / (R_GAS * T);
        return tangent(F, p, T, mu) >= -F->m->mutol;
    }
}

static void consider(Flash* F, Eval* cand, Eval* best, int* have) {
    if (stable(F, cand)) {
        ++F->stable;
        if (!*have || cand->entropyDensity > best->entropyDensity) { *best = *cand; *have = 1; }
    } else ++F->failures;
}

static const double SEEDS[5] = {-1, .5, .95, .1, .9999};
static const double RESTARTS[4] = {0.02, 0.25, 0.5, 0.75};

static int search(Flash* F, Eval* best) {
    const ReactiveB200HemModel* m = F->m;
    Eval cand;
    int have = 0, gasStable = 0;
    const int pruneOk = m->stableGasPrune && m->nl == 1 && m->condensedKind[0] == 0 && m->condensedKind[1] == 0;
    if (frozen(F, 0.0, &cand, pruneOk ? 4 : 0)) {
        const uint64_t before = F->stable;
        consider(F, &cand, best, &have);
        gasStable = F->stable > before && cand.st.gasMass > 0;
    } else ++F->failures;
    /* no non-condensable inventory in a pure fluid: the all-liquid partition */
    if (frozen(F, F->q, &cand, 0)) consider(F, &cand, best, &have);
    else ++F->failures;
    if (!(pruneOk && gasStable) && F->q > 0)
        for (int j = 0; j < 5; ++j) {
            if (active_flash(F, SEEDS[j], &cand, 0)) consider(F, &cand, best, &have);
            else ++F->failures;
        }
    if (!have && F->q > 0) {
        const double lower = hi(m->Tmin, m->liquidTmin[0]), upper = lo(m->Tmax, m->liquidTc[0] * (1 - 1e-10));
        if (upper > lower)
            for (int t = 0; t < 4; ++t) {
                ReactiveThermoState restart = F->guess;
                restart.T = lower + (upper - lower) * RESTARTS[t];
                for (int j = 0; j < 5; ++j) {
                    if (active_flash(F, SEEDS[j], &cand, &restart)) consider(F, &cand, best, &have);
                    else ++F->failures;
                }
            }
    }
    return have;
}

static void make_pure(Pure* P, const ReactiveB200Table* t) {
    memset(P, 0, sizeof(*P));
    P->sp = &t->species[0];
    P->refP = t->refPressure;
    P->Tc = P->sp->a * OMEGA_B / (P->sp->b * OMEGA_A * R_GAS);
    build_phase_cache(P);
}

int oracle_flash_recover(const char* image, size_t count, const double* q, const double* energy,
                         const ReactiveThermoState* guess, ReactiveThermoState* out, int* success, uint64_t* counters,
                         int threads) {
    const ReactiveB200HemModel* m = (const ReactiveB200HemModel*)image;
    Pure gasT, liqT;
    (void)threads;
    if (m->ns != 1 || m->nl != 1 || m->condensable[0] != 0 || m->boundaryRecovery || m->condensedKind[0]) return 1;
    make_pure(&gasT, &m->phase[0]);
    make_pure(&liqT, &m->phase[1]);
    for (size_t c = 0; c < count; ++c) {
        Flash F;
        Eval best;
        int ok = 0;
        memset(&F, 0, sizeof(F));
        F.m = m; F.gasT = gasT; F.liqT = liqT; F.q = q[c]; F.e = energy[c]; F.guess = guess[c];
        if (fin(F.e) && fin(F.q) && F.q > 0) ok = search(&F, &best);
        out[c] = ok ? best.st : guess[c];
        success[c] = ok;
        if (counters) {
            uint64_t* k = counters + 7 * c;
            k[0] = F.phases; k[1] = F.residuals; k[2] = F.candidates; k[3] = F.stable; k[4] = F.failures;
            k[5] = F.analytic; k[6] = F.fd;
        }
    }
    return 0;
}

/* PR evaluation at (T, p) with a root choice, for EOS unit checks.
 * out: T p W V rho e h s cp cv alpha kappaT sound dpdT dpdV mu */
int oracle_pr_evaluate_tp(const char* image, int table, double T, double p, int choice, int chem, double* out,
                          int* phase) {
    const ReactiveB200HemModel* m = (const ReactiveB200HemModel*)image;
    Pure P;
    Prop s;
    int st;
    make_pure(&P, &m->phase[table]);
    st = evaluate_tp(&P, T, p, choice, chem, &s);
    if (st == OK) {
        const double v[16] = {s.T, s.p, s.W, s.V, s.rho, s.e, s.h, s.s, s.cp, s.cv, s.alpha, s.kappaT, s.sound,
                              s.dpdT, s.dpdV, s.mu};
        memcpy(out, v, sizeof(v));
        *phase = s.phase;
    }
    return st;
}
