// Lane-level work queue for the HEM candidate solves.
//
// Each candidate solve of hem_flash.cuh is rewritten as a per-lane state
// machine whose only expensive step is one thermodynamic evaluation. A
// persistent kernel loops: lanes without work take the next (cell, candidate)
// item from an on-device counter (one warp-aggregated atomic per warp), every
// lane advances its own solver until it needs an evaluation, and then all lanes
// of the warp perform their evaluations together. A lane whose Newton finished
// early picks up a new item instead of idling beside a lane that is still
// iterating, so the PR evaluations, which are nearly all of the arithmetic, run
// with (almost) full warps whatever the spread of iteration counts.
//
// Every solver requests exactly the evaluation points its recursive form in
// hem_flash.cuh visits, in the same order, so results are bitwise identical:
//   all-gas    scalar T-Newton at fixed rho (bracket, Newton, final point),
//              then the frozen (ln p, ln T) Newton if that fails
//   all-liquid frozen (ln p, ln T) Newton
//   two-phase  (ln p, ln T, beta) Newton, 30-fraction line search
//   stability  affinity at the converged point (two-phase: the converged
//              residual evaluation itself, which is the point the stability
//              test evaluates), or one virtual-liquid evaluation (all-gas), or
//              the tangent-plane test (all-liquid)
#pragma once
#include "hem_flash.cuh"

namespace rb200 {

enum QueueRequest : int { REQ_NONE = 0, REQ_POINT, REQ_PROBE, REQ_TANGENT };

enum QueueState : int {
    Q_FREE = 0,
    Q_FZ_START, Q_FZ_NEWTON_INIT, Q_FZ_INIT_AFTER, Q_FZ_ITER, Q_FZ_LS, Q_FZ_LS_AFTER,
    Q_SG_AFTER0, Q_SG_BR_LOOP, Q_SG_LO_AFTER, Q_SG_HI_CHECK, Q_SG_HI_AFTER, Q_SG_BR_TAIL, Q_SG_BR_SET,
    Q_SG_BR_END, Q_SG_NEWTON, Q_SG_NEWTON_AFTER, Q_SG_FINAL,
    Q_TP_START, Q_TP_AFTER_INIT, Q_TP_ITER, Q_TP_LS, Q_TP_LS_AFTER,
    Q_STAB_GAS_AFTER, Q_STAB_LIQ_AFTER
};

struct QueueLane {
    unsigned cell;
    int kind;  // 0 all-gas, 1 all-liquid, 2..6 two-phase seed index + 2
    int st;
    CellInput x;
    // pending request and its result
    int req;
    double rm, rp, rT;
    bool rv, ok;
    double pF, pCv, pP, pCp;
    // frozen and two-phase Newton
    double mass, a0, a1, a2;  // frozen: p, T; two-phase: ln p, ln T, beta
    double f0, f1, f2, s0, s1, s2, prev, frac, scale;
    int it, k, stalled;
    // scalar all-gas recovery; g: the last probe's gas-table terms, which the
    // candidate's final point and stability test take once it converged (known)
    double T0, lower, upper, fl, fh, radius, cand, F, cv, P;
    int j, retry;
    bool known;
    GasPoint g;
    CandidateOut o;
};

// Record of a finished candidate: the converged state first, the status after
// the stability test.
__device__ __forceinline__ void recordState(const Eval& v, const QueueLane& L, ReactiveThermoState* st,
                                            double* entropy) {
    stateFromEval(v, L.x.q, L.o, *st);
    *entropy = v.entropyD;
}

// Stability of an all-liquid candidate at (p, T): the gas tangent plane at the
// liquid's chemical potential (no gas branch counts as stable).
__device__ RB200_FLASH_FN bool tangentStable(const HemConst& C, double p, double T, Counts& n) {
    PhaseProps liq, gas;
    if (liquidPhase(C, p, T, true, liq, n) != EOS_OK) return false;
    const double muL = liq.mu / (kGas * T);
    const int status = gasPhase(C, p, T, false, gas, n);
    if (status != EOS_OK) return unavailableStatus(status);
    return (gas.h - T * gas.s) * C.gas.W / (kGas * T) - muL >= -C.mutol;
}

// Acceptance tests of a line-search trial evaluated into v: the residual must
// fall below the current one by the Armijo factor (the frozen partition's also
// accepts a residual already within tolerance).
__device__ __forceinline__ bool tpAccepts(const Eval& v, bool ok, double eIn, double scale, double prev, double frac,
                                          double& t0, double& t1, double& t2) {
    if (!(ok && v.gasMass > 0)) return false;
    t0 = v.volume - 1; t1 = (v.energy - eIn) / scale; t2 = v.muL - v.muG;
    return fin(t2) && fmax(fabs(t0), fmax(fabs(t1), fabs(t2))) < prev * (1 - 1e-4 * frac);
}
__device__ __forceinline__ bool fzAccepts(const HemConst& C, const Eval& v, bool ok, double eIn, double scale,
                                          double prev, double frac) {
    if (!ok) return false;
    const double next = fmax(fabs(v.volume - 1), fabs(v.energy - eIn) / scale);
    return next < prev * (1 - 1e-4 * frac) || next < fmin(C.vtol, C.etol);
}

// Advances one lane's solver until it issues a request (returns true) or the
// candidate is finished (record written; returns false, lane becomes free).
template <class Record>
__device__ inline bool plan(const HemConst& C, QueueLane& L, Eval& v, Record rec, Counts& n, int stallLimitGas) {
    const double q = L.x.q, eIn = L.x.e;
    for (int guard = 0; guard < 256; ++guard) {
        switch (L.st) {
        // ---------------------------------------------------- frozen partition
        case Q_FZ_START:
            if (!fin(eIn)) goto failed;
            if (L.kind == 1 && q * (1 + 1e-12) < C.liquidFloor) goto failed;  // provably cannot converge
            if (L.kind == 0 && C.scalarRecovery && L.mass == 0) {
                L.T0 = clampd(L.x.gT, C.Tmin, C.Tmax);
                L.req = REQ_PROBE; L.rT = L.T0; L.st = Q_SG_AFTER0;
                return true;
            }
            L.st = Q_FZ_NEWTON_INIT;
            continue;
        case Q_FZ_NEWTON_INIT: {
            L.known = false;
            L.a0 = clampd(L.x.gp, C.pmin, C.pmax);
            L.a1 = clampd(L.x.gT, C.Tmin, C.Tmax);
            L.req = REQ_POINT; L.rm = L.mass; L.rp = L.a0; L.rT = L.a1; L.rv = false;
            L.st = Q_FZ_INIT_AFTER;
            return true;
        }
        case Q_FZ_INIT_AFTER:
            if (!L.ok) goto failed;
            L.it = 0; L.stalled = 0; L.st = Q_FZ_ITER;
            continue;
        case Q_FZ_ITER: {
            if (L.it >= 70) goto failed;
            L.scale = energyScale(v, q);
            const double rv = v.volume - 1, re = (v.energy - eIn) / L.scale;
            L.o.vres = fabs(rv); L.o.eres = fabs(re); L.o.cres = 0; L.o.iterations = L.it;
            L.o.soundEq = v.soundFrozen;
            if (fabs(rv) <= C.vtol && fabs(re) <= C.etol) goto converged;
            double a[3][3] = {{v.Vp * L.a0, v.VT * L.a1, 0}, {v.Ep * L.a0 / L.scale, v.ET * L.a1 / L.scale, 0},
                              {0, 0, 0}};
            double b[3] = {-rv, -re, 0}, step[3] = {0, 0, 0};
            if (!solveSmall(a, b, 2, step)) goto failed;
            const double limit = fmax(1., fmax(fabs(step[0]) / .7, fabs(step[1]) / .2));
            L.s0 = step[0] / limit; L.s1 = step[1] / limit;
            L.prev = fmax(fabs(rv), fabs(re));
            L.k = 0; L.frac = 1; L.st = Q_FZ_LS;
            continue;
        }
        case Q_FZ_LS:
            if (L.k >= 30) goto failed;
            L.req = REQ_POINT; L.rm = L.mass; L.rp = L.a0 * exp(L.frac * L.s0); L.rT = L.a1 * exp(L.frac * L.s1);
            L.rv = false; L.st = Q_FZ_LS_AFTER;
            return true;
        case Q_FZ_LS_AFTER:
            {
                if (fzAccepts(C, v, L.ok, eIn, L.scale, L.prev, L.frac)) {
                    L.a0 = L.rp; L.a1 = L.rT;
                    L.stalled = L.frac < 1. / 32 ? L.stalled + 1 : 0;
                    const int limit = L.kind == 0 ? stallLimitGas : 0;
                    if (limit > 0 && L.stalled >= limit
                        && !(fabs(v.volume - 1) <= C.vtol && fabs(v.energy - eIn) / energyScale(v, q) <= C.etol))
                        goto failed;
                    ++L.it; L.st = Q_FZ_ITER;
                    continue;
                }
            }
            ++L.k; L.frac *= .5; L.st = Q_FZ_LS;
            continue;
        // ------------------------------------------------ scalar all-gas recovery
        case Q_SG_AFTER0:
            if (!L.ok) { L.st = Q_FZ_NEWTON_INIT; continue; }
            L.F = L.pF; L.cv = L.pCv; L.P = L.pP;
            L.scale = fmax(1e5 * q, q * L.pCp * L.T0);
            L.lower = L.upper = L.T0; L.fl = L.fh = L.F;
            if (fabs(L.F) > C.etol * L.scale) {
                L.radius = fmax(1., .01 * L.T0); L.j = 0; L.st = Q_SG_BR_LOOP;
            } else { L.it = 0; L.st = Q_SG_NEWTON; }
            continue;
        case Q_SG_BR_LOOP:
            if (!(L.j < 24 && (L.fl > 0 || L.fh < 0))) { L.st = Q_SG_BR_END; continue; }
            if (L.fl > 0) {
                L.cand = fmax(C.Tmin, L.T0 - L.radius); L.retry = 0;
                L.req = REQ_PROBE; L.rT = L.cand; L.st = Q_SG_LO_AFTER;
                return true;
            }
            L.st = Q_SG_HI_CHECK;
            continue;
        case Q_SG_LO_AFTER:
            if (L.ok) { L.fl = L.pF; L.lower = L.cand; L.st = Q_SG_HI_CHECK; continue; }
            L.cand = .5 * (L.lower + L.cand);
            if (++L.retry >= 8) { L.st = Q_FZ_NEWTON_INIT; continue; }
            L.req = REQ_PROBE; L.rT = L.cand;
            return true;
        case Q_SG_HI_CHECK:
            if (L.fh < 0) {
                L.cand = fmin(C.Tmax, L.T0 + L.radius); L.retry = 0;
                L.req = REQ_PROBE; L.rT = L.cand; L.st = Q_SG_HI_AFTER;
                return true;
            }
            L.st = Q_SG_BR_TAIL;
            continue;
        case Q_SG_HI_AFTER:
            if (L.ok) { L.fh = L.pF; L.upper = L.cand; L.st = Q_SG_BR_TAIL; continue; }
            L.cand = .5 * (L.upper + L.cand);
            if (++L.retry >= 8) { L.st = Q_FZ_NEWTON_INIT; continue; }
            L.req = REQ_PROBE; L.rT = L.cand;
            return true;
        case Q_SG_BR_TAIL:
            if (fabs(L.fl) <= C.etol * L.scale) {
                L.T0 = L.lower; L.req = REQ_PROBE; L.rT = L.T0; L.st = Q_SG_BR_SET;
                return true;
            }
            if (fabs(L.fh) <= C.etol * L.scale) {
                L.T0 = L.upper; L.req = REQ_PROBE; L.rT = L.T0; L.st = Q_SG_BR_SET;
                return true;
            }
            if (L.lower == C.Tmin && L.upper == C.Tmax) { L.st = Q_SG_BR_END; continue; }
            ++L.j; L.radius *= 2; L.st = Q_SG_BR_LOOP;
            continue;
        case Q_SG_BR_SET:
            if (!L.ok) { L.st = Q_FZ_NEWTON_INIT; continue; }
            L.F = L.pF; L.cv = L.pCv; L.P = L.pP; L.st = Q_SG_BR_END;
            continue;
        case Q_SG_BR_END:
            if (!(fabs(L.F) <= C.etol * L.scale || (L.fl <= 0 && L.fh >= 0 && L.upper > L.lower))) {
                L.st = Q_FZ_NEWTON_INIT;
                continue;
            }
            L.it = 0; L.st = Q_SG_NEWTON;
            continue;
        case Q_SG_NEWTON: {
            if (!(L.it < 70 && fabs(L.F) > C.etol * L.scale)) {
                if (fabs(L.F) > C.etol * L.scale) { L.st = Q_FZ_NEWTON_INIT; continue; }
                // (P, T0) are the last probe's point: its terms serve the final evaluation
                L.req = REQ_POINT; L.rm = 0; L.rp = L.P; L.rT = L.T0; L.rv = false; L.known = true;
                L.st = Q_SG_FINAL;
                return true;
            }
            if (L.F > 0) L.upper = L.T0; else L.lower = L.T0;
            const double next = L.T0 - L.F / L.cv;
            L.T0 = fin(next) && next > L.lower && next < L.upper ? next : .5 * (L.lower + L.upper);
            L.req = REQ_PROBE; L.rT = L.T0; L.st = Q_SG_NEWTON_AFTER;
            return true;
        }
        case Q_SG_NEWTON_AFTER:
            if (!L.ok) { L.st = Q_FZ_NEWTON_INIT; continue; }
            L.F = L.pF; L.cv = L.pCv; L.P = L.pP; ++L.it; L.st = Q_SG_NEWTON;
            continue;
        case Q_SG_FINAL:
            if (!L.ok) { L.st = Q_FZ_NEWTON_INIT; continue; }
            L.o.vres = fabs(v.volume - 1);
            L.o.eres = fabs(v.energy - eIn) / energyScale(v, q);
            L.o.cres = 0;
            L.o.iterations = L.it;
            L.o.soundEq = v.soundFrozen;
            if (L.o.vres <= C.vtol && L.o.eres <= C.etol) goto converged;
            L.st = Q_FZ_NEWTON_INIT;
            continue;
        // ------------------------------------------------------------ two-phase
        case Q_TP_START: {
            ++n.candidates;
            const double gT = L.x.gT;
            L.scale = fmax(1e5 * q, fmax(fabs(eIn), q * 2000 * fmax(gT, C.Tmin)));
            L.a0 = log(clampd(L.x.gp, C.pmin, C.pmax));
            L.a1 = log(clampd(gT, C.Tmin, C.Tmax));
            const int si = L.kind - 2;
            const double seed = si == 0 ? -1.0 : si == 1 ? .5 : si == 2 ? .95 : si == 3 ? .1 : .9999;
            L.a2 = seed < 0 ? clampd(L.x.gml / q, 1e-8, 1 - 1e-8) : seed;
            ++n.residuals;
            if (!(L.a2 >= 0 && L.a2 < 1)) goto failed;
            L.req = REQ_POINT; L.rm = L.a2 * q; L.rp = exp(L.a0); L.rT = exp(L.a1); L.rv = true;
            L.st = Q_TP_AFTER_INIT;
            return true;
        }
        case Q_TP_AFTER_INIT:
            if (!(L.ok && v.gasMass > 0)) goto failed;
            L.f0 = v.volume - 1; L.f1 = (v.energy - eIn) / L.scale; L.f2 = v.muL - v.muG;
            if (!fin(L.f2)) goto failed;
            L.it = 0; L.st = Q_TP_ITER;
            continue;
        case Q_TP_ITER: {
            if (L.it >= 90) goto failed;
            double J[3][3];
            const double x[3] = {L.a0, L.a1, L.a2}, f[3] = {L.f0, L.f1, L.f2};
            const double chemical = fabs(L.f2);
            if (fabs(L.f0) <= C.vtol && fabs(L.f1) <= C.etol && chemical <= C.mutol) {
                L.o.vres = fabs(L.f0); L.o.eres = fabs(L.f1); L.o.cres = chemical; L.o.iterations = L.it;
                if (!jacobian(C, L.x, x, L.scale, f, v, J, n)) goto failed;
                double rhs[3] = {-1 / q, v.p / (q * L.scale), 0}, response[3] = {0, 0, 0};
                if (!solveSmall(J, rhs, 3, response)) goto failed;
                const double squared = v.p * response[0];
                if (!fin(squared) || squared <= 0) goto failed;
                L.o.soundEq = sqrt(squared);
                if (!(L.o.soundEq <= v.soundFrozen * (1 + 2e-3))) goto failed;
                goto converged;
            }
            if (!jacobian(C, L.x, x, L.scale, f, v, J, n)) goto failed;
            double rhs[3] = {-L.f0, -L.f1, -L.f2}, step[3] = {0, 0, 0};
            if (!solveSmall(J, rhs, 3, step)) goto failed;
            const double limiter =
                fmax(fmax(1., fmax(fabs(step[0]) / .7, fabs(step[1]) / .18)), fabs(step[2]) / .3);
            L.s0 = step[0] / limiter; L.s1 = step[1] / limiter; L.s2 = step[2] / limiter;
            L.prev = fmax(fabs(L.f0), fmax(fabs(L.f1), fabs(L.f2)));
            L.k = 0; L.frac = 1; L.st = Q_TP_LS;
            continue;
        }
        case Q_TP_LS: {
            // beta outside [0, 1) is rejected without an evaluation
            while (L.k < 30 && !(L.a2 + L.frac * L.s2 >= 0 && L.a2 + L.frac * L.s2 < 1)) {
                ++n.residuals; ++L.k; L.frac *= .5;
            }
            if (L.k >= 30) goto failed;
            ++n.residuals;
            L.req = REQ_POINT;
            L.rm = (L.a2 + L.frac * L.s2) * q;
            L.rp = exp(L.a0 + L.frac * L.s0);
            L.rT = exp(L.a1 + L.frac * L.s1);
            L.rv = true;
            L.st = Q_TP_LS_AFTER;
            return true;
        }
        case Q_TP_LS_AFTER: {
            double t0, t1, t2;
            if (tpAccepts(v, L.ok, eIn, L.scale, L.prev, L.frac, t0, t1, t2)) {
                L.a0 = L.a0 + L.frac * L.s0; L.a1 = L.a1 + L.frac * L.s1; L.a2 = L.a2 + L.frac * L.s2;
                L.f0 = t0; L.f1 = t1; L.f2 = t2;
                ++L.it; L.st = Q_TP_ITER;
                continue;
            }
            ++L.k; L.frac *= .5; L.st = Q_TP_LS;
            continue;
        }
        // ----------------------------------------------------------- stability
        case Q_STAB_GAS_AFTER: {
            bool stable = false;
            if (L.ok) {
                const double affinity = v.muL - v.muG;
                stable = L.rm > 0 ? (fin(affinity) && fabs(affinity) <= C.mutol * 2) : !(affinity < -C.mutol);
            }
            rec.status(L, stable ? 2 : 1);
            if (stable) ++n.stable; else ++n.failures;
            L.st = Q_FREE;
            return false;
        }
        case Q_STAB_LIQ_AFTER: {
            const bool stable = L.ok;
            rec.status(L, stable ? 2 : 1);
            if (stable) ++n.stable; else ++n.failures;
            L.st = Q_FREE;
            return false;
        }
        default:
            L.st = Q_FREE;
            return false;
        }
    converged:
        rec.state(L, v);
        if (v.gasMass > 0) {
            if (L.kind >= 2) {  // the converged residual evaluation is the stability point
                const double affinity = L.f2;
                const bool stable = v.liqMass > 0 ? (fin(affinity) && fabs(affinity) <= C.mutol * 2)
                                                  : !(affinity < -C.mutol);
                rec.status(L, stable ? 2 : 1);
                if (stable) ++n.stable; else ++n.failures;
                L.st = Q_FREE;
                return false;
            }
            L.req = REQ_POINT; L.rm = v.liqMass; L.rp = v.p; L.rT = v.T; L.rv = true;
            L.st = Q_STAB_GAS_AFTER;
            return true;
        }
        if (!(v.liqMass > 0)) {
            rec.status(L, 1);
            ++n.failures;
            L.st = Q_FREE;
            return false;
        }
        L.req = REQ_TANGENT; L.rp = v.p; L.rT = v.T; L.st = Q_STAB_LIQ_AFTER;
        return true;
    failed:
        rec.status(L, 0);
        ++n.failures;
        L.st = Q_FREE;
        return false;
    }
    rec.status(L, 0);
    ++n.failures;
    L.st = Q_FREE;
    return false;
}

}  // namespace rb200
