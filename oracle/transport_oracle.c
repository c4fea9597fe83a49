/* TEST INFRASTRUCTURE ONLY (see oracle.h): serial CPU restatement of the
 * reference transport operator as a face loop that scatters each face's flux to
 * its owner (-) and neighbour (+), the structure of the reference's independent
 * NumPy check (tools/validate_reactive_transport.py:64-127). Physics per face
 * follows src/reactiveTransport/reactiveTransportKernels.h:
 *   right-state rules (slip mirror, extrapolate, fixed state)   :134-149
 *   Green-Gauss velocity gradient                               :290-301
 *   WALE nu_t (src/reactiveTransport/reactiveWale.h:87-190)      :303-313
 *   CFL face speed                                              :315-341
 *   HLL coefficients, viscous/WALE traction, conduction, Fick   :343-461
 *   flux assembly per variable                                  :180-191
 *   mechanical dilatation source                                :520-524
 *   CFL step and absorbing invalid minimum                      :529-549, reactiveTransport.cpp:222-232 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

typedef struct {
    const ReactiveTransportConfig* cfg;
    const ReactiveTransportFace* faces;
    const double* volume;
    const double* q; const ReactiveTransportState* s;
    const double* fq; const ReactiveTransportState* fs;
    const double* gy; const double* gh; const double* fy; const double* fh;
    double* u;  /* cells x 3 velocities */
    double* fu; /* fixed x 3 */
    double* grad; /* cells x 9 */
    double* nut;  /* cells */
    int wale;
} Ctx;

static double minimum(double a, double b) { return a < b ? a : b; }
static double maximum(double a, double b) { return a > b ? a : b; }

static void velocities(const double* row, size_t ns, double* u) {
    double rho = 0;
    for (size_t k = 0; k < ns; ++k) rho += row[k];
    for (int d = 0; d < 3; ++d) u[d] = row[ns + d] / rho;
}

/* Left/right conserved rows, states and velocities of one face. */
static void sides(const Ctx* c, const ReactiveTransportFace* f, const double** ql, double* qrBuf,
                  const double** qr, const ReactiveTransportState** sl, const ReactiveTransportState** sr,
                  double* ul, double* ur) {
    const size_t nv = c->cfg->variables, ns = c->cfg->species;
    *ql = c->q + (size_t)f->owner * nv;
    *sl = c->s + f->owner;
    memcpy(ul, c->u + 3 * f->owner, 3 * sizeof(double));
    if (f->neighbour >= 0) {
        *qr = c->q + (size_t)f->neighbour * nv;
        *sr = c->s + f->neighbour;
        memcpy(ur, c->u + 3 * f->neighbour, 3 * sizeof(double));
    } else if (f->kind == 3) {
        *qr = c->fq + (size_t)f->fixed * nv;
        *sr = c->fs + f->fixed;
        memcpy(ur, c->fu + 3 * f->fixed, 3 * sizeof(double));
    } else {
        *qr = *ql;
        *sr = *sl;
        memcpy(ur, ul, 3 * sizeof(double));
        if (f->kind == 1) {
            double dm = 0, du = 0;
            memcpy(qrBuf, *ql, nv * sizeof(double));
            for (int d = 0; d < 3; ++d) { dm += (*ql)[ns + d] * f->normal[d]; du += ul[d] * f->normal[d]; }
            for (int d = 0; d < 3; ++d) { qrBuf[ns + d] -= 2 * dm * f->normal[d]; ur[d] -= 2 * du * f->normal[d]; }
            *qr = qrBuf;
        }
    }
}

/* WALE (Nicoud-Ducros) with normalised invariants and binary-exponent scaling. */
static int wale_nut(const double* g, double delta, double cw, double* nut) {
    double scale = 0, h[9], sq[9], trace, ss = 0, dd = 0;
    *nut = 0;
    if (!isfinite(delta) || delta < 0 || !isfinite(cw) || cw < 0) return 0;
    for (int i = 0; i < 9; ++i) { if (!isfinite(g[i])) return 0; scale = maximum(scale, fabs(g[i])); }
    if (scale == 0 || cw == 0 || delta == 0) return 1;
    for (int i = 0; i < 9; ++i) h[i] = g[i] / scale;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            sq[3 * i + j] = 0;
            for (int k = 0; k < 3; ++k) sq[3 * i + j] += h[3 * i + k] * h[3 * k + j];
        }
    trace = sq[0] + sq[4] + sq[8];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const double s = 0.5 * (h[3 * i + j] + h[3 * j + i]);
            double dv = 0.5 * (sq[3 * i + j] + sq[3 * j + i]);
            if (i == j) dv -= trace / 3.0;
            ss += s * s; dd += dv * dv;
        }
    if (!isfinite(ss) || !isfinite(dd)) return 0;
    if (dd == 0) return 1;
    {
        const double num = dd * sqrt(dd), den = ss * ss * sqrt(ss) + dd * sqrt(sqrt(dd));
        int e1, e2, e3, e4, e5;
        double ratio, m;
        if (!(den > 0) || !isfinite(den) || !isfinite(num)) return 0;
        ratio = num / den;
        if (ratio == 0) return 1;
        {
            const double mc = frexp(cw, &e1), md = frexp(delta, &e2), mg = frexp(scale, &e3), mr = frexp(ratio, &e4);
            m = frexp(mc * mc * md * md * mg * mr, &e5);
        }
        *nut = ldexp(m, 2 * e1 + 2 * e2 + e3 + e4 + e5);
        return isfinite(*nut);
    }
}

/* Exported for the WALE known-answer tests. */
int oracle_wale_nut(const double* g, double delta, double cw, double* nut) { return wale_nut(g, delta, cw, nut); }

static int setup(Ctx* c, int needGradients) {
    const ReactiveTransportConfig* cfg = c->cfg;
    const size_t ns = cfg->species, nv = cfg->variables;
    int ok = 1;
    c->u = malloc(3 * cfg->cells * sizeof(double));
    c->fu = malloc(3 * (cfg->fixed + 1) * sizeof(double));
    c->grad = calloc(9 * cfg->cells, sizeof(double));
    c->nut = calloc(cfg->cells, sizeof(double));
    for (size_t i = 0; i < cfg->cells; ++i) velocities(c->q + i * nv, ns, c->u + 3 * i);
    for (size_t i = 0; i < cfg->fixed; ++i) velocities(c->fq + i * nv, ns, c->fu + 3 * i);
    if (!needGradients) return 1;
    for (size_t fi = 0; fi < cfg->faces; ++fi) {
        const ReactiveTransportFace* f = c->faces + fi;
        const double *ql, *qr;
        const ReactiveTransportState *sl, *sr;
        double buf[1024], ul[3], ur[3];
        double* big = nv > 1024 ? malloc(nv * sizeof(double)) : buf;
        sides(c, f, &ql, big, &qr, &sl, &sr, ul, ur);
        for (int i = 0; i < 3; ++i) {
            const double uf = f->ownerWeight * ul[i] + (1 - f->ownerWeight) * ur[i];
            for (int d = 0; d < 3; ++d) {
                const double contribution = uf * f->normal[d] * f->area;
                c->grad[9 * f->owner + 3 * i + d] += contribution / c->volume[f->owner];
                if (f->neighbour >= 0) c->grad[9 * f->neighbour + 3 * i + d] -= contribution / c->volume[f->neighbour];
            }
        }
        if (big != buf) free(big);
    }
    return ok;
}

static int compute_nut(Ctx* c, double cw) {
    for (size_t i = 0; i < c->cfg->cells; ++i) {
        double nut;
        const double delta = cbrt(c->volume[i]);
        if (!wale_nut(c->grad + 9 * i, delta, cw, &nut) || !isfinite(nut) || nut < 0
            || !isfinite(c->s[i].rho * nut))
            return 0;
        c->nut[i] = nut;
    }
    return 1;
}

static void teardown(Ctx* c) { free(c->u); free(c->fu); free(c->grad); free(c->nut); }

static double face_nut(const Ctx* c, const ReactiveTransportFace* f, int right) {
    if (!c->wale) return 0;
    return c->nut[right && f->neighbour >= 0 ? f->neighbour : f->owner];
}

/* WALE scalar closure (src/reactiveTransport/reactiveTransport.cpp:653-702,
 * reactiveTransportKernels.h:150-168, :323-336, :440-444, :462-477): turbulent
 * Prandtl / Schmidt numbers (0 disables that flux) and the caller's fields:
 * mixture cp per cell and per fixed state, effective species enthalpies
 * (cell-major). Active only together with WALE. */
static double g_pr = 0, g_sc = 0;
static const double *g_cellCp, *g_fixedCp, *g_cellH, *g_fixedH;
void oracle_set_wale_scalars(double pr, double sc, const double* cellCp, const double* fixedCp,
                             const double* cellH, const double* fixedH) {
    g_pr = pr; g_sc = sc; g_cellCp = cellCp; g_fixedCp = fixedCp; g_cellH = cellH; g_fixedH = fixedH;
}

/* cp and species enthalpies of the face's right cell (the owner's for slip and extrapolate). */
static double right_cp(const ReactiveTransportFace* f) {
    if (f->neighbour >= 0) return g_cellCp[f->neighbour];
    if (f->kind == 3) return g_fixedCp[f->fixed];
    return g_cellCp[f->owner];
}
static const double* right_h(const ReactiveTransportFace* f, size_t ns) {
    if (f->neighbour >= 0) return g_cellH + (size_t)f->neighbour * ns;
    if (f->kind == 3) return g_fixedH + (size_t)f->fixed * ns;
    return g_cellH + (size_t)f->owner * ns;
}

/* CFL face speed (-1 when invalid). */
static double face_speed(const Ctx* c, const ReactiveTransportFace* f) {
    const ReactiveTransportConfig* cfg = c->cfg;
    const double *ql, *qr;
    const ReactiveTransportState *sl, *sr;
    double buf[1024], ul[3], ur[3], unL = 0, unR = 0;
    double* big = cfg->variables > 1024 ? malloc(cfg->variables * sizeof(double)) : buf;
    double aL, aR, left, right, rhoNut, mu, D, speed;
    sides(c, f, &ql, big, &qr, &sl, &sr, ul, ur);
    for (int d = 0; d < 3; ++d) { unL += ul[d] * f->normal[d]; unR += ur[d] * f->normal[d]; }
    aL = cfg->waveFactor * sl->sound; aR = cfg->waveFactor * sr->sound;
    left = minimum(0, minimum(unL - aL, unR - aR)); right = maximum(0, maximum(unL + aL, unR + aR));
    rhoNut = c->wale ? f->ownerWeight * sl->rho * face_nut(c, f, 0) + (1 - f->ownerWeight) * sr->rho * face_nut(c, f, 1) : 0;
    mu = cfg->viscosity + rhoNut;
    D = cfg->diffusivity + maximum(maximum(4 * mu / (3 * sl->rho), 4 * mu / (3 * sr->rho)),
                                   maximum(cfg->conductivity / (sl->rho * sl->cv), cfg->conductivity / (sr->rho * sr->cv)));
    {
        double scalar = 0;
        if (c->wale && (g_pr > 0 || g_sc > 0) && f->kind != 1) {
            if (g_pr > 0) {
                const double k = rhoNut * (f->ownerWeight * g_cellCp[f->owner] + (1 - f->ownerWeight) * right_cp(f))
                    / g_pr;
                scalar = maximum(scalar, maximum(k / (sl->rho * sl->cv), k / (sr->rho * sr->cv)));
            }
            if (g_sc > 0) scalar = maximum(scalar, maximum(rhoNut / sl->rho, rhoNut / sr->rho) / g_sc);
        }
        speed = maximum(fabs(unL) + aL, fabs(unR) + aR) + 2 * (D + scalar) / f->distance;
    }
    if (!isfinite(unL) || !isfinite(unR) || !isfinite(speed) || !isfinite(1 / (right - left)) || right <= left) speed = -1;
    if (big != buf) free(big);
    return speed;
}

static void gas_side(const Ctx* c, const ReactiveTransportFace* f, int right, const double** y, const double** h) {
    const size_t ns = c->cfg->species;
    if (!right || f->neighbour >= 0) {
        const size_t cell = (size_t)(right ? f->neighbour : f->owner);
        *y = c->gy + cell * ns; *h = c->gh + cell * ns;
    } else if (f->kind == 3) {
        *y = c->fy + (size_t)f->fixed * ns; *h = c->fh + (size_t)f->fixed * ns;
    } else {
        *y = c->gy + (size_t)f->owner * ns; *h = c->gh + (size_t)f->owner * ns;
    }
}

/* Flux scheme of oracle_transport_rhs: 0 HLL, 1 HLLC. */
static int g_scheme = 0;
void oracle_set_flux_scheme(int scheme) { g_scheme = scheme; }

/* HLLC face coefficients: the reference's contact-preserving core
 * (src/reactiveInterface/reactiveBalancedCapillary.h:55-142) with no capillary
 * terms (sigma = 0, so pi = p), as the transport's Faces functor applies it
 * (src/reactiveTransport/reactiveTransportKernels.h:357-417): wave speeds from
 * waveFactor * sound, star speed from the two one-sided momentum balances,
 * the HLL coefficients when the star speed leaves (S_L, S_R), else the upwind
 * star (or supersonic) state of the side the contact moves away from.
 * out = {contact speed, advectLeft, advectRight, pressureMomentum, pressureEnergy}.
 * Returns 0 when the face cannot be formed (the reference's capillary failure). */
int oracle_hllc_face(double rhoL, const double uL[3], double pL, double aL, double EL, double rhoR,
                     const double uR[3], double pR, double aR, double ER, const double normal[3], double out[5]) {
    double unL = 0, unR = 0, sl, sr, den, star;
    if (!(isfinite(rhoL) && rhoL > 0 && isfinite(rhoR) && rhoR > 0 && isfinite(pL) && pL > 0 && isfinite(pR)
          && pR > 0 && isfinite(aL) && aL > 0 && isfinite(aR) && aR > 0 && isfinite(EL) && isfinite(ER)))
        return 0;
    for (int d = 0; d < 3; ++d) { unL += uL[d] * normal[d]; unR += uR[d] * normal[d]; }
    sl = minimum(0, minimum(unL - aL, unR - aR));
    sr = maximum(0, maximum(unL + aL, unR + aR));
    den = rhoL * (sl - unL) - rhoR * (sr - unR);
    if (!isfinite(den) || den == 0 || !isfinite(sl) || !isfinite(sr) || sr <= sl) return 0;
    star = (pR - pL + rhoL * unL * (sl - unL) - rhoR * unR * (sr - unR)) / den;
    if (!isfinite(star) || star <= sl || star >= sr) {
        const double inv = 1 / (sr - sl);
        out[0] = (sr * unL - sl * unR) * inv;
        out[1] = sr * (unL - sl) * inv;
        out[2] = sl * (sr - unR) * inv;
        out[3] = (sr * pL - sl * pR) * inv;
        out[4] = (sr * pL * unL - sl * pR * unR) * inv;
    } else {
        const int left = star >= 0;
        const double rho = left ? rhoL : rhoR, un = left ? unL : unR, wave = left ? sl : sr;
        const double p = left ? pL : pR, E = left ? EL : ER;
        const int supersonic = (left && sl >= 0) || (!left && sr <= 0);
        double mass;
        out[0] = supersonic ? un : star;
        if (supersonic) {
            mass = rho * un;
            out[3] = p;
            out[4] = p * un;
        } else {
            const double rhoStar = rho * (wave - un) / (wave - star);
            const double pStar = p + rho * (wave - un) * (star - un);
            const double eStar = ((wave - un) * E - p * un + pStar * star) / (wave - star);
            mass = rhoStar * star;
            out[3] = pStar + mass * (star - un);
            out[4] = star * (eStar + pStar) - mass * E / rho;
        }
        out[1] = left ? mass / rhoL : 0;
        out[2] = left ? 0 : mass / rhoR;
    }
    for (int k = 0; k < 5; ++k)
        if (!isfinite(out[k])) return 0;
    return 1;
}

int oracle_transport_rhs(const ReactiveTransportConfig* cfg, const double* volume,
    const ReactiveTransportFace* faces, const double* fixedQ, const ReactiveTransportState* fixedStates,
    const double* fixedY, const double* fixedH, double waleCw,
    const double* q, const ReactiveTransportState* states, const double* gasY, const double* gasH,
    double* rhs, double* boundary, double* nutOut, double* denominator) {
    const size_t ns = cfg->species, nv = cfg->variables, nc = cfg->cells;
    Ctx c = {cfg, faces, volume, q, states, fixedQ, fixedStates, gasY, gasH, fixedY, fixedH,
             NULL, NULL, NULL, NULL, waleCw >= 0};
    double* flux = malloc(nv * sizeof(double));
    double* qrBuf = malloc(nv * sizeof(double));
    double* div = calloc(nc, sizeof(double));
    int status = 0;
    setup(&c, cfg->viscosity > 0 || c.wale);
    if (c.wale && !compute_nut(&c, waleCw)) status = 1;
    if (nutOut) memcpy(nutOut, c.nut, nc * sizeof(double));
    memset(rhs, 0, nc * nv * sizeof(double));
    memset(boundary, 0, nv * sizeof(double));
    if (denominator) memset(denominator, 0, nc * sizeof(double));
    for (size_t fi = 0; fi < cfg->faces; ++fi) {
        const ReactiveTransportFace* f = faces + fi;
        const double *ql, *qr;
        const ReactiveTransportState *sl, *sr;
        const double w = f->ownerWeight;
        double ul[3], ur[3], unL = 0, unR = 0, aL, aR, left, right, inv;
        double advL, advR, pM, pE, fv, traction[3] = {0, 0, 0}, energy = 0;
        sides(&c, f, &ql, qrBuf, &qr, &sl, &sr, ul, ur);
        for (int d = 0; d < 3; ++d) { unL += ul[d] * f->normal[d]; unR += ur[d] * f->normal[d]; }
        aL = cfg->waveFactor * sl->sound; aR = cfg->waveFactor * sr->sound;
        left = minimum(0, minimum(unL - aL, unR - aR)); right = maximum(0, maximum(unL + aL, unR + aR));
        inv = 1 / (right - left);
        fv = (right * unL - left * unR) * inv;
        advL = right * (unL - left) * inv;
        advR = left * (right - unR) * inv;
        pM = (right * sl->p - left * sr->p) * inv;
        pE = (right * sl->p * unL - left * sr->p * unR) * inv;
        if (g_scheme == 1) {
            double h[5];
            const double EL = ql[ns + 3], ER = qr[ns + 3];
            if (!oracle_hllc_face(sl->rho, ul, sl->p, aL, EL, sr->rho, ur, sr->p, aR, ER, f->normal, h)) status = 3;
            fv = h[0]; advL = h[1]; advR = h[2]; pM = h[3]; pE = h[4];
        }
        if (denominator) {
            const double speed = face_speed(&c, f);
            if (speed < 0) status = 2;
            denominator[f->owner] += f->area * speed;
            if (f->neighbour >= 0) denominator[f->neighbour] += f->area * speed;
        }
        if (cfg->viscosity > 0 || c.wale) {
            double g[9], dv, mu;
            for (int j = 0; j < 9; ++j) {
                g[j] = c.grad[9 * f->owner + j];
                if (f->neighbour >= 0) g[j] = w * g[j] + (1 - w) * c.grad[9 * f->neighbour + j];
            }
            for (int i = 0; i < 3; ++i) {
                double normal = 0, target;
                for (int d = 0; d < 3; ++d) normal += g[3 * i + d] * f->normal[d];
                target = (ur[i] - ul[i]) / ((f->kind == 1 ? 2 : 1) * f->distance);
                for (int d = 0; d < 3; ++d) g[3 * i + d] += f->normal[d] * (target - normal);
            }
            dv = g[0] + g[4] + g[8];
            mu = cfg->viscosity + (c.wale ? w * sl->rho * face_nut(&c, f, 0) + (1 - w) * sr->rho * face_nut(&c, f, 1) : 0);
            for (int i = 0; i < 3; ++i)
                for (int d = 0; d < 3; ++d)
                    traction[i] += mu * (g[3 * i + d] + g[3 * d + i] - (i == d ? 2 * dv / 3 : 0)) * f->normal[d];
            if (f->kind == 1) {
                double dot = 0;
                for (int d = 0; d < 3; ++d) dot += traction[d] * f->normal[d];
                for (int d = 0; d < 3; ++d) traction[d] = dot * f->normal[d];
            }
            for (int d = 0; d < 3; ++d) energy -= traction[d] * (w * ul[d] + (1 - w) * ur[d]);
        }
        if (cfg->conductivity > 0 && f->kind != 1) energy -= cfg->conductivity * (sr->T - sl->T) / f->distance;
        if (c.wale && g_pr > 0 && f->kind != 1) {
            const double rhoNut = w * sl->rho * face_nut(&c, f, 0) + (1 - w) * sr->rho * face_nut(&c, f, 1);
            const double cp = w * g_cellCp[f->owner] + (1 - w) * right_cp(f);
            energy -= rhoNut * cp / g_pr * (sr->T - sl->T) / f->distance;
        }
        for (size_t k = 0; k < nv; ++k) flux[k] = advL * ql[k] + advR * qr[k];
        for (int d = 0; d < 3; ++d) flux[ns + d] += pM * f->normal[d] - traction[d];
        flux[ns + 3] += pE + energy;
        if (cfg->diffusivity > 0 && sl->gasMass > 0 && sr->gasMass > 0 && f->kind != 1) {
            const double *yl, *yr, *hl, *hr;
            const double mass = f->neighbour >= 0 ? sl->gasMass * sr->gasMass / ((1 - w) * sr->gasMass + w * sl->gasMass)
                                                  : sl->gasMass;
            const double diffusion = -mass * cfg->diffusivity / f->distance;
            double sumJ = 0, largest = -1, carrierFlux = 0, hc;
            size_t carrier = 0;
            gas_side(&c, f, 0, &yl, &hl);
            gas_side(&c, f, 1, &yr, &hr);
            for (size_t k = 0; k < ns; ++k) {
                const double y = w * yl[k] + (1 - w) * yr[k];
                sumJ += diffusion * (yr[k] - yl[k]);
                if (y > largest) { largest = y; carrier = k; }
            }
            hc = w * hl[carrier] + (1 - w) * hr[carrier];
            for (size_t k = 0; k < ns; ++k) {
                double J;
                if (k == carrier) continue;
                J = diffusion * (yr[k] - yl[k]) - (w * yl[k] + (1 - w) * yr[k]) * sumJ;
                carrierFlux -= J;
                flux[k] += J;
                flux[ns + 3] += J * ((w * hl[k] + (1 - w) * hr[k]) - hc);
            }
            flux[carrier] += carrierFlux;
        }
        if (c.wale && g_sc > 0 && f->kind != 1) {
            const double rhoNut = w * sl->rho * face_nut(&c, f, 0) + (1 - w) * sr->rho * face_nut(&c, f, 1);
            const double sgs = -rhoNut / g_sc / f->distance;
            const double *hl = g_cellH + (size_t)f->owner * ns, *hr = right_h(f, ns);
            double sumJ = 0, largest = -1, carrierFlux = 0, hc;
            size_t carrier = 0;
            for (size_t k = 0; k < ns; ++k) {
                const double yl = ql[k] / sl->rho, yr = qr[k] / sr->rho;
                const double y = w * yl + (1 - w) * yr;
                sumJ += sgs * (yr - yl);
                if (y > largest) { largest = y; carrier = k; }
            }
            hc = w * hl[carrier] + (1 - w) * hr[carrier];
            for (size_t k = 0; k < ns; ++k) {
                double J;
                const double yl = ql[k] / sl->rho, yr = qr[k] / sr->rho;
                if (k == carrier) continue;
                J = sgs * (yr - yl) - (w * yl + (1 - w) * yr) * sumJ;
                carrierFlux -= J;
                flux[k] += J;
                flux[ns + 3] += J * ((w * hl[k] + (1 - w) * hr[k]) - hc);
            }
            flux[carrier] += carrierFlux;
        }
        for (size_t k = 0; k < nv; ++k) {
            const double rate = flux[k] * f->area;
            rhs[f->owner * nv + k] -= rate / volume[f->owner];
            if (f->neighbour >= 0) rhs[f->neighbour * nv + k] += rate / volume[f->neighbour];
            else boundary[k] += rate;
        }
        if (cfg->mechanical) {
            div[f->owner] += fv * f->area / volume[f->owner];
            if (f->neighbour >= 0) div[f->neighbour] -= fv * f->area / volume[f->neighbour];
        }
    }
    if (cfg->mechanical)
        for (size_t i = 0; i < nc; ++i) {
            rhs[i * nv + ns + 4] += (q[i * nv + ns + 4] + states[i].dilatation) * div[i];
            rhs[i * nv + ns + 5] += (q[i * nv + ns + 5] - states[i].dilatation) * div[i];
        }
    free(flux); free(qrBuf); free(div);
    teardown(&c);
    return status;
}

double oracle_transport_stable_dt(const ReactiveTransportConfig* cfg, const double* volume,
    const ReactiveTransportFace* faces, const double* fixedQ, const ReactiveTransportState* fixedStates,
    double waleCw, const double* q, const ReactiveTransportState* states, double cfl, double maximumStep) {
    const size_t nc = cfg->cells;
    Ctx c = {cfg, faces, volume, q, states, fixedQ, fixedStates, NULL, NULL, NULL, NULL,
             NULL, NULL, NULL, NULL, waleCw >= 0};
    double* denominator = calloc(nc, sizeof(double));
    double dt = maximumStep;
    int bad = 0;
    setup(&c, c.wale);
    if (c.wale && !compute_nut(&c, waleCw)) bad = 1;
    for (size_t fi = 0; fi < cfg->faces && !bad; ++fi) {
        const double speed = face_speed(&c, faces + fi);
        if (!(speed >= 0) || !isfinite(speed)) { bad = 1; break; }
        denominator[faces[fi].owner] += faces[fi].area * speed;
        if (faces[fi].neighbour >= 0) denominator[faces[fi].neighbour] += faces[fi].area * speed;
    }
    for (size_t i = 0; i < nc && !bad; ++i) {
        if (!isfinite(denominator[i]) || denominator[i] < 0) { bad = 1; break; }
        if (denominator[i] > 0) dt = minimum(dt, cfl * volume[i] / denominator[i]);
    }
    free(denominator);
    teardown(&c);
    return bad || !(dt > 0) ? -1 : dt;
}
