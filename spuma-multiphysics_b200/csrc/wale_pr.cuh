// Phase-aware Peng-Robinson scalar properties of the WALE closure at an
// accepted UV state (src/reactiveThermo/reactiveDeviceWalePr.h:20-103): the
// mixture heat capacity of the state and, per species, the effective enthalpy
// h_k = (gas_k hbar_k^gas + [k condensable] m_l h_l) / q_k that the turbulent
// species flux carries, with the gas phase at p - color*jump and the liquid at
// p + (1 - color)*jump. A property evaluation at a state the flash accepted,
// never another flash: every inventory, density, volume and energy of the
// state is checked against the phases it implies (within max(1e-8, 50 vtol)),
// and a mismatch is a status, not a repair. Host and device from one source.
#pragma once
#include <cfloat>
#include "pr_mixture.cuh"

namespace rb200 {
namespace walepr {

enum Status : int {
    SUCCESS = 0, SCOPE = 1, INPUT = 2, INVENTORY = 3, GAS_EOS = 4, PARTIAL_H = 5, LIQUID_EOS = 6,
    RECOVERED_STATE = 7, ENERGY = 8
};

RB200_HD inline bool fin(double x) { return x == x && fabs(x) <= DBL_MAX; }

// The gas mixture (Y) at (T, p) on its gas root, as the flash evaluates it.
RB200_HD inline bool gasAt(const ReactiveB200HemModel& m, double p, double T, const double* Y, mix::Props& out) {
    if (!(fin(p) && fin(T) && p >= m.pmin && p <= m.pmax && T >= m.Tmin && T <= m.Tmax)) return false;
    if (m.enforceSpeciesTemperatureBounds)
        for (int k = 0; k < m.ns; ++k)
            if (Y[k] > 0) {
                const ReactiveB200Species& sp = m.phase[0].species[k];
                if (T < sp.regions[0].minimumTemperature || T > sp.regions[sp.regionCount - 1].maximumTemperature)
                    return false;
            }
    return mix::tp(m.phase[0], T, p, Y, mix::GAS, false, out) == mix::OK;
}

// The pure liquid of condensed phase 0 at (T, p).
RB200_HD inline bool liquidAt(const ReactiveB200HemModel& m, double p, double T, mix::Props& out) {
    if (!(fin(p) && fin(T) && p >= m.pmin && p <= m.pmax && T >= m.Tmin && T <= m.Tmax)) return false;
    if (T < m.liquidTmin[0] || T >= m.liquidTc[0] * (1 - 1e-10)) return false;
    const double pure[mix::kMaxNs] = {1, 0, 0, 0};
    return mix::tp(m.phase[1], T, p, pure, mix::LIQUID, false, out) == mix::OK;
}

// total: the cell's species densities (required with enthalpies); effective
// receives ns enthalpies [J/kg], cp the state's heat capacity.
RB200_HD inline int properties(const ReactiveB200HemModel& m, const double* total, const ReactiveThermoState& s,
                               double color, double jump, double* effective, double& cp, bool enthalpies) {
    if (m.nl != 1 || m.condensedKind[0] != 0 || m.ns < 1 || m.ns > mix::kMaxNs) return SCOPE;
    if (!fin(s.cp) || s.cp <= 0) return RECOVERED_STATE;
    if (!enthalpies) {
        cp = s.cp;
        return SUCCESS;
    }
    if (!total || !effective || !fin(color) || color < 0 || color > 1 || !fin(jump) || !fin(s.p) || s.p <= 0
        || !fin(s.T) || s.T <= 0)
        return INPUT;
    const double pg = s.p - color * jump, pl = s.p + (1 - color) * jump;
    if (!fin(pg) || pg <= 0 || !fin(pl) || pl <= 0) return INPUT;
    const int cond = m.condensable[0];
    const double ml = s.liquidMass[0];
    if (!fin(ml) || ml < 0 || !fin(s.gasMass) || s.gasMass < 0) return INVENTORY;
    double gas[mix::kMaxNs] = {}, Y[mix::kMaxNs] = {}, hbar[mix::kMaxNs] = {};
    double rho = 0, other = 0;
    for (int k = 0; k < m.ns; ++k) {
        if (!fin(total[k]) || total[k] < 0) return INVENTORY;
        gas[k] = total[k];
        rho += total[k];
        if (k != cond) other += total[k];
    }
    if (!(rho > 0) || ml > total[cond]) return INVENTORY;
    gas[cond] -= ml;
    // the condensable's vapour two ways: the total less the liquid, and the gas
    // mass less the other species; they must agree to rounding, and the one
    // from the smaller operands is kept (a trace of vapour beside a liquid)
    const double fromGas = s.gasMass - other, fromLiquid = gas[cond];
    const double scale = fmax(fmax(fmax(1.0, fabs(total[cond])), fmax(fabs(ml), fabs(s.gasMass))), fabs(other));
    if (!fin(fromGas) || fabs(fromGas - fromLiquid) > 16 * DBL_EPSILON * scale) return INVENTORY;
    if (fromGas >= 0 && fromGas <= total[cond] && fabs(s.gasMass) + fabs(other) < fabs(total[cond]) + fabs(ml))
        gas[cond] = fromGas;
    double mg = 0;
    for (int k = 0; k < m.ns; ++k) {
        if (!fin(gas[k]) || gas[k] < 0) return INVENTORY;
        mg += gas[k];
    }
    const double tol = fmax(1e-8, 50 * m.vtol);
    if (!fin(rho) || !fin(mg) || !fin(s.rho) || fabs(s.rho - rho) > tol * fmax(1.0, rho)
        || fabs(s.gasMass - mg) > tol * fmax(1.0, rho))
        return RECOVERED_STATE;
    for (int k = 0; k < m.ns; ++k) Y[k] = mg > 0 ? gas[k] / mg : total[k] / rho;
    mix::Props g{}, l{};  // a cell without liquid carries 0 * l.h = 0
    if (!gasAt(m, pg, s.T, Y, g)) return GAS_EOS;
    if (mix::partialEnthalpies(m.phase[0], s.T, Y, g, hbar) != mix::OK) return PARTIAL_H;
    for (int k = 0; k < m.ns; ++k) {
        hbar[k] /= m.weights[k];
        if (!fin(hbar[k])) return PARTIAL_H;
    }
    if (ml > 0) {
        if (!liquidAt(m, pl, s.T, l)) return LIQUID_EOS;
        if (!fin(s.rhoLiquid[0]) || s.rhoLiquid[0] <= 0 || fabs(s.rhoLiquid[0] / l.rho - 1) > tol
            || !fin(s.alphaLiquid[0]) || fabs(s.alphaLiquid[0] - ml / l.rho) > tol)
            return RECOVERED_STATE;
    }
    if (mg > 0 && (!fin(s.rhoGas) || s.rhoGas <= 0 || fabs(s.rhoGas / g.rho - 1) > tol || !fin(s.alphaGas)
                   || fabs(s.alphaGas - mg / g.rho) > tol))
        return RECOVERED_STATE;
    const double volume = (mg > 0 ? mg / g.rho : 0) + (ml > 0 ? ml / l.rho : 0);
    if (!fin(volume) || fabs(volume - 1) > tol * fmax(1.0, volume)) return RECOVERED_STATE;
    double local[mix::kMaxNs] = {}, enthalpy = 0;
    for (int k = 0; k < m.ns; ++k) {
        const double carried = gas[k] * hbar[k] + (k == cond ? ml * l.h : 0);
        local[k] = total[k] > 0 ? carried / total[k] : hbar[k];
        if (!fin(local[k])) return PARTIAL_H;
        enthalpy += total[k] * local[k];
    }
    // the enthalpy density must equal rho e + the pressure work of both phases
    const double work = jump == 0 ? s.p : pg * s.alphaGas + pl * (s.alphaLiquid[0] + s.alphaLiquid[1]);
    const double expected = rho * s.e + work;
    if (!fin(s.e) || !fin(expected) || !fin(enthalpy)
        || fabs(enthalpy - expected) > tol * fmax(1.0, fmax(fabs(enthalpy), fabs(expected))))
        return ENERGY;
    for (int k = 0; k < m.ns; ++k) effective[k] = local[k];
    cp = s.cp;
    return SUCCESS;
}

}  // namespace walepr
}  // namespace rb200
