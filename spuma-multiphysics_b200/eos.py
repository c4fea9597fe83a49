"""Vectorised host-side Peng-Robinson relations for one species (numpy, FP64).

Used only to construct case inputs on the host (initial (rho, e) fields, the
liquid inlet state, saturated two-phase batches); every recovery during a run is
done by the CUDA HEM flash. The relations are the same Peng-Robinson / NASA9
forms the device evaluates (alpha(T) with kappa(omega), the cubic in V, residual
enthalpy/entropy and the molar chemical potential).
"""
import math

import numpy as np

from .thermo_data import GAS_CONSTANT as R, OMEGA_A, OMEGA_B, ONE_ATM, kappa

SQRT2 = math.sqrt(2.0)


class PureFluid:
    def __init__(self, sp):
        self.sp = sp
        self.a, self.b, self.W = sp["a"], sp["b"], sp["W"]
        self.kappa = kappa(sp["omega"])
        self.Tc = self.a * OMEGA_B / (self.b * OMEGA_A * R)
        self.pc = OMEGA_B * R * self.Tc / self.b
        self.ranges = np.array(sp["ranges"])
        self.coeffs = np.array(sp["nasa9"])

    def _alpha(self, T):
        sq = np.sqrt(T / self.Tc)
        f = 1.0 + self.kappa * (1.0 - sq)
        s = np.sign(f)
        q = np.abs(f)
        dq = -s * self.kappa / (2.0 * self.Tc * sq)
        d2q = s * self.kappa / (4.0 * self.Tc ** 2 * sq ** 3)
        return self.a * q * q, self.a * 2 * q * dq, self.a * (2 * q * d2q + 2 * dq * dq)

    def _nasa(self, T):
        idx = np.clip(np.searchsorted(self.ranges[1:-1], T, side="right"), 0, len(self.coeffs) - 1)
        a = self.coeffs[idx].T
        iT, lT = 1.0 / T, np.log(T)
        c0, c1, c2, c3, c4, c5, c6 = a[0] * iT * iT, a[1] * iT, a[2], a[3] * T, a[4] * T * T, a[5] * T ** 3, a[6] * T ** 4
        cp = c0 + c1 + c2 + c3 + c4 + c5 + c6
        h = -c0 + lT * c1 + c2 + .5 * c3 + c4 / 3 + .25 * c5 + .2 * c6 + a[7] * iT
        s = -.5 * c0 - c1 + lT * c2 + c3 + .5 * c4 + c5 / 3 + .25 * c6 + a[8]
        return cp, h, s

    def trho(self, T, rho):
        """Properties at (T, rho): dict of p, e, h, s (per kg), cp, cv, sound, mu (J/kmol)."""
        T = np.asarray(T, dtype=float)
        rho = np.asarray(rho, dtype=float)
        b, W = self.b, self.W
        aa, da, d2a = self._alpha(T)
        V = W / rho
        den = V * V + 2 * V * b - b * b
        vmb = V - b
        p = R * T / vmb - aa / den
        dpdV = -R * T / vmb ** 2 + 2 * aa * (V + b) / den ** 2
        dpdT = R / vmb - da / den
        logr = np.log((V + (1 + SQRT2) * b) / (V + (1 - SQRT2) * b))
        L = logr / (2 * SQRT2 * b)
        cpR, hRT, sR = self._nasa(T)
        z = p * V / (R * T)
        hM = R * T * hRT + (R * T * (z - 1) + L * (T * da - aa))
        sM = (R * sR - R * np.log(p / ONE_ATM)) + (R * np.log(z * (1 - b / V)) + L * da)
        cpM = (R * cpR + V * dpdT - R + L * T * d2a) - (V + T * dpdT / dpdV) * dpdT
        cvM = cpM + T * dpdT ** 2 / dpdV
        RT = R * T
        mu = (RT * (hRT - sR) + RT * np.log(p / ONE_ATM) - RT * np.log(p * V / RT) + RT * np.log(V / vmb)
              + RT * b / vmb - (2 * b * aa - aa * b) / (2 * SQRT2 * b * b) * logr - aa * V / den)
        sound = np.sqrt(V * V * (-cpM / cvM * dpdV / W))
        return dict(p=p, e=(hM - p * V) / W, h=hM / W, s=sM / W, cp=cpM / W, cv=cvM / W, sound=sound, mu=mu,
                    V=V, dpdV=dpdV)

    def roots(self, T, p):
        """Physical molar-volume roots (smallest, largest) of the cubic at (T, p)."""
        T = np.asarray(T, dtype=float)
        p = np.asarray(p, dtype=float)
        b = self.b
        aa, _, _ = self._alpha(T)
        RTp, aap = R * T / p, aa / p
        bn = b - RTp
        cn = -(2 * RTp * b - aap + 3 * b * b)
        dn = b * b * RTp + b ** 3 - aap * b
        center = -bn / 3
        delta2 = (bn * bn - 3 * cn) / 9
        q = 2 * bn ** 3 / 27 - bn * cn / 3 + dn
        delta = np.sqrt(np.maximum(delta2, 0))
        disc = q * q - (2 * delta * delta2) ** 2
        sd = .5 * np.sqrt(np.maximum(disc, 0))
        one = center + np.cbrt(-.5 * q + sd) + np.cbrt(-.5 * q - sd)
        with np.errstate(invalid="ignore", divide="ignore"):
            theta = np.arccos(np.clip(-.5 * q / np.where(delta > 0, delta ** 3, 1), -1, 1)) / 3
        three = np.stack([center + 2 * delta * np.cos(theta + k * 2 * np.pi / 3) for k in range(3)])
        multi = (disc < 0) & (delta2 > 0)
        cand = np.where(multi[None], three, np.stack([one, one, one]))
        for _ in range(12):
            f = ((cand + bn) * cand + cn) * cand + dn
            d = (3 * cand + 2 * bn) * cand + cn
            cand = cand - np.where(np.abs(d) > 1e-300, f / np.where(d == 0, 1, d), 0)
        valid = np.isfinite(cand) & (cand > b)
        out_lo = np.where(valid, cand, np.inf).min(axis=0)
        out_hi = np.where(valid, cand, -np.inf).max(axis=0)
        out_lo = np.where(np.isfinite(out_lo), out_lo, np.nan)
        out_hi = np.where(np.isfinite(out_hi), out_hi, np.nan)
        return out_lo, out_hi

    def tp(self, T, p, root="gas"):
        lo, hi = self.roots(T, p)
        V = hi if root in ("gas", "auto") else lo
        props = self.trho(T, self.W / V)
        props["rho"] = self.W / V
        return props

    def saturation(self, T, iterations=200):
        """(p_sat, gas props, liquid props) by bisection on mu_gas - mu_liquid."""
        T = np.atleast_1d(np.asarray(T, dtype=float))
        lo = np.full_like(T, 1e2)
        hi = np.full_like(T, self.pc * 0.9999)
        for _ in range(iterations):
            mid = np.sqrt(lo * hi)
            vlo, vhi = self.roots(T, mid)
            two = np.isfinite(vlo) & (vhi > vlo * (1 + 1e-9))
            g = self.trho(T, self.W / vhi)["mu"]
            l = self.trho(T, self.W / vlo)["mu"]
            # gas chemical potential above liquid: pressure too high
            too_high = (~two & (vhi < 3 * self.b)) | (two & (g > l))
            hi = np.where(too_high, mid, hi)
            lo = np.where(too_high, lo, mid)
        p = np.sqrt(lo * hi)
        vlo, vhi = self.roots(T, p)
        gas = self.trho(T, self.W / vhi)
        gas["rho"] = self.W / vhi
        liq = self.trho(T, self.W / vlo)
        liq["rho"] = self.W / vlo
        return p, gas, liq
