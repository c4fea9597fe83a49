"""The capillary UV closure of the reference solver
(src/reactiveFoam/reactiveCapillary.H:6-246) on this library: the outer
iteration between the capillary HEM flash (the gas at p - c J, the liquid at
p + (1 - c) J, J = sigma * curvature) and the diffuse interface geometry of the
transported color, until the color, the surface energy and the jump stop
changing. Two paths, as the reference has them:

* `recover_host`: host arrays through reactive_gpu_hem_run_v2 and
  reactive_transport_capillary_geometry_v1 (the reference's host path);
* `recover_resident`: the resident entries reactive_transport_capillary_resident_*
  with reactive_gpu_hem_run_resident_v1 on their device view; returns False
  (nothing changed) when the host path must run instead.

Each cell is re-flashed only while its color, jump or surface energy changes
bitwise; the relaxation halves the color update when the residual stalls.
"""
import ctypes as C

import numpy as np

from . import _abi as A, _lib

MAX_ITERATIONS = 40
TOLERANCE = 1e-9


class CapillaryError(RuntimeError):
    pass


def internal_energy(q, ns):
    """Bulk internal energy density of cell-major q: total energy less the
    kinetic energy (surface energy not removed)."""
    rho = q[:, :ns].sum(axis=1)
    m = q[:, ns:ns + 3]
    return q[:, ns + 3] - .5 * (m[:, 0] * m[:, 0] + m[:, 1] * m[:, 1] + m[:, 2] * m[:, 2]) / rho


def liquid_color(states):
    """Liquid volume fraction V_l / (V_l + V_g) of each recovered state
    (reactiveCapillary.H:6-29); raises for a state whose phase volumes do not close."""
    ml = states["liquidMass"][:, 0]
    if not (np.isfinite(ml).all() and (ml >= 0).all()):
        raise CapillaryError("Invalid capillary liquid inventory")
    rl = states["rhoLiquid"][:, 0]
    if not (np.isfinite(rl[ml > 0]).all() and (rl[ml > 0] > 0).all()):
        raise CapillaryError("Missing capillary liquid density")
    color = np.zeros(len(states))
    with np.errstate(divide="ignore", invalid="ignore"):
        color[ml > 0] = ml[ml > 0] / rl[ml > 0]
        mg = states["gasMass"]
        gas = np.where(mg > 0, mg / np.where(mg > 0, states["rhoGas"], 1.0), 0.0)
        total = color + gas
        if not (np.isfinite(total).all() and (total > 0).all() and (np.abs(total - 1) < 1e-6).all()):
            raise CapillaryError("Capillary phase volumes do not close")
        color = color / total
    if not (np.isfinite(color).all() and (color >= 0).all() and (color <= 1).all()):
        raise CapillaryError("Liquid material volume outside [0,1]")
    return color


class CapillaryClosure:
    """One transport handle with the capillary model installed and one HEM handle
    (`hem`, a GpuHem) whose model has the liquid of the transport's capillary
    species. ns: transport species; nv = ns + 5 (the liquid inventory at ns + 4)."""

    def __init__(self, transport, hem, ns, sigma, fixed_color=None, frozen=False):
        self.lib = _lib.load()
        self.t = transport
        self.hem = hem
        self.ns = ns
        self.sigma = float(sigma)
        self.fixed_color = None if fixed_color is None else np.ascontiguousarray(fixed_color, dtype=np.float64)
        self.frozen = bool(frozen)
        self.iterations = 0
        self.residual = None
        self.color = self.surface_energy = self.curvature = self.jump = None

    def _error(self):
        return self.lib.reactive_transport_error(self.t).decode()

    def geometry(self, color):
        n = len(color)
        energy, curvature = np.zeros(n), np.zeros(n)
        rc = self.lib.reactive_transport_capillary_geometry_v1(
            self.t, A.dptr(np.ascontiguousarray(color)), A.dptr(self.fixed_color), A.dptr(energy),
            A.dptr(curvature), None)
        if rc:
            raise CapillaryError(self._error())
        self.color, self.surface_energy, self.curvature = np.ascontiguousarray(color).copy(), energy, curvature
        self.jump = self.sigma * curvature
        return energy, curvature

    def recover_host(self, q, states):
        """The host closure on cell-major q (updated: the liquid inventory column
        becomes the recovered liquid mass in equilibrium) and states (seeds in,
        the converged states out)."""
        ns, n = self.ns, len(q)
        self.geometry(liquid_color(states))
        seeds = states.copy()
        seeds["liquidMass"][:, 0] = q[:, ns + 4]
        flashed = np.zeros((3, n))
        bulk = internal_energy(q, ns)
        previous = np.inf
        for iteration in range(MAX_ITERATIONS):
            self.iterations += 1
            before = np.stack([self.color, self.jump, self.surface_energy])
            dirty = np.arange(n) if iteration == 0 else np.flatnonzero(
                (before.view(np.int64) != flashed.view(np.int64)).any(axis=0))
            if len(dirty):
                cap = np.zeros(len(dirty), dtype=A.CAPILLARY_DTYPE)
                cap["color"], cap["pressureJump"] = before[0, dirty], before[1, dirty]
                cap["equilibrium"] = 0 if self.frozen else 1
                batch = np.ascontiguousarray(seeds[dirty])
                ok, prof = self.hem.run_capillary(np.ascontiguousarray(q[dirty, :ns]), bulk[dirty] - before[2, dirty],
                                                  cap, batch)
                if prof.deviceFailures:
                    raise CapillaryError(f"Capillary HEM batch: {int(prof.deviceFailures)} cells failed")
                states[dirty] = batch
                flashed[:, dirty] = before[:, dirty]
            candidate = liquid_color(states)
            self.geometry(candidate)
            scale = np.maximum(np.abs(bulk), states["rho"] * 1e5)
            residual = max(np.max(np.abs(candidate - before[0])),
                           np.max(np.abs(self.surface_energy - before[2]) / scale),
                           np.max(np.abs(self.jump - before[1]) / np.maximum(states["p"], 1.0)))
            self.residual = residual
            if residual <= TOLERANCE:
                if not self.frozen:
                    q[:, ns + 4] = states["liquidMass"][:, 0]
                return
            if iteration > 0 and residual > previous * .9:
                self.geometry(.5 * (before[0] + candidate))
            previous = residual
        raise CapillaryError(f"Surface-energy / curved UV closure did not converge (residual {self.residual})")

    def recover_resident(self, q, states):
        """The resident closure; returns False, with q and states unchanged, when
        the host path must run instead (an input it would reject, a failed
        device cell, no convergence)."""
        L, ns, n = self.lib, self.ns, len(q)
        fallback = C.c_int()
        qs = np.ascontiguousarray(q[:, :ns])
        liquid = np.ascontiguousarray(q[:, ns + 4])
        bulk = np.ascontiguousarray(internal_energy(q, ns))
        seed = np.ascontiguousarray(states)
        rc = L.reactive_transport_capillary_resident_begin_v1(
            self.t, ns, A.dptr(qs), A.dptr(liquid), A.dptr(bulk), seed.ctypes.data_as(C.c_void_p),
            A.dptr(self.fixed_color), self.sigma, 0 if self.frozen else 1, C.byref(fallback))
        if rc:
            raise CapillaryError(self._error())
        if fallback.value:
            return False
        previous = np.inf
        for iteration in range(MAX_ITERATIONS):
            view = A.CapillaryResidentView(1, C.sizeof(A.CapillaryResidentView))
            if L.reactive_transport_capillary_resident_select_v1(self.t, iteration, C.byref(view), C.byref(fallback)):
                raise CapillaryError(self._error())
            if fallback.value:
                return False
            self.iterations += 1
            if view.count:
                for first in range(0, view.count, self.hem.capacity):
                    part = min(self.hem.capacity, view.count - first)
                    prof = self.hem.run_resident(view.q, view.energy, view.seed, view.capillary,
                                                 view.order + 4 * first, part, view.output)
                    if prof.deviceFailures:
                        return False
            residual = C.c_double()
            if L.reactive_transport_capillary_resident_update_v1(self.t, view.count, C.byref(residual),
                                                                 C.byref(fallback)):
                raise CapillaryError(self._error())
            if fallback.value:
                return False
            self.residual = residual.value
            if residual.value <= TOLERANCE:
                out = np.zeros(n, dtype=A.THERMO_DTYPE)
                color, energy, curvature = np.zeros(n), np.zeros(n), np.zeros(n)
                if L.reactive_transport_capillary_resident_commit_v1(self.t, out.ctypes.data_as(C.c_void_p),
                                                                     A.dptr(color), A.dptr(energy),
                                                                     A.dptr(curvature)):
                    raise CapillaryError(self._error())
                states[:] = out
                self.color, self.surface_energy, self.curvature = color, energy, curvature
                self.jump = self.sigma * curvature
                if not self.frozen:
                    q[:, ns + 4] = states["liquidMass"][:, 0]
                return True
            if iteration > 0 and residual.value > previous * .9:
                if L.reactive_transport_capillary_resident_relax_v1(self.t):
                    raise CapillaryError(self._error())
            previous = residual.value
        return False
