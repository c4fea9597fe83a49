"""CPU restatement of the RK stage driver (src/reactiveFoam/ReactiveFoam.C:961-1019,
chemistry off) over the reference's own CPU transport (oracle/_ref, backend 0,
host-array reactive_transport_stage) and the reference flash compiled for the
host: stage 0, recovery seeded by the step-start states, stage 1, recovery
again seeded by the step-start states. Test infrastructure only."""
import ctypes as C

import numpy as np

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A


def compact(states):
    tr = np.zeros(len(states), dtype=A.STATE_DTYPE)
    for k_out, k_in in (("p", "p"), ("T", "T"), ("rho", "rho"), ("cv", "cv"), ("sound", "soundFrozen"),
                        ("gasMass", "gasMass")):
        tr[k_out] = states[k_in]
    return tr


def internal_energy(q):
    return q[:, 4] - .5 * np.sum(q[:, 1:4] ** 2, axis=1) / q[:, 0]


class ReferenceFlow:
    def __init__(self, faces, volume, q0, guess0, fixed_q, fixed_guess, viscosity, conductivity, wale_cw, image,
                 wave_factor=1.1, threads=1, turbulent_prandtl=None, turbulent_schmidt=None):
        self.lib = oracle.ref_transport_lib()
        self.image = image
        self.threads = threads
        self.fixed_state, ok, _ = oracle.ref_flash_recover(image, fixed_q[:, 0], internal_energy(fixed_q), fixed_guess)
        assert ok.all()
        self.states, ok, _ = oracle.ref_flash_recover(image, q0[:, 0], internal_energy(q0), guess0, threads)
        assert ok.all()
        self.q = np.ascontiguousarray(q0.copy())
        self.faces = np.ascontiguousarray(faces)
        self.volume = np.ascontiguousarray(volume, dtype=np.float64)
        fixed_tr = compact(self.fixed_state)
        self.fixed_q = np.ascontiguousarray(fixed_q, dtype=np.float64)
        cfg = A.Config(len(volume), 1, 5, len(faces), len(fixed_q), viscosity, conductivity, 0.0, wave_factor,
                       1e11, 0)
        d = C.POINTER(C.c_double)
        self.lib.reactive_transport_create.restype = C.c_void_p
        self.lib.reactive_transport_stage.argtypes = [C.c_void_p, d, C.c_void_p, d, d, C.c_double, C.c_int, d]
        self.lib.reactive_transport_error.restype = C.c_char_p
        self.lib.reactive_transport_error.argtypes = [C.c_void_p]
        err = C.create_string_buffer(2048)
        h = self.lib.reactive_transport_create(
            0, C.byref(cfg), self.volume.ctypes.data_as(d), self.faces.ctypes.data_as(C.c_void_p),
            self.fixed_q.ctypes.data_as(d), fixed_tr.ctypes.data_as(C.c_void_p), None, None, err, len(err))
        assert h, err.value
        self.h = C.c_void_p(h)
        if wale_cw is not None:
            opts = A.WaleOptions(1, C.sizeof(A.WaleOptions), wale_cw)
            assert self.lib.reactive_transport_set_wale_v1(self.h, C.byref(opts)) == 0
        self.scalars = turbulent_prandtl is not None or turbulent_schmidt is not None
        if self.scalars:
            # the WALE scalar closure, fed each stage with that stage's mixture
            # cp through the host field upload (one species: the enthalpies
            # carry no flux, zeros stand in for them)
            opts = A.WaleScalarOptions(1, C.sizeof(A.WaleScalarOptions), turbulent_prandtl or 0.0,
                                       turbulent_schmidt or 0.0)
            assert self.lib.reactive_transport_set_wale_scalars_v1(self.h, C.byref(opts)) == 0, \
                self.lib.reactive_transport_error(self.h)
            self.lib.reactive_transport_wale_scalar_fields_v1.argtypes = [C.c_void_p, d, d, d, d]
            self.zero_h = np.zeros(len(volume) + len(fixed_q))
        self.boundary = np.zeros(5)

    def _stage(self, states, dt, stage):
        if self.scalars:
            d = C.POINTER(C.c_double)
            cp = np.ascontiguousarray(states["cp"])
            fixed_cp = np.ascontiguousarray(self.fixed_state["cp"])
            rc = self.lib.reactive_transport_wale_scalar_fields_v1(
                self.h, cp.ctypes.data_as(d), self.zero_h.ctypes.data_as(d), fixed_cp.ctypes.data_as(d),
                self.zero_h.ctypes.data_as(d))
            assert rc == 0, self.lib.reactive_transport_error(self.h)
        tr = compact(states)
        br = np.zeros(5)
        rc = self.lib.reactive_transport_stage(self.h, self.q.ctypes.data_as(C.POINTER(C.c_double)),
                                               tr.ctypes.data_as(C.c_void_p), None, None, dt, stage,
                                               br.ctypes.data_as(C.POINTER(C.c_double)))
        assert rc == 0, self.lib.reactive_transport_error(self.h)
        return br

    def step(self, dt):
        start = self.states.copy()
        b0 = self._stage(start, dt, 0)
        s1, ok, _ = oracle.ref_flash_recover(self.image, self.q[:, 0].copy(), internal_energy(self.q), start,
                                             self.threads)
        assert ok.all()
        b1 = self._stage(s1, dt, 1)
        s2, ok, _ = oracle.ref_flash_recover(self.image, self.q[:, 0].copy(), internal_energy(self.q), start,
                                             self.threads)
        assert ok.all()
        self.states = s2
        self.boundary = .5 * dt * (b0 + b1)

    def close(self):
        self.lib.reactive_transport_destroy(self.h)
