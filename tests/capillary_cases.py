"""Capillary closure cases and the comparison walk shared by the GPU parity
tests: this library (backend 1) against the reference's own CPU build
(oracle/_ref/libreactiveTransport_ref.so, backend 0) on the same inputs.

Cases restate the reference's capillary transport test
(tools/capillary_transport_test.cpp:31-103: a periodic 32-cell tanh interface,
two species, one liquid inventory, sigma 0.072, capillary CFL 0.5, geometry
threshold 1e-10, with WALE and WALE scalars installed) and widen it to the face
graphs of the transport validation cases (all four boundary kinds, oblique
normals, irregular incidence, extra boundary faces, up to 53 species) with a
smooth color field plus noise, its liquid inventory a share of the condensable
species' density.
"""
import ctypes as C

import numpy as np

from spuma_multiphysics_b200 import _abi as A
import transport_cases as T

GEOMETRY_TOL = 1e-12   # relative, surface energy / curvature / normal
SIGMA = .072
MODEL_HASH = b"a" * 64


def bind(lib):
    d, v = C.POINTER(C.c_double), C.c_void_p
    T.bind(lib)
    sig = {"set_capillary_v1": ([v, C.POINTER(A.CapillaryOptions)], C.c_int),
           "capillary_geometry_v1": ([v, d, d, d, d, d], C.c_int),
           "capillary_profile_v1": ([v, C.POINTER(A.CapillaryProfile)], C.c_int),
           "begin_attempt": ([v, C.c_char_p, C.c_uint64], C.c_int),
           "end_attempt": ([v, C.c_uint64, C.c_int], C.c_int),
           "advance_resident_v2": ([v, A.Token, A.Token, C.POINTER(A.State), v, d, d, C.c_double, d], C.c_int),
           "download_conserved": ([v, A.Token, d], C.c_int),
           "replace_stage_state_v1": ([v, A.Token, C.c_uint64, d], C.c_int),
           "create_v2": ([C.c_int, C.POINTER(A.Config), C.POINTER(A.OptionsV2), d, C.POINTER(A.Face), d,
                          C.POINTER(A.State), d, d, C.c_char_p, C.c_size_t], v)}
    for name, (args, ret) in sig.items():
        fn = getattr(lib, "reactive_transport_" + name)
        fn.argtypes, fn.restype = args, ret
    return lib


def options(sigma=SIGMA, cfl=.5, eps=1e-10, species=0):
    return A.CapillaryOptions(1, C.sizeof(A.CapillaryOptions), sigma, cfl, eps, species)


def graph_case(ns, nc, kind, transport=True, spatial=True, extra_boundary=0, species=0, seed=0, noise=.05):
    """A transport validation face graph with a liquid inventory (variables =
    species + 5) and a material color: a tanh front across the cell index plus
    seeded noise, clipped to [0, 1], pure cells at both ends."""
    case = T.make_case(ns, nc, kind, transport=transport, spatial=spatial, extra_boundary=extra_boundary,
                       frozen=1, seed=seed)
    rng = np.random.default_rng(4400 + nc + 31 * ns + 7 * kind + seed)
    x = (np.arange(nc) + .5) / nc
    color = .5 * (1 - np.tanh((x - .5) / .12)) + noise * rng.uniform(-1, 1, nc)
    color = np.clip(color, 0, 1)
    if nc > 4:
        color[0], color[-1] = 1.0, 0.0
    q = case["q"]
    q[:, ns + 4] = q[:, species] * color * rng.uniform(.2, .95, nc)
    fixed = case["config"].fixed
    case["color"] = color
    case["fixed_color"] = np.full(max(fixed, 1), .25)[:fixed] if fixed else None
    if fixed:
        case["fixed_q"][:, ns + 4] = case["fixed_q"][:, species] * .25
    case["species"] = species
    case["name"] += f"-cap{species}"
    return case


def periodic_interface(n=32, ns=2):
    """The reference's periodic tanh interface (capillary_transport_test.cpp:33-79):
    unit-area faces along x, h = 1/n, color 0.5 (1 - tanh((x - 0.5) / 1.5h)),
    density 1000 c + 1.2 (1 - c), p 101325, T 300, cv 1000, sound 340."""
    nv = ns + 5
    h = 1.0 / n
    faces = (A.Face * n)()
    for i in range(n):
        faces[i] = A.Face(i, (i + 1) % n, -1, (C.c_double * 3)(1, 0, 0), 1.0, h, .5, 0)
    x = (np.arange(n) + .5) * h
    color = .5 * (1 - np.tanh((x - .5) / (1.5 * h)))
    density = 1000 * color + 1.2 * (1 - color)
    states = np.zeros(n, dtype=A.STATE_DTYPE)
    states["p"], states["T"], states["rho"], states["cv"], states["sound"] = 101325, 300, density, 1000, 340
    q = np.zeros((n, nv))
    q[:, 0] = 1000 * color
    q[:, 1] = 1.2 * (1 - color)
    q[:, ns + 3] = 250000   # the surface energy is added once the geometry is known
    q[:, ns + 4] = 1000 * color
    cfg = A.Config(n, ns, nv, n, 0, 0.0, 0.0, 0.0, 1.0, 64e6, 0)
    fixed_states = np.zeros(1, dtype=A.STATE_DTYPE)
    return dict(config=cfg, faces=faces, volume=np.full(n, h), q=q, states=states, y=None, h=None,
                fixed_q=np.zeros((1, nv)), fixed_states=fixed_states,
                fixed_states_ptr=C.cast(T.states_ptr(fixed_states), C.c_void_p), fixed_y=np.zeros((1, ns)),
                fixed_h=np.zeros((1, ns)), ns=ns, nc=n, nv=nv, mechanical=False, color=color, fixed_color=None,
                species=0, name=f"periodic{n}")


class Handle:
    """One transport handle with the capillary closure installed."""

    def __init__(self, lib, backend, case, wale_cw=None, wale_scalars=None, opts=None):
        self.lib, self.case = lib, case
        error = C.create_string_buffer(4096)
        o2 = A.OptionsV2(1, C.sizeof(A.OptionsV2), 8, 0, MODEL_HASH)
        handle = lib.reactive_transport_create_v2(
            backend, C.byref(case["config"]), C.byref(o2), T.dp(case["volume"]), case["faces"],
            T.dp(case["fixed_q"]), T.states_ptr(case["fixed_states"]), T.dp(case["fixed_y"]), T.dp(case["fixed_h"]),
            error, len(error))
        if not handle:
            raise RuntimeError(error.value.decode())
        self.h = C.c_void_p(handle)
        self.check(lib.reactive_transport_set_capillary_v1(self.h, C.byref(opts or options(species=case["species"]))))
        if wale_cw is not None:
            self.check(lib.reactive_transport_set_wale_v1(self.h, C.byref(A.WaleOptions(1, C.sizeof(A.WaleOptions),
                                                                                         wale_cw))))
        if wale_scalars is not None:
            o = A.WaleScalarOptions(1, C.sizeof(A.WaleScalarOptions), *wale_scalars)
            self.check(lib.reactive_transport_set_wale_scalars_v1(self.h, C.byref(o)))

    def check(self, status):
        if status:
            raise RuntimeError(self.lib.reactive_transport_error(self.h).decode())

    def error(self):
        return self.lib.reactive_transport_error(self.h).decode()

    def geometry(self, color=None, fixed_color=None, curvature=True, normal=True):
        nc = self.case["nc"]
        color = self.case["color"] if color is None else color
        fixed_color = self.case["fixed_color"] if fixed_color is None else fixed_color
        energy = np.zeros(nc)
        kappa = np.zeros(nc) if curvature else None
        nrm = np.zeros((nc, 3)) if normal else None
        self.check(self.lib.reactive_transport_capillary_geometry_v1(
            self.h, T.dp(np.ascontiguousarray(color)), T.dp(fixed_color), T.dp(energy), T.dp(kappa), T.dp(nrm)))
        return energy, kappa, nrm

    def rhs(self, q, states, y=None, h=None):
        rhs, br = np.empty_like(q), np.empty(q.shape[1])
        self.check(self.lib.reactive_transport_rhs(self.h, T.dp(q), T.states_ptr(states), T.dp(y), T.dp(h),
                                                   T.dp(rhs), T.dp(br)))
        return rhs, br

    def stable_step(self, q, states, cfl=.23, maximum=.1):
        dt = C.c_double()
        self.check(self.lib.reactive_transport_stable_step(self.h, T.dp(q), T.states_ptr(states), cfl, maximum,
                                                           C.byref(dt)))
        return dt.value

    def stage(self, q, states, dt, stage, y=None, h=None):
        br = np.empty(q.shape[1])
        self.check(self.lib.reactive_transport_stage(self.h, T.dp(q), T.states_ptr(states), T.dp(y), T.dp(h), dt,
                                                     stage, T.dp(br)))
        return br

    def profile(self):
        p = A.CapillaryProfile(1, C.sizeof(A.CapillaryProfile))
        self.check(self.lib.reactive_transport_capillary_profile_v1(self.h, C.byref(p)))
        return {n: getattr(p, n) for n, _ in A.CapillaryProfile._fields_[2:]}

    def close(self):
        self.lib.reactive_transport_destroy(self.h)


def relative(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(1e-300, np.maximum(np.abs(b), np.max(np.abs(b)) * 1e-3)),
                        initial=0))


def drop_case(n=10, temperature=270.0, pressure=5e6, radius=.3, vapour=.6):
    """A liquid N2O drop in air and N2O vapour on an n^3 box of the production
    model's four species (N2, O2, N2O, isopropanol; nv = 9, the liquid inventory
    at 8): color 0.5 (1 - tanh((r - R) / 1.5h)) with R = radius * edge; each cell
    mixes, by that volume fraction, compressed liquid N2O and the gas (air with N2O
    mass fraction `vapour`), both at (temperature, pressure), from the reference's
    mixture evaluator; the states are their flash (the production model,
    finite-difference Jacobian), the liquid inventory their liquid mass. Returns
    the case dict, the model image and the states."""
    from oracle import oracle
    from spuma_multiphysics_b200 import cases, thermo_data as td
    from spuma_multiphysics_b200.hem import GpuHem
    ns, nv = 4, 9
    image = td.model_bytes(td.production_model(analytic_jacobian=0))
    lib = oracle.ref_flash_lib()

    def props(Y, choice):
        out = (C.c_double * (15 + ns))()
        phase = C.c_int()
        st = lib.ref_pr_mix_tp(image, 0, C.c_double(temperature), C.c_double(pressure), (C.c_double * ns)(*Y),
                               choice, 0, out,
                               C.byref(phase))
        assert st == 0
        return out[4], out[5]   # rho, e

    rho_l, e_l = props([0, 0, 1, 0], 2)
    y_gas = np.array([.767 * (1 - vapour), .233 * (1 - vapour), vapour, 0.0])
    rho_g, e_g = props(y_gas, 1)
    faces, volume = cases.box_faces((n, n, n), .08 / n)
    h = .08 / n
    x = (np.arange(n) + .5) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt((X - .04) ** 2 + (Y - .04) ** 2 + (Z - .04) ** 2).transpose(2, 1, 0).ravel()  # x fastest
    color = .5 * (1 - np.tanh((r - radius * .08) / (1.5 * h)))
    nc = n ** 3
    q = np.zeros((nc, nv))
    q[:, :ns] = (color * rho_l)[:, None] * np.array([0, 0, 1.0, 0]) + ((1 - color) * rho_g)[:, None] * y_gas
    energy = color * rho_l * e_l + (1 - color) * rho_g * e_g
    q[:, ns + 3] = energy
    guess = np.zeros(nc, dtype=A.THERMO_DTYPE)
    guess["p"], guess["T"], guess["rho"] = pressure, temperature, q[:, :ns].sum(axis=1)
    guess["liquidMass"][:, 0] = color * rho_l
    hem = GpuHem(model=image, capacity=nc)
    try:
        states = guess.copy()
        ok, _ = hem.run(np.ascontiguousarray(q[:, :ns]), energy, states)
    finally:
        hem.close()
    assert ok.all(), int((ok == 0).sum())
    q[:, ns + 4] = states["liquidMass"][:, 0]
    fa = (A.Face * len(faces)).from_buffer_copy(np.ascontiguousarray(faces).tobytes())
    cfg = A.Config(nc, ns, nv, len(faces), 0, 0.0, 0.0, 0.0, 1.1, 4e9, 0)
    fixed_states = np.zeros(1, dtype=A.STATE_DTYPE)
    case = dict(config=cfg, faces=fa, volume=np.ascontiguousarray(volume), q=q, states=None, y=None, h=None,
                fixed_q=np.zeros((1, nv)), fixed_states=fixed_states,
                fixed_states_ptr=C.cast(T.states_ptr(fixed_states), C.c_void_p), fixed_y=np.zeros((1, ns)),
                fixed_h=np.zeros((1, ns)), ns=ns, nc=nc, nv=nv, mechanical=False, color=color, fixed_color=None,
                species=2, name=f"drop{n}")
    return case, image, states

