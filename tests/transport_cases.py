"""Transport parity cases and the ABI contract walk, shared by the CPU tests
(oracle vs the reference's own CPU build) and the GPU tests (this library vs
the oracle and the reference).

The case list restates the configurations of the reference's operator
validation (tools/validate_reactive_transport.py:149-324): species 1-413, cells
1-65,537, all four boundary kinds, periodic closure, oblique normals with
irregular incidence, extra boundary faces, the mechanical two-environment
variables and one or two frozen liquid inventories, plus WALE cases. Inputs are
generated here from recorded seeds with an ideal-gas closure (gamma 1.4, R 287)
for the recovered states, as the reference harness does.
"""
import ctypes as C

import numpy as np

from spuma_multiphysics_b200 import _abi as A

RHS_TOL = 3e-12      # scaled operator error (validate_reactive_transport.py:191-195)
DT_TOL = 3e-14       # relative CFL step (:204)
BALANCE_TOL = 2e-11  # conservation (:206-208)


def ideal_states(q, ns, mechanical=False):
    """Ideal-gas (gamma=1.4, R=287) recovered states, Y and species enthalpies."""
    rho = q[:, :ns].sum(axis=1)
    p = .4 * (q[:, ns + 3] - .5 * np.sum(q[:, ns:ns + 3] ** 2, axis=1) / rho)
    T = p / rho / 287
    arr = np.zeros(len(q), dtype=A.STATE_DTYPE)
    arr["p"], arr["T"], arr["rho"], arr["cv"] = p, T, rho, 287 / .4
    arr["sound"], arr["gasMass"] = np.sqrt(1.4 * p / rho), rho
    arr["dilatation"] = .03 if mechanical else 0.0
    y = np.ascontiguousarray(q[:, :ns] / rho[:, None])
    h = np.ascontiguousarray(T[:, None] * 1004.5 + np.arange(ns)[None, :] * 17423.0)
    return arr, y, h


def states_ptr(arr):
    return arr.ctypes.data_as(C.POINTER(A.State))


def make_case(ns, nc, kind, transport=False, mechanical=False, spatial=False, extra_boundary=0, frozen=0,
              seed=0, viscous_only=False, conduction=False):
    rng = np.random.default_rng(9100 + 17 * ns + nc + 131 * kind + 7 * frozen + int(spatial) + seed)
    nv = ns + 4 + 2 * int(mechanical) + frozen
    q = np.zeros((nc, nv))
    q[:, :ns] = rng.uniform(.002, 1, (nc, ns))
    q[:, :ns] /= q[:, :ns].sum(axis=1)[:, None]
    q[:, :ns] *= rng.uniform(.75, 1.35, (nc, 1))
    rho = q[:, :ns].sum(axis=1)
    vel = rng.normal(0, 11, (nc, 3))
    q[:, ns:ns + 3] = rho[:, None] * vel
    q[:, ns + 3] = rng.uniform(7.5e4, 1.25e5, nc) / .4 + .5 * rho * np.sum(vel ** 2, axis=1)
    if mechanical:
        q[:, ns + 4] = rng.uniform(.1, .9, nc)
        q[:, ns + 5] = 1 - q[:, ns + 4]
    for i in range(frozen):
        q[:, ns + 4 + i] = q[:, i] * rng.uniform(.1, .9, nc)
    volume = rng.uniform(.1, .3, nc)
    faces = [(i, i + 1, -1, (1., 0., 0.), 1.0, .2, .41, 0) for i in range(nc - 1)]
    fixed_q = np.ascontiguousarray(q[:1] * 1.013)
    n_fixed = 0
    if kind == 0:
        faces.append((nc - 1, 0, -1, (1., 0., 0.), 1.0, .2, .59, 0))
    else:
        weight = {1: .5, 2: 1.0, 3: 0.0}[kind]
        for c, normal in ((0, -1.0), (nc - 1, 1.0)):
            faces.append((c, -1, 0 if kind == 3 else -1, (normal, 0., 0.), 1.0, .1, weight, kind))
        n_fixed = int(kind == 3)
    if spatial:
        faces += [(i, i + 2, -1, (1., 0., 0.), .33, .29, .57, 0) for i in range(max(0, nc - 2))]
        out = []
        for f in faces:
            n = rng.normal(size=3)
            n /= np.linalg.norm(n)
            out.append(f[:3] + (tuple(n), f[4] * rng.uniform(.5, 1.5)) + f[5:])
        faces = out
    for j in range(extra_boundary):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        faces.append((j % nc, -1, -1, tuple(n), .004, .13, 1.0, 2))
    arr = (A.Face * len(faces))()
    for i, (o, nb, fx, n, area, dist, w, k) in enumerate(faces):
        arr[i] = A.Face(o, nb, fx, (C.c_double * 3)(*n), area, dist, w, k)
    fixed_states, fixed_y, fixed_h = ideal_states(fixed_q, ns)
    visc = .007 if (transport or viscous_only) else 0.0
    cfg = A.Config(nc, ns, nv, len(faces), n_fixed, visc, 2.0 if (transport or conduction) else 0.0,
                   .003 if transport else 0.0, 1.1, 2e8, int(mechanical))
    states, y, h = ideal_states(q, ns, mechanical)
    return dict(config=cfg, faces=arr, volume=volume, q=q, states=states, y=y, h=h,
                fixed_q=fixed_q if n_fixed else np.zeros((1, nv)), fixed_states=fixed_states,
                fixed_states_ptr=C.cast(states_ptr(fixed_states), C.c_void_p),
                fixed_y=fixed_y, fixed_h=fixed_h, ns=ns, nc=nc, nv=nv, mechanical=mechanical,
                name=f"ns{ns}-nc{nc}-b{kind}-t{int(transport)}-m{int(mechanical)}-s{int(spatial)}"
                     f"-x{extra_boundary}-f{frozen}")


# (ns, nc, boundary kind, transport, mechanical, spatial, extra boundary faces, frozen liquids)
CASES = ([(4, 7, b, t, False, False, 0, 0) for b in range(4) for t in (False, True)]
         + [(413, 7, 0, False, False, False, 0, 0), (53, 257, 0, True, False, False, 0, 0),
            (4, 1, 3, True, False, False, 0, 0), (8, 7, 0, False, True, False, 0, 0),
            (8, 7, 1, False, True, False, 0, 0), (4, 1, 0, False, False, False, 0, 0)]
         + [(4, 255, 3, True, False, True, 0, 0), (4, 256, 3, True, False, True, 0, 0),
            (4, 257, 3, True, False, True, 4097, 0), (413, 17, 3, True, False, True, 513, 0)]
         + [(4, 7, b, True, False, False, 0, nl) for nl in (1, 2) for b in range(4)])

# WALE cases: (ns, nc, kind, spatial, viscosity on, Cw)
WALE_CASES = [(1, 9, 0, True, False, .325), (2, 33, 3, True, True, .325), (4, 64, 1, True, False, .5),
              (1, 40, 2, True, True, .325)]


def case_from_tuple(t):
    ns, nc, kind, transport, mechanical, spatial, extra, frozen = t
    return make_case(ns, nc, kind, transport, mechanical, spatial, extra, frozen)


def primitives(q, states, ns):
    arr = (A.Primitive * len(q))()
    u = q[:, ns:ns + 3] / states["rho"][:, None]
    for c in range(len(q)):
        arr[c] = A.Primitive(states["rho"][c], (C.c_double * 3)(*u[c]))
    return arr


def dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def scaled_error(a, b):
    scale = np.maximum(1., np.max(np.abs(b), axis=0))
    return float(np.max(np.abs(a - b) / scale))


def create(lib, backend, case, wale_cw=None, wale_scalars=None):
    error = C.create_string_buffer(4096)
    cfg = case["config"]
    handle = lib.reactive_transport_create(
        backend, C.byref(cfg), dp(case["volume"]), case["faces"], dp(case["fixed_q"]),
        states_ptr(case["fixed_states"]), dp(case["fixed_y"]), dp(case["fixed_h"]), error, len(error))
    if not handle:
        raise RuntimeError(error.value.decode())
    if wale_cw is not None:
        opts = A.WaleOptions(1, C.sizeof(A.WaleOptions), wale_cw)
        if lib.reactive_transport_set_wale_v1(C.c_void_p(handle), C.byref(opts)):
            raise RuntimeError(lib.reactive_transport_error(C.c_void_p(handle)).decode())
    if wale_scalars is not None:
        opts = A.WaleScalarOptions(1, C.sizeof(A.WaleScalarOptions), *wale_scalars)
        if lib.reactive_transport_set_wale_scalars_v1(C.c_void_p(handle), C.byref(opts)):
            raise RuntimeError(lib.reactive_transport_error(C.c_void_p(handle)).decode())
    return C.c_void_p(handle)


def scalar_fields(case, seed=0):
    """Mixture cp (J/kg/K) and effective species enthalpies (J/kg, cell-major)
    for the cells and the fixed states of a case."""
    rng = np.random.default_rng(700 + seed)
    nc, ns, nf = case["nc"], case["ns"], max(1, case["config"].fixed)
    return dict(cell_cp=rng.uniform(900, 1600, nc), fixed_cp=rng.uniform(900, 1600, nf),
                cell_h=rng.uniform(-2e6, 3e6, (nc, ns)), fixed_h=rng.uniform(-2e6, 3e6, (nf, ns)))


def upload_scalar_fields(lib, handle, fields, with_h=True):
    return lib.reactive_transport_wale_scalar_fields_v1(
        handle, dp(fields["cell_cp"]), dp(fields["cell_h"]) if with_h else None, dp(fields["fixed_cp"]),
        dp(fields["fixed_h"]) if with_h else None)


def bind(lib):
    d, s, v = C.POINTER(C.c_double), C.POINTER(A.State), C.c_void_p
    sig = {
        "create": ([C.c_int, C.POINTER(A.Config), d, C.POINTER(A.Face), d, s, d, d, C.c_char_p, C.c_size_t], v),
        "destroy": ([v], None), "error": ([v], C.c_char_p), "is_cuda": ([v], C.c_int),
        "stats": ([v, C.POINTER(A.Stats)], C.c_int), "profile": ([v, C.POINTER(A.Profile)], C.c_int),
        "upload_conserved": ([v, d, C.c_uint64], C.c_int),
        "stable_step_primitives": ([v, C.POINTER(A.Primitive), s, C.c_double, C.c_double, d], C.c_int),
        "stage_resident": ([v, s, d, d, C.c_double, C.c_int, C.c_uint64, C.c_uint64, d, d], C.c_int),
        "rhs": ([v, d, s, d, d, d, d], C.c_int), "stage": ([v, d, s, d, d, C.c_double, C.c_int, d], C.c_int),
        "stable_step": ([v, d, s, C.c_double, C.c_double, d], C.c_int),
        "set_wale_v1": ([v, C.POINTER(A.WaleOptions)], C.c_int),
        "wale_primitives_v1": ([v, C.POINTER(A.Primitive), s, d], C.c_int),
        "set_wale_scalars_v1": ([v, C.POINTER(A.WaleScalarOptions)], C.c_int),
        "wale_scalar_profile_v1": ([v, C.POINTER(A.WaleScalarProfile)], C.c_int),
        "wale_scalar_fields_v1": ([v, d, d, d, d], C.c_int),
    }
    for name, (args, ret) in sig.items():
        fn = getattr(lib, "reactive_transport_" + name)
        fn.argtypes, fn.restype = args, ret
    return lib


def contract_walk(lib, backend, case, oracle):
    """Runs the reference's RHS/CFL/RK-stage/residency contract on `lib` and
    compares every numeric result with the oracle. Returns a summary dict."""
    ns, nc, nv = case["ns"], case["nc"], case["nv"]
    q = case["q"].copy()
    states, y, h = case["states"], case["y"], case["h"]
    handle = create(lib, backend, case)

    def check(status):
        if status:
            raise AssertionError(lib.reactive_transport_error(handle).decode())

    def oracle_rhs(qq, st, yy, hh):
        rhs, br, _, _, status = oracle.transport_rhs(case, qq, st.ctypes.data_as(C.c_void_p), yy, hh)
        assert status == 0
        return rhs, br

    def oracle_dt(qq, st):
        return oracle.transport_stable_dt(case, qq, st.ctypes.data_as(C.c_void_p), .23, .1)

    summary = {}
    try:
        assert bool(lib.reactive_transport_is_cuda(handle)) == bool(backend)
        rhs, br = np.empty_like(q), np.empty(nv)
        check(lib.reactive_transport_rhs(handle, dp(q), states_ptr(states), dp(y), dp(h), dp(rhs), dp(br)))
        expected, expected_br = oracle_rhs(q, states, y, h)
        summary["rhs_error"] = err = scaled_error(rhs, expected)
        assert err <= RHS_TOL, f"operator mismatch {err}"
        berr = scaled_error(br[None, :], expected_br[None, :])
        assert berr <= RHS_TOL, f"boundary ledger mismatch {berr}: {br} vs {expected_br}"
        dt = C.c_double()
        check(lib.reactive_transport_stable_step(handle, dp(q), states_ptr(states), .23, .1, C.byref(dt)))
        expected_dt = oracle_dt(q, states)
        summary["dt_error"] = abs(dt.value / expected_dt - 1)
        assert summary["dt_error"] < DT_TOL
        balance = (rhs * case["volume"][:, None]).sum(axis=0) + br
        lim = ns + 4
        assert np.all(np.abs(balance[:lim]) <= BALANCE_TOL * np.maximum(
            1, np.sum(np.abs(rhs[:, :lim] * case["volume"][:, None]), axis=0)))
        if case["mechanical"]:
            assert np.max(np.abs(rhs[:, -2:].sum(axis=1))) < 1e-10
        original = q.copy()
        step = .1 * dt.value
        # An orphan stage 1 is rejected; a fresh stage 0 recovers.
        assert lib.reactive_transport_stage(handle, dp(q), states_ptr(states), dp(y), dp(h), step, 1, dp(br)) != 0
        check(lib.reactive_transport_stage(handle, dp(q), states_ptr(states), dp(y), dp(h), step, 0, dp(br)))
        assert scaled_error(q, original + step * expected) <= RHS_TOL
        st1, y1, h1 = ideal_states(q, ns, case["mechanical"])
        rhs1, _ = oracle_rhs(q, st1, y1, h1)
        expected_final = .5 * original + .5 * (q + step * rhs1)
        check(lib.reactive_transport_stable_step(handle, dp(q), states_ptr(st1), .23, .1, C.byref(dt)))
        check(lib.reactive_transport_stage(handle, dp(q), states_ptr(st1), dp(y1), dp(h1), step, 1, dp(br)))
        summary["stage_error"] = scaled_error(q, expected_final)
        assert summary["stage_error"] <= RHS_TOL
        # Rollback: a rejected step restarts stage 0 from the caller's copy.
        q[:] = original
        check(lib.reactive_transport_stage(handle, dp(q), states_ptr(states), dp(y), dp(h), step / 2, 0, dp(br)))
        assert scaled_error(q, original + step / 2 * expected) <= RHS_TOL
        # Resident cycle: three CFL queries, two stages, exactly one upload.
        q[:] = original
        before = A.Profile()
        check(lib.reactive_transport_profile(handle, C.byref(before)))
        prim = primitives(q, states, ns)
        check(lib.reactive_transport_stable_step_primitives(handle, prim, states_ptr(states), .23, .1, C.byref(dt)))
        assert abs(dt.value / expected_dt - 1) < DT_TOL
        check(lib.reactive_transport_upload_conserved(handle, dp(q), 10))
        check(lib.reactive_transport_upload_conserved(handle, dp(q), 10))
        check(lib.reactive_transport_stable_step_primitives(handle, prim, states_ptr(states), .23, .1, C.byref(dt)))
        check(lib.reactive_transport_stage_resident(handle, states_ptr(states), dp(y), dp(h), step, 0, 10, 11,
                                                    dp(q), dp(br)))
        assert scaled_error(q, original + step * expected) <= RHS_TOL
        rs, ry, rh = ideal_states(q, ns, case["mechanical"])
        check(lib.reactive_transport_stable_step_primitives(handle, primitives(q, rs, ns), states_ptr(rs), .23, .1,
                                                            C.byref(dt)))
        check(lib.reactive_transport_stage_resident(handle, states_ptr(rs), dp(ry), dp(rh), step, 1, 11, 12, dp(q),
                                                    dp(br)))
        assert scaled_error(q, expected_final) <= RHS_TOL
        after = A.Profile()
        check(lib.reactive_transport_profile(handle, C.byref(after)))
        assert after.conservedUploads - before.conservedUploads == 1
        assert after.conservedUploadBytes - before.conservedUploadBytes == q.nbytes
        assert after.conservedDownloadBytes - before.conservedDownloadBytes == 2 * q.nbytes
        assert after.residentStages - before.residentStages == 2
        # A stale input version fails and invalidates residency.
        assert lib.reactive_transport_stage_resident(handle, states_ptr(rs), dp(ry), dp(rh), step, 1, 11, 13, dp(q),
                                                     dp(br)) != 0
        q[:] = original
        check(lib.reactive_transport_upload_conserved(handle, dp(q), 20))
        check(lib.reactive_transport_stage_resident(handle, states_ptr(states), dp(y), dp(h), step / 2, 0, 20, 21,
                                                    dp(q), dp(br)))
        assert scaled_error(q, original + step / 2 * expected) <= RHS_TOL
        # The same host storage, changed content, new version.
        q[:] = original * 1.001
        altered = q.copy()
        ar, ay, ah = ideal_states(q, ns, case["mechanical"])
        arhs, _ = oracle_rhs(q, ar, ay, ah)
        check(lib.reactive_transport_upload_conserved(handle, dp(q), 30))
        check(lib.reactive_transport_stage_resident(handle, states_ptr(ar), dp(ay), dp(ah), step / 2, 0, 30, 31,
                                                    dp(q), dp(br)))
        assert scaled_error(q, altered + step / 2 * arhs) <= RHS_TOL
        # Invalid velocities at different reduction positions fail.
        for c in sorted({0, nc // 2, nc - 1}):
            bad = primitives(original, states, ns)
            bad[c].u[1] = float("nan")
            assert lib.reactive_transport_stable_step_primitives(handle, bad, states_ptr(states), .23, .1,
                                                                 C.byref(dt)) != 0
        check(lib.reactive_transport_stable_step_primitives(handle, prim, states_ptr(states), .23, .1, C.byref(dt)))
        assert abs(dt.value / expected_dt - 1) < DT_TOL
        return summary
    finally:
        lib.reactive_transport_destroy(handle)


def large_cfl_walk(lib, backend, nc):
    """Multi-level CFL reduction with an overflowing cell at three positions."""
    cfg = A.Config(nc, 1, 5, nc, 0, 0, 0, 0, 1.1, 2e8, 0)
    volume = np.full(nc, .2)
    st = np.zeros(nc, dtype=A.STATE_DTYPE)
    st["p"], st["T"], st["rho"], st["cv"], st["sound"], st["gasMass"] = 1e5, 300, 1, 717, 300, 1
    prim = (A.Primitive * nc)(*[A.Primitive(1, (C.c_double * 3)(5, 0, 0))] * nc)
    faces = (A.Face * nc)(*[A.Face(c, (c + 1) % nc, -1, (C.c_double * 3)(1, 0, 0), 1, .2, .5, 0)
                            for c in range(nc)])
    error = C.create_string_buffer(4096)
    handle = lib.reactive_transport_create(backend, C.byref(cfg), dp(volume), faces, None, None, None, None,
                                           error, len(error))
    assert handle, error.value.decode()
    handle = C.c_void_p(handle)
    try:
        dt = C.c_double()
        expected = .23 * .2 / (2 * (5 + 1.1 * 300))
        assert lib.reactive_transport_stable_step_primitives(handle, prim, states_ptr(st), .23, .1, C.byref(dt)) == 0
        assert abs(dt.value / expected - 1) < DT_TOL
        for c in (0, nc // 2, nc - 1):
            prim[c].u[0] = 1e308
            assert lib.reactive_transport_stable_step_primitives(handle, prim, states_ptr(st), .23, .1,
                                                                 C.byref(dt)) != 0
            prim[c].u[0] = 5
        assert lib.reactive_transport_stable_step_primitives(handle, prim, states_ptr(st), .23, .1, C.byref(dt)) == 0
        prof = A.Profile()
        assert lib.reactive_transport_profile(handle, C.byref(prof)) == 0
        assert prof.conservedUploadBytes == 0
    finally:
        lib.reactive_transport_destroy(handle)


def wale_scalar_contract(lib, backend):
    """The WALE scalar closure's install preconditions, field validation and
    stage/CFL preconditions (src/reactiveTransport/reactiveTransport.cpp:653-702,
    :1395-1397, :1415-1416) on one implementation."""
    ns, nc, kind, spatial, viscous, cw = WALE_CASES[1]
    case = make_case(ns, nc, kind, spatial=spatial, viscous_only=viscous, seed=5)
    fields = scalar_fields(case)
    q, st = case["q"], case["states"]
    rhs, br, dt = np.empty_like(q), np.empty(case["nv"]), C.c_double()
    opts = lambda pr, sc: C.byref(A.WaleScalarOptions(1, C.sizeof(A.WaleScalarOptions), pr, sc))
    h = create(lib, backend, case)
    try:  # without WALE
        assert lib.reactive_transport_set_wale_scalars_v1(h, opts(.9, .7)) != 0
    finally:
        lib.reactive_transport_destroy(h)
    h = create(lib, backend, case, wale_cw=cw)
    try:
        assert lib.reactive_transport_set_wale_scalars_v1(h, opts(-1, .7)) != 0
        assert lib.reactive_transport_set_wale_scalars_v1(h, opts(.9, float("nan"))) != 0
        bad = A.WaleScalarOptions(2, C.sizeof(A.WaleScalarOptions), .9, .7)
        assert lib.reactive_transport_set_wale_scalars_v1(h, C.byref(bad)) != 0
        assert lib.reactive_transport_set_wale_scalars_v1(h, opts(.9, .7)) == 0
        assert lib.reactive_transport_set_wale_scalars_v1(h, opts(.9, .7)) != 0  # immutable
        # not uploaded: stage and CFL refuse
        assert lib.reactive_transport_rhs(h, dp(q), states_ptr(st), None, None, dp(rhs), dp(br)) != 0
        assert lib.reactive_transport_stable_step(h, dp(q), states_ptr(st), .23, .1, C.byref(dt)) != 0
        badcp = dict(fields, cell_cp=fields["cell_cp"].copy())
        badcp["cell_cp"][3] = 0.0
        assert upload_scalar_fields(lib, h, badcp) != 0
        badh = dict(fields, fixed_h=fields["fixed_h"].copy())
        badh["fixed_h"][0, 1] = float("inf")
        assert upload_scalar_fields(lib, h, badh) != 0
        # cp only: the CFL runs, the RHS needs the enthalpies too
        assert upload_scalar_fields(lib, h, fields, with_h=False) == 0
        assert lib.reactive_transport_stable_step(h, dp(q), states_ptr(st), .23, .1, C.byref(dt)) == 0
        assert lib.reactive_transport_rhs(h, dp(q), states_ptr(st), None, None, dp(rhs), dp(br)) != 0
        assert upload_scalar_fields(lib, h, fields) == 0
        assert lib.reactive_transport_rhs(h, dp(q), states_ptr(st), None, None, dp(rhs), dp(br)) == 0
        prof = A.WaleScalarProfile(1, C.sizeof(A.WaleScalarProfile))
        assert lib.reactive_transport_wale_scalar_profile_v1(h, C.byref(prof)) == 0
        all_ = nc + case["config"].fixed
        assert prof.fieldUploads == 2
        assert prof.fieldUploadBytes == 2 * all_ * 8 + all_ * ns * 8
    finally:
        lib.reactive_transport_destroy(h)
    # species mixing needs variables == species + 4
    frozen = make_case(2, 7, 2, transport=True, frozen=1)
    h = create(lib, backend, frozen, wale_cw=.325)
    try:
        assert lib.reactive_transport_set_wale_scalars_v1(h, opts(.9, .7)) != 0
        assert lib.reactive_transport_set_wale_scalars_v1(h, opts(.9, 0)) == 0
    finally:
        lib.reactive_transport_destroy(h)
