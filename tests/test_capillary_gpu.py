"""GPU parity of the diffuse capillary closure on the face graph
(reactive_transport_set_capillary_v1 / capillary_geometry_v1 /
capillary_profile_v1 and every stage entry with the closure installed) against
the reference's own CPU build (backend 0) on the same inputs: interface
geometry (surface energy, curvature, normal) within 1e-12, operator and RK
stages within the transport tolerance (3e-12 scaled), CFL steps within 3e-14,
the same profile counters and the same error messages."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, _lib
import capillary_cases as K
import transport_cases as T

pytestmark = pytest.mark.gpu

GRAPH_CASES = [dict(ns=4, nc=7, kind=0), dict(ns=4, nc=33, kind=1), dict(ns=2, nc=40, kind=2),
               dict(ns=3, nc=64, kind=3), dict(ns=4, nc=257, kind=3, extra_boundary=300, species=2),
               dict(ns=53, nc=57, kind=0, species=7), dict(ns=1, nc=129, kind=1, spatial=False)]


@pytest.fixture(scope="module")
def libs():
    # a private handle on the reference build: the shared one keeps the untyped
    # signatures other tests give it
    oracle.ref_transport_lib()
    return K.bind(C.CDLL(str(oracle.REF_TRANSPORT))), K.bind(_lib.load())


def pair(libs, case, **kw):
    ref, ours = libs
    return K.Handle(ref, 0, case, **kw), K.Handle(ours, 1, case, **kw)


def compare_geometry(a, b):
    for x, y in zip(a, b):
        assert K.relative(y, x) <= K.GEOMETRY_TOL


def test_periodic_interface_with_wale_scalars_matches_reference(libs):
    """The reference's own capillary transport scenario, end to end."""
    case = K.periodic_interface()
    n, ns, nv = case["nc"], case["ns"], case["nv"]
    r, o = pair(libs, case, wale_cw=.325, wale_scalars=(.9, .7))
    try:
        cp, sh = np.full(n, 1000.0), np.full((n, ns), 5e4)
        for h in (r, o):
            h.check(h.lib.reactive_transport_wale_scalar_fields_v1(h.h, T.dp(cp), T.dp(sh), None, None))
        bad = case["color"].copy()
        bad[0] = -1
        for h in (r, o):
            with pytest.raises(RuntimeError, match="Invalid material color"):
                h.geometry(bad)
        gr, go = r.geometry(), o.geometry()
        compare_geometry(gr, go)
        q = case["q"].copy()
        q[:, ns + 3] += gr[0]
        rr, br = r.rhs(q, case["states"])
        ro, bo = o.rhs(q, case["states"])
        assert T.scaled_error(ro, rr) <= T.RHS_TOL
        assert T.scaled_error(bo[None], br[None]) <= T.RHS_TOL
        assert np.all(np.abs((ro * case["volume"][:, None]).sum(axis=0)) < 1e-7)   # periodic conservation
        pr, po = r.profile(), o.profile()
        assert po == pr
        assert po["geometryBuilds"] == 1 and po["geometryKernels"] == 2 and po["faceFluxBuilds"] == n
        # the resident RK attempt with a post-RK1 replacement, as the reference drives it
        results = []
        for h in (r, o):
            L = h.lib
            qq = q.copy()
            h.check(L.reactive_transport_begin_attempt(h.h, K.MODEL_HASH, 1))
            h.check(L.reactive_transport_upload_conserved(h.h, T.dp(qq), 1))
            bnd = np.empty(nv)
            st = case["states"]
            h.check(L.reactive_transport_advance_resident_v2(h.h, A.Token(1, 0, 1), A.Token(1, 1, 2),
                                                             T.states_ptr(st), None, None, None, 1e-9, T.dp(bnd)))
            h.check(L.reactive_transport_download_conserved(h.h, A.Token(1, 1, 2), T.dp(qq)))
            qq[:, ns + 3] += 1
            h.check(L.reactive_transport_replace_stage_state_v1(h.h, A.Token(1, 1, 2), 3, T.dp(qq)))
            h.check(L.reactive_transport_advance_resident_v2(h.h, A.Token(1, 1, 3), A.Token(1, 2, 4),
                                                             T.states_ptr(st), None, None, None, 1e-9, T.dp(bnd)))
            h.check(L.reactive_transport_download_conserved(h.h, A.Token(1, 2, 4), T.dp(qq)))
            h.check(L.reactive_transport_end_attempt(h.h, 1, 1))
            results.append((qq, bnd.copy()))
        assert T.scaled_error(results[1][0], results[0][0]) <= T.RHS_TOL
        assert T.scaled_error(results[1][1][None], results[0][1][None]) <= T.RHS_TOL
    finally:
        r.close()
        o.close()


@pytest.mark.parametrize("spec", GRAPH_CASES, ids=lambda s: "-".join(f"{k}{v}" for k, v in s.items()))
def test_face_graph_capillary_contract_matches_reference(libs, spec):
    case = K.graph_case(**spec)
    ns, nv = case["ns"], case["nv"]
    r, o = pair(libs, case)
    try:
        compare_geometry(r.geometry(), o.geometry())
        q, st, y, h = case["q"], case["states"], case["y"], case["h"]
        rr, br = r.rhs(q, st, y, h)
        ro, bo = o.rhs(q, st, y, h)
        assert T.scaled_error(ro, rr) <= T.RHS_TOL
        assert T.scaled_error(bo[None], br[None]) <= T.RHS_TOL
        dr, do = r.stable_step(q, st), o.stable_step(q, st)
        assert abs(do / dr - 1) < T.DT_TOL
        step = .1 * dr
        qs = []
        for hd in (r, o):
            qq = q.copy()
            hd.stage(qq, st, step, 0, y, h)
            st1, y1, h1 = T.ideal_states(qq, ns)
            hd.stage(qq, st1, step, 1, y1, h1)
            qs.append(qq)
        assert T.scaled_error(qs[1], qs[0]) <= T.RHS_TOL
        assert o.profile() == r.profile()
    finally:
        r.close()
        o.close()


def test_capillary_wave_step_bounds_the_cfl_like_reference(libs):
    """A large surface tension makes the capillary wave bound
    capCfl sqrt(rho V / (pi sigma)) the smallest step."""
    case = K.graph_case(4, 64, 3)
    sigma = 2e9
    opts = K.options(sigma=sigma, cfl=.4)
    r, o = pair(libs, case, opts=opts)
    try:
        compare_geometry(r.geometry(), o.geometry())
        q, st = case["q"], case["states"]
        dr, do = r.stable_step(q, st), o.stable_step(q, st)
        assert abs(do / dr - 1) < T.DT_TOL
        energy = o.geometry()[0]
        area = energy / sigma
        active = area * np.cbrt(case["volume"]) > 1e-10
        bound = .4 * np.sqrt(st["rho"] * case["volume"] / (np.pi * sigma))
        assert active.any()
        assert abs(do / bound[active].min() - 1) < 1e-13
        rr, _ = r.rhs(q, st, case["y"], case["h"])
        ro, _ = o.rhs(q, st, case["y"], case["h"])
        assert T.scaled_error(ro, rr) <= T.RHS_TOL
    finally:
        r.close()
        o.close()


def test_wale_scalar_liquid_share_matches_reference(libs):
    """WALE with total-species mixing: the liquid inventory moves with its
    species' turbulent flux in proportion to its liquid fraction."""
    case = K.graph_case(3, 48, 3, species=1, seed=3)
    r, o = pair(libs, case, wale_cw=.325, wale_scalars=(.85, .7))
    try:
        f = T.scalar_fields(case, seed=4)
        for hd in (r, o):
            hd.check(T.upload_scalar_fields(hd.lib, hd.h, f))
        compare_geometry(r.geometry(), o.geometry())
        q, st, y, h = case["q"], case["states"], case["y"], case["h"]
        rr, br = r.rhs(q, st, y, h)
        ro, bo = o.rhs(q, st, y, h)
        assert T.scaled_error(ro, rr) <= T.RHS_TOL
        assert T.scaled_error(bo[None], br[None]) <= T.RHS_TOL
        assert np.abs(rr[:, case["ns"] + 4]).max() > 0
    finally:
        r.close()
        o.close()


def test_identical_geometry_request_skips_the_device(libs):
    case = K.graph_case(4, 33, 1)
    r, o = pair(libs, case)
    try:
        first = [hd.geometry(normal=False) for hd in (r, o)]
        again = [hd.geometry(normal=False) for hd in (r, o)]
        for a, b in zip(first, again):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        assert o.profile() == r.profile()
        assert o.profile()["geometryBuilds"] == 1
        changed = case["color"].copy()
        changed[3] = .5 * changed[3]
        for hd in (r, o):
            hd.geometry(changed, normal=False)
        assert o.profile() == r.profile()
        assert o.profile()["geometryBuilds"] == 2
    finally:
        r.close()
        o.close()


def test_capillary_errors_match_reference(libs):
    ref, ours = libs
    case = K.graph_case(4, 33, 3)
    messages = []
    for lib, backend in ((ref, 0), (ours, 1)):
        got = []
        h = K.Handle(lib, backend, case)
        try:
            q, st = case["q"], case["states"]
            # a stage before the geometry
            with pytest.raises(RuntimeError) as e:
                h.rhs(q, st, case["y"], case["h"])
            got.append(str(e.value))
            with pytest.raises(RuntimeError) as e:
                h.geometry(fixed_color=np.array([1.5]))
            got.append(str(e.value))
            # a second installation
            got.append(lib.reactive_transport_set_capillary_v1(h.h, C.byref(K.options())) != 0 and h.error())
            h.geometry()
            # a liquid inventory above its species' density
            bad = q.copy()
            bad[5, case["ns"] + 4] = 1.5 * bad[5, 0]
            with pytest.raises(RuntimeError) as e:
                h.rhs(bad, st, case["y"], case["h"])
            got.append(str(e.value))
            p = A.CapillaryProfile(1, 8)
            got.append(lib.reactive_transport_capillary_profile_v1(h.h, C.byref(p)) != 0 and h.error())
        finally:
            h.close()
        for opts in (K.options(sigma=0.0), K.options(cfl=1.5), K.options(eps=1.0), K.options(species=4)):
            h = T.create(lib, backend, case)
            try:
                got.append(lib.reactive_transport_set_capillary_v1(h, C.byref(opts)) != 0
                           and lib.reactive_transport_error(h).decode())
            finally:
                lib.reactive_transport_destroy(h)
        plain = T.make_case(4, 9, 0)
        h = T.create(lib, backend, plain)
        try:
            got.append(lib.reactive_transport_set_capillary_v1(h, C.byref(K.options())) != 0
                       and lib.reactive_transport_error(h).decode())
        finally:
            lib.reactive_transport_destroy(h)
        messages.append(got)
    assert messages[1] == messages[0]
    assert "Capillary geometry must be uploaded for this stage" in messages[1][0]
    assert "Invalid fixed material color" in messages[1][1]
    assert "installed once before stepping" in messages[1][2]
    assert "Invalid capillary face flux" in messages[1][3]
    assert "Invalid capillary profile ABI" in messages[1][4]
    assert all("Invalid capillary options ABI/model" in m for m in messages[1][5:8])
    assert "one mapped conserved liquid inventory" in messages[1][8]
    assert "one mapped conserved liquid inventory" in messages[1][9]


def test_device_stage_with_capillary_matches_host_stage(libs):
    """The device-resident stage consumes the published geometry and reports a
    failed capillary face in bit 3 of the status word."""
    import torch
    ref, ours = libs
    L = _lib.load()
    case = K.graph_case(4, 40, 3, transport=False, seed=2)
    ns, nc, nv = case["ns"], case["nc"], case["nv"]
    r, o = pair(libs, case)
    try:
        r.geometry()
        o.geometry()
        q, st = case["q"], case["states"]
        step = .1 * r.stable_step(q, st)
        expected = q.copy()
        r.stage(expected, st, step, 0, case["y"], case["h"])
        cells, fixed, nvar, nsp = (C.c_size_t() for _ in range(4))
        assert L.reactive_transport_layout_v3(o.h, C.byref(cells), C.byref(fixed), C.byref(nvar), C.byref(nsp)) == 0
        all_ = nc + fixed.value
        stream = torch.cuda.current_stream().cuda_stream
        q0 = torch.zeros((nv, all_), dtype=torch.float64, device="cuda")
        q0[:, :nc] = torch.from_numpy(q.T.copy()).cuda()
        sd = torch.zeros((all_, 7), dtype=torch.float64, device="cuda")
        sd[:nc] = torch.from_numpy(st.view(np.float64).reshape(nc, 7)).cuda()
        assert L.reactive_transport_fill_fixed_v3(o.h, q0.data_ptr(), sd.data_ptr(), stream) == 0
        q1 = q0.clone()
        status = C.c_uint()
        assert L.reactive_transport_status_v3(o.h, C.byref(status), 1, stream) == 0
        assert L.reactive_transport_stage_device_v3(o.h, q0.data_ptr(), q1.data_ptr(), sd.data_ptr(), step, 0, None,
                                                    stream) == 0, o.error()
        assert L.reactive_transport_status_v3(o.h, C.byref(status), 1, stream) == 0
        assert status.value == 0
        assert T.scaled_error(q1[:, :nc].cpu().numpy().T, expected) <= T.RHS_TOL
        q0[ns + 4, 7] = 2 * q0[0, 7]
        assert L.reactive_transport_stage_device_v3(o.h, q0.data_ptr(), q1.data_ptr(), sd.data_ptr(), step, 0, None,
                                                    stream) == 0
        assert L.reactive_transport_status_v3(o.h, C.byref(status), 1, stream) == 0
        assert status.value & 8
    finally:
        r.close()
        o.close()
