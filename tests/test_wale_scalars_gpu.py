"""GPU: the WALE scalar closure (turbulent Prandtl heat flux and turbulent
Schmidt species mixing, src/reactiveTransport/reactiveTransportKernels.h:150-168,
:323-336, :440-477) on this library: the face graph's host entries against the
oracle (itself pinned to the reference CPU build), the reference's install and
upload contract, the structured path (FP64 bitwise equal to the face graph, the
mixed form within its FP32 tolerance), the device-resident field entry against
the host upload, and the SSPRK2 + HEM step driver with the closure against the
reference's RK driver over its own CPU transport."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, _lib, thermo_data as td
from spuma_multiphysics_b200.flow import Flow
import rk_oracle
import transport_cases as T
from test_structured_gpu import BOXES, _stage_pair, box_case, mixed_kinds
from test_wale_scalars_oracle import SCALAR_CASES, oracle_rhs_dt

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return T.bind(_lib.load())


@pytest.mark.parametrize("spec,pr,sc", SCALAR_CASES, ids=lambda s: "-".join(map(str, s)) if isinstance(s, tuple)
                         else str(s))
def test_face_graph_host_entries_against_oracle(lib, spec, pr, sc):
    ns, nc, kind, spatial, viscous, cw = spec
    case = T.make_case(ns, nc, kind, transport=False, spatial=spatial, viscous_only=viscous, seed=5)
    fields = T.scalar_fields(case, seed=nc)
    h = T.create(lib, 1, case, wale_cw=cw, wale_scalars=(pr, sc))
    try:
        q, st = case["q"], case["states"]
        assert T.upload_scalar_fields(lib, h, fields) == 0, lib.reactive_transport_error(h)
        rhs, br = np.empty_like(q), np.empty(case["nv"])
        assert lib.reactive_transport_rhs(h, T.dp(q), T.states_ptr(st), None, None, T.dp(rhs), T.dp(br)) == 0, \
            lib.reactive_transport_error(h)
        dt = C.c_double()
        assert lib.reactive_transport_stable_step(h, T.dp(q), T.states_ptr(st), .23, .1, C.byref(dt)) == 0
        exp, exp_br, status, odt = oracle_rhs_dt(case, q, st, cw, pr, sc, fields)
        assert status == 0
        assert T.scaled_error(rhs, exp) <= T.RHS_TOL
        assert T.scaled_error(br[None], exp_br[None]) <= T.RHS_TOL
        assert abs(dt.value / odt - 1) < T.DT_TOL
        prof = A.WaleScalarProfile(1, C.sizeof(A.WaleScalarProfile))
        assert lib.reactive_transport_wale_scalar_profile_v1(h, C.byref(prof)) == 0
        all_ = nc + case["config"].fixed
        assert prof.fieldUploads == 1
        assert prof.fieldUploadBytes == (all_ * 8 if pr > 0 else 0) + (all_ * ns * 8 if sc > 0 else 0)
    finally:
        lib.reactive_transport_destroy(h)


def test_contract(lib):
    T.wale_scalar_contract(lib, 1)


def box_fields(case, seed):
    rng = np.random.default_rng(seed)
    nc, ns, nf = case["nc"], case["ns"], max(1, case["config"].fixed)
    return dict(cell_cp=rng.uniform(900, 1600, nc), fixed_cp=rng.uniform(900, 1600, nf),
                cell_h=rng.uniform(-2e6, 3e6, (nc, ns)), fixed_h=rng.uniform(-2e6, 3e6, (nf, ns)))


SCALAR_BOXES = [(b, pr, sc) for b in BOXES if b.get("wale") for pr, sc in ((.9, .7), (.85, 0.0), (0.0, .6))]


@pytest.mark.parametrize("spec,pr,sc", SCALAR_BOXES,
                         ids=lambda s: "x".join(map(str, s["dims"])) + f"-ns{s['ns']}" if isinstance(s, dict)
                         else str(s))
def test_structured_matches_face_graph_and_oracle(lib, spec, pr, sc):
    import torch
    L = _lib.load()
    kinds = mixed_kinds(spec["dims"], 17) if spec["kinds"] == "mixed" else spec["kinds"]
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    cw = spec["wale"]
    fields = box_fields(case, 3)
    h = T.create(lib, 1, case, wale_cw=cw, wale_scalars=(pr, sc))
    try:
        active = C.c_int(-1)
        assert L.reactive_transport_structured_v3(h, -1, C.byref(active)) == 0 and active.value == 1
        stream = torch.cuda.current_stream().cuda_stream
        # the device stage entries refuse until the fields are set
        q0 = torch.zeros((case["nv"], case["nc"] + case["config"].fixed), dtype=torch.float64, device="cuda")
        st0 = torch.zeros((case["nc"] + case["config"].fixed, 7), dtype=torch.float64, device="cuda")
        assert L.reactive_transport_stage_device_v3(h, q0.data_ptr(), q0.clone().data_ptr(), st0.data_ptr(), 1e-9, 0,
                                                    None, stream) != 0
        assert b"were not uploaded" in lib.reactive_transport_error(h)
        assert T.upload_scalar_fields(lib, h, fields) == 0, lib.reactive_transport_error(h)
        box = _stage_pair(L, h, case, stream, torch)
        assert L.reactive_transport_structured_v3(h, 0, None) == 0
        graph = _stage_pair(L, h, case, stream, torch)
        assert box["status"] == 0 and graph["status"] == 0
        assert box["dt"] == graph["dt"]
        assert np.array_equal(box["q1"], graph["q1"])
        assert np.array_equal(box["qn"], graph["qn"])
        for k in ("br0", "br1"):
            assert T.scaled_error(box[k][None], graph[k][None]) <= T.RHS_TOL
        # the oracle with the same fields for both stages
        exp, exp_br, status, odt = oracle_rhs_dt(case, case["q"], case["states"], cw, pr, sc, fields)
        assert status == 0
        assert abs(box["dt"] / odt - 1) < T.DT_TOL
        step = box["step"]
        assert T.scaled_error(box["q1"], case["q"] + step * exp) <= T.RHS_TOL
        assert T.scaled_error(box["br0"][None], exp_br[None]) <= T.RHS_TOL
        exp1, exp_br1, _, _ = oracle_rhs_dt(case, box["q1"], box["st1"], cw, pr, sc, fields)
        assert T.scaled_error(box["qn"], .5 * case["q"] + .5 * (box["q1"] + step * exp1)) <= T.RHS_TOL
        assert T.scaled_error(box["br1"][None], exp_br1[None]) <= T.RHS_TOL
        # the mixed form against the oracle at its FP32 tolerance
        assert L.reactive_transport_structured_v3(h, 1, None) == 0
        assert L.reactive_transport_precision_v3(h, 1, None) == 0
        mixed = _stage_pair(L, h, case, stream, torch)
        assert mixed["status"] == 0
        assert T.scaled_error((mixed["q1"] - case["q"]) / mixed["step"], exp) <= 2e-5
        assert T.scaled_error(mixed["br0"][None], exp_br[None]) <= 2e-5
        # the closure is not the identity here (one species mixes nothing: only
        # its diffusivity enters the CFL step)
        plain, _, _, pdt = oracle_rhs_dt(case, case["q"], case["states"], cw, 0, 0, fields)
        if spec["ns"] > 1 or pr > 0:
            assert T.scaled_error(plain, exp) > 1e-9
        assert pdt > odt
        # the rate VJP does not cover the closure
        w = torch.zeros((case["nv"], case["nc"]), dtype=torch.float64, device="cuda")
        qb, sb = torch.zeros_like(w), torch.zeros((case["nc"], 7), dtype=torch.float64, device="cuda")
        assert L.reactive_transport_precision_v3(h, 0, None) == 0
        assert L.reactive_transport_rate_vjp_v3(h, q0.data_ptr(), st0.data_ptr(), w.data_ptr(), qb.data_ptr(),
                                                sb.data_ptr(), stream) != 0
    finally:
        lib.reactive_transport_destroy(h)


def test_device_field_entry_matches_host_upload(lib):
    """Strided device fields (cp every 3rd double, enthalpies in rows of ns+2)
    give the same stages as the host upload, bit for bit; an invalid device cp
    sets bit 2 of the status word."""
    import torch
    L = _lib.load()
    spec = BOXES[3]
    kinds = mixed_kinds(spec["dims"], 17)
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    fields = box_fields(case, 5)
    nc, ns, nf = case["nc"], case["ns"], case["config"].fixed
    assert nf == 1
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for route in ("host", "device"):
        h = T.create(lib, 1, case, wale_cw=spec["wale"], wale_scalars=(.9, .7))
        try:
            if route == "host":
                assert T.upload_scalar_fields(lib, h, fields) == 0
            else:
                def strided(cp, hh):
                    a = np.zeros((len(cp), 3))
                    a[:, 1] = cp
                    b = np.zeros((len(cp), ns + 2))
                    b[:, :ns] = hh
                    return torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
                ccp, ch = strided(fields["cell_cp"], fields["cell_h"])
                fcp, fh = strided(fields["fixed_cp"], fields["fixed_h"])
                assert L.reactive_transport_wale_scalar_fields_device_v3(
                    h, ccp.data_ptr() + 8, ch.data_ptr(), fcp.data_ptr() + 8, fh.data_ptr(), 3, ns + 2, stream) == 0
                # NULL enthalpies invalidate them (more than one species)
                assert L.reactive_transport_wale_scalar_fields_device_v3(
                    h, ccp.data_ptr() + 8, None, None, None, 3, ns + 2, stream) == 0
                q0 = torch.zeros((case["nv"], nc + nf), dtype=torch.float64, device="cuda")
                st0 = torch.zeros((nc + nf, 7), dtype=torch.float64, device="cuda")
                assert L.reactive_transport_stage_device_v3(h, q0.data_ptr(), q0.clone().data_ptr(), st0.data_ptr(),
                                                            1e-9, 0, None, stream) != 0
                assert L.reactive_transport_wale_scalar_fields_device_v3(
                    h, ccp.data_ptr() + 8, ch.data_ptr(), None, None, 3, ns + 2, stream) == 0
            results.append(_stage_pair(L, h, case, stream, torch))
            if route == "device":
                bad = ccp.clone()
                bad[7, 1] = -5.0
                assert L.reactive_transport_wale_scalar_fields_device_v3(
                    h, bad.data_ptr() + 8, ch.data_ptr(), None, None, 3, ns + 2, stream) == 0
                status = C.c_uint()
                assert L.reactive_transport_status_v3(h, C.byref(status), 1, stream) == 0
                assert status.value == 4
        finally:
            lib.reactive_transport_destroy(h)
    a, b = results
    assert a["status"] == 0 and b["status"] == 0
    assert a["dt"] == b["dt"]
    assert np.array_equal(a["q1"], b["q1"]) and np.array_equal(a["qn"], b["qn"])


@pytest.mark.parametrize("graph", [False, True])
def test_flow_with_closure_matches_reference_rk_driver(graph):
    """The step driver with the closure fed by the flash's mixture cp against
    the reference RK driver with the same cp uploaded each stage through the
    reference's own host entry."""
    from test_flow_gpu import FIELD_TOL, small_case
    n, steps, dt = 12, 3, 1e-8
    faces, volume, init = small_case(n)
    kw = dict(viscosity=1.821e-5, conductivity=0.02587, wale_cw=0.325, turbulent_prandtl=.85,
              turbulent_schmidt=.7)
    flow = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], **kw)
    ref = rk_oracle.ReferenceFlow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"],
                                  image=td.model_bytes(td.pure_model()), **kw)
    plain = rk_oracle.ReferenceFlow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"],
                                    image=td.model_bytes(td.pure_model()), viscosity=kw["viscosity"],
                                    conductivity=kw["conductivity"], wale_cw=kw["wale_cw"])
    try:
        for _ in range(steps):
            flow.step(dt, graph=graph)
            ref.step(dt)
            plain.step(dt)
        flow.check(dt)
        q, s = flow.conserved(), flow.states()
        rel = lambda a, b, scale: float(np.max(np.abs(a - b)) / scale)
        assert rel(q[:, 0], ref.q[:, 0], ref.q[:, 0].max()) < FIELD_TOL
        assert rel(q[:, 1:4], ref.q[:, 1:4], max(1.0, np.abs(ref.q[:, 1:4]).max())) < 1e-7
        assert rel(q[:, 4], ref.q[:, 4], np.abs(ref.q[:, 4]).max()) < FIELD_TOL
        assert rel(s["p"], ref.states["p"], ref.states["p"].max()) < FIELD_TOL
        assert rel(s["T"], ref.states["T"], ref.states["T"].max()) < FIELD_TOL
        # the turbulent heat flux moves the energy by more than the tolerance
        assert rel(plain.q[:, 4], ref.q[:, 4], np.abs(ref.q[:, 4]).max()) > 10 * FIELD_TOL
    finally:
        ref.close()
        plain.close()
        flow.close()
