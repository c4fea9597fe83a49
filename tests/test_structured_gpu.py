"""GPU: the structured Cartesian path of the device-resident transport entries.

A uniform box in the mesh tool's canonical face ordering is detected at create;
reactive_transport_stage_device_v3 and reactive_transport_stable_step_device_v3
then run cell-stencil kernels instead of the face graph. Both SSPRK2 stages and
the CFL step must be bitwise identical to the face-graph path on the same handle
and inputs, and match the oracle within the reference validation tolerances
(tools/validate_reactive_transport.py:191-208). The boundary ledger is summed in
a different order, so it is compared within the operator tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, _lib, cases
import transport_cases as T

pytestmark = pytest.mark.gpu

H = 2e-3


def box_case(dims, ns, side_kinds, viscous=False, conduction=False, seed=0):
    faces_np, volume = cases.box_faces(dims, H, side_kinds)
    nc = volume.size
    rng = np.random.default_rng(4100 + 31 * ns + nc + seed)
    nv = ns + 4
    q = np.zeros((nc, nv))
    q[:, :ns] = rng.uniform(.002, 1, (nc, ns))
    q[:, :ns] /= q[:, :ns].sum(axis=1)[:, None]
    q[:, :ns] *= rng.uniform(.75, 1.35, (nc, 1))
    rho = q[:, :ns].sum(axis=1)
    vel = rng.normal(0, 11, (nc, 3))
    q[:, ns:ns + 3] = rho[:, None] * vel
    q[:, ns + 3] = rng.uniform(7.5e4, 1.25e5, nc) / .4 + .5 * rho * np.sum(vel ** 2, axis=1)
    n_fixed = int(np.any(faces_np["kind"] == 3))
    # a fixed (inlet) state with its own velocity: no face's wave speeds tie
    fixed_q = np.ascontiguousarray(q[:1] * 1.013)
    fixed_q[0, ns:ns + 3] += 7.0 * fixed_q[0, :ns].sum()
    fixed_states, fixed_y, fixed_h = T.ideal_states(fixed_q, ns)
    states, y, h = T.ideal_states(q, ns)
    arr = (A.Face * len(faces_np)).from_buffer_copy(faces_np.tobytes())
    cfg = A.Config(nc, ns, nv, len(faces_np), n_fixed, .007 if viscous else 0.0, 2.0 if conduction else 0.0, 0.0,
                   1.1, 2e8, 0)
    return dict(config=cfg, faces=arr, volume=volume, q=q, states=states, y=y, h=h,
                fixed_q=fixed_q if n_fixed else np.zeros((1, nv)), fixed_states=fixed_states,
                fixed_states_ptr=C.cast(T.states_ptr(fixed_states), C.c_void_p), fixed_y=fixed_y, fixed_h=fixed_h,
                ns=ns, nc=nc, nv=nv, mechanical=False)


def mixed_kinds(dims, seed):
    """Per-face boundary kinds: every side mixes slip, extrapolate and fixed state."""
    rng = np.random.default_rng(seed)
    sizes = [dims[1] * dims[2]] * 2 + [dims[0] * dims[2]] * 2 + [dims[0] * dims[1]] * 2
    return [rng.choice([1, 2, 3], size=n) for n in sizes]


BOXES = [
    dict(dims=(5, 4, 3), ns=1, kinds=(2, 2, 2, 2, 2, 2)),
    dict(dims=(6, 5, 4), ns=2, kinds=(1, 2, 3, 1, 2, 1), viscous=True, conduction=True),
    dict(dims=(4, 4, 4), ns=1, kinds="mixed", viscous=True, conduction=True, wale=.325),
    dict(dims=(7, 3, 5), ns=4, kinds="mixed", wale=.5),
    dict(dims=(9, 8, 10), ns=3, kinds=(3, 1, 1, 2, 2, 3), conduction=True, wale=.325),
]


def _stage_pair(L, h, case, stream, torch):
    """CFL step, stage 0 and stage 1 on the handle's current path."""
    nc, nv, ns = case["nc"], case["nv"], case["ns"]
    cells, fixed, nvar, nsp = (C.c_size_t() for _ in range(4))
    assert L.reactive_transport_layout_v3(h, C.byref(cells), C.byref(fixed), C.byref(nvar), C.byref(nsp)) == 0
    all_ = nc + fixed.value
    q0 = torch.zeros((nv, all_), dtype=torch.float64, device="cuda")
    q0[:, :nc] = torch.from_numpy(case["q"].T.copy()).cuda()
    st = torch.zeros((all_, 7), dtype=torch.float64, device="cuda")
    st[:nc] = torch.from_numpy(case["states"].view(np.float64).reshape(nc, 7)).cuda()
    assert L.reactive_transport_fill_fixed_v3(h, q0.data_ptr(), st.data_ptr(), stream) == 0
    dt = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.reactive_transport_stable_step_device_v3(h, q0.data_ptr(), st.data_ptr(), .23, .1, dt.data_ptr(),
                                                      stream) == 0
    torch.cuda.synchronize()
    step = .1 * dt.item()
    q1 = q0.clone()
    br0 = torch.zeros(nv, dtype=torch.float64, device="cuda")
    assert L.reactive_transport_stage_device_v3(h, q0.data_ptr(), q1.data_ptr(), st.data_ptr(), step, 0,
                                                br0.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    got1 = np.ascontiguousarray(q1[:, :nc].cpu().numpy().T)
    st1, _, _ = T.ideal_states(got1, ns)
    st[:nc] = torch.from_numpy(st1.view(np.float64).reshape(nc, 7)).cuda()
    qn = q0.clone()
    br1 = torch.zeros(nv, dtype=torch.float64, device="cuda")
    assert L.reactive_transport_stage_device_v3(h, q1.data_ptr(), qn.data_ptr(), st.data_ptr(), step, 1,
                                                br1.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    status = C.c_uint()
    assert L.reactive_transport_status_v3(h, C.byref(status), 1, stream) == 0
    return dict(dt=dt.item(), step=step, q1=got1, qn=qn[:, :nc].cpu().numpy().T, br0=br0.cpu().numpy(),
                br1=br1.cpu().numpy(), st1=st1, status=status.value, tail=bool(torch.equal(qn[:, nc:], q0[:, nc:])))


@pytest.mark.parametrize("spec", BOXES, ids=lambda s: "x".join(map(str, s["dims"])) + f"-ns{s['ns']}")
def test_structured_path_matches_face_graph_and_oracle(spec):
    import torch
    L = _lib.load()
    lib = T.bind(L)
    kinds = mixed_kinds(spec["dims"], 17) if spec["kinds"] == "mixed" else spec["kinds"]
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    cw = spec.get("wale")
    h = T.create(lib, 1, case, wale_cw=cw)
    try:
        active = C.c_int(-1)
        assert L.reactive_transport_structured_v3(h, -1, C.byref(active)) == 0
        assert active.value == 1, "canonical box not detected"
        stream = torch.cuda.current_stream().cuda_stream
        box = _stage_pair(L, h, case, stream, torch)
        assert L.reactive_transport_structured_v3(h, 0, C.byref(active)) == 0 and active.value == 0
        graph = _stage_pair(L, h, case, stream, torch)
        assert box["status"] == 0 and graph["status"] == 0
        assert box["tail"] and graph["tail"]
        # same arithmetic in the same order: bitwise identical stage results
        assert box["dt"] == graph["dt"]
        assert np.array_equal(box["q1"], graph["q1"])
        assert np.array_equal(box["qn"], graph["qn"])
        for k in ("br0", "br1"):
            assert T.scaled_error(box[k][None], graph[k][None]) <= T.RHS_TOL
        # against the oracle (itself pinned to the reference's CPU build)
        wale_cw = -1.0 if cw is None else cw
        states_p = case["states"].ctypes.data_as(C.c_void_p)
        odt = oracle.transport_stable_dt(case, case["q"], states_p, .23, .1, wale_cw=wale_cw)
        assert abs(box["dt"] / odt - 1) < T.DT_TOL
        rhs, exp_br, _, _, status = oracle.transport_rhs(case, case["q"], states_p, wale_cw=wale_cw)
        assert status == 0
        step = box["step"]
        assert T.scaled_error(box["q1"], case["q"] + step * rhs) <= T.RHS_TOL
        assert T.scaled_error(box["br0"][None], exp_br[None]) <= T.RHS_TOL
        rhs1, exp_br1, _, _, _ = oracle.transport_rhs(case, box["q1"], box["st1"].ctypes.data_as(C.c_void_p),
                                                      wale_cw=wale_cw)
        assert T.scaled_error(box["qn"], .5 * case["q"] + .5 * (box["q1"] + step * rhs1)) <= T.RHS_TOL
        assert T.scaled_error(box["br1"][None], exp_br1[None]) <= T.RHS_TOL
    finally:
        lib.reactive_transport_destroy(h)


def test_non_canonical_face_order_uses_the_face_graph():
    L = _lib.load()
    lib = T.bind(L)
    case = box_case((4, 3, 3), 1, (2, 2, 2, 2, 2, 2))
    faces = case["faces"]
    # swap two internal faces: still a valid face graph, no longer canonical
    a, b = A.Face(), A.Face()
    C.memmove(C.byref(a), C.byref(faces[3]), C.sizeof(A.Face))
    C.memmove(C.byref(b), C.byref(faces[4]), C.sizeof(A.Face))
    faces[3], faces[4] = b, a
    h = T.create(lib, 1, case)
    try:
        active = C.c_int(-1)
        assert L.reactive_transport_structured_v3(h, -1, C.byref(active)) == 0 and active.value == 0
        assert L.reactive_transport_structured_v3(h, 1, C.byref(active)) == 1
        assert b"not a structured Cartesian box" in lib.reactive_transport_error(h)
    finally:
        lib.reactive_transport_destroy(h)


@pytest.mark.parametrize("spec", BOXES, ids=lambda s: "x".join(map(str, s["dims"])) + f"-ns{s['ns']}")
def test_mixed_precision_stage_against_oracle(spec):
    """The mixed form's stage-0 rate ((q1 - q0) / dt) against the FP64 oracle:
    FP32 flux arithmetic, so a scaled error of order 1e-7 instead of 1e-12."""
    import torch
    L = _lib.load()
    lib = T.bind(L)
    kinds = mixed_kinds(spec["dims"], 17) if spec["kinds"] == "mixed" else spec["kinds"]
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    cw = spec.get("wale")
    h = T.create(lib, 1, case, wale_cw=cw)
    try:
        active = C.c_int(-1)
        assert L.reactive_transport_precision_v3(h, 1, C.byref(active)) == 0 and active.value == 1
        stream = torch.cuda.current_stream().cuda_stream
        got = _stage_pair(L, h, case, stream, torch)
        assert got["status"] == 0 and got["tail"]
        wale_cw = -1.0 if cw is None else cw
        rhs, exp_br, _, _, status = oracle.transport_rhs(case, case["q"], case["states"].ctypes.data_as(C.c_void_p),
                                                         wale_cw=wale_cw)
        assert status == 0
        rate = (got["q1"] - case["q"]) / got["step"]
        assert T.scaled_error(rate, rhs) <= 2e-5
        assert T.scaled_error(got["br0"][None], exp_br[None]) <= 2e-5
        # selecting the face graph returns to FP64
        assert L.reactive_transport_structured_v3(h, 0, None) == 0
        assert L.reactive_transport_precision_v3(h, -1, C.byref(active)) == 0 and active.value == 0
        assert L.reactive_transport_precision_v3(h, 1, None) == 1
    finally:
        lib.reactive_transport_destroy(h)


@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "mixed"])
@pytest.mark.parametrize("spec", BOXES[1:4], ids=lambda s: "x".join(map(str, s["dims"])) + f"-ns{s['ns']}")
def test_hllc_stage_against_oracle(spec, mixed):
    """HLLC on the structured path against the oracle's HLLC (itself equal to the
    reference's core bit for bit): both stages, FP64 at the reference tolerance,
    the mixed form at its FP32 tolerance."""
    import torch
    L = _lib.load()
    lib = T.bind(L)
    kinds = mixed_kinds(spec["dims"], 17) if spec["kinds"] == "mixed" else spec["kinds"]
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    cw = spec.get("wale")
    h = T.create(lib, 1, case, wale_cw=cw)
    oracle.set_flux_scheme(1)
    try:
        active = C.c_int(-1)
        assert L.reactive_transport_flux_v3(h, 1, C.byref(active)) == 0 and active.value == 1
        if mixed:
            assert L.reactive_transport_precision_v3(h, 1, None) == 0
        stream = torch.cuda.current_stream().cuda_stream
        got = _stage_pair(L, h, case, stream, torch)
        assert got["status"] == 0 and got["tail"]
        wale_cw = -1.0 if cw is None else cw
        states_p = case["states"].ctypes.data_as(C.c_void_p)
        rhs, exp_br, _, _, status = oracle.transport_rhs(case, case["q"], states_p, wale_cw=wale_cw)
        assert status == 0
        tol = 2e-5 if mixed else T.RHS_TOL
        step = got["step"]
        if mixed:
            assert T.scaled_error((got["q1"] - case["q"]) / step, rhs) <= tol
        else:
            assert T.scaled_error(got["q1"], case["q"] + step * rhs) <= tol
        assert T.scaled_error(got["br0"][None], exp_br[None]) <= tol
        rhs1, exp_br1, _, _, _ = oracle.transport_rhs(case, got["q1"], got["st1"].ctypes.data_as(C.c_void_p),
                                                      wale_cw=wale_cw)
        if not mixed:
            assert T.scaled_error(got["qn"], .5 * case["q"] + .5 * (got["q1"] + step * rhs1)) <= tol
            assert T.scaled_error(got["br1"][None], exp_br1[None]) <= tol
        # HLLC differs from HLL on these states
        oracle.set_flux_scheme(0)
        hll, _, _, _, _ = oracle.transport_rhs(case, case["q"], states_p, wale_cw=wale_cw)
        assert T.scaled_error(rhs, hll) > 1e-6
        # the face graph is HLL only
        assert L.reactive_transport_structured_v3(h, 0, None) == 0
        assert L.reactive_transport_flux_v3(h, -1, C.byref(active)) == 0 and active.value == 0
    finally:
        oracle.set_flux_scheme(0)
        lib.reactive_transport_destroy(h)


def _host_walk(lib, h, case, y=None, hh=None):
    """The host-array entries on one handle: RHS, CFL (both forms), a stage
    pair, and a resident stage pair under an attempt."""
    q, st = case["q"].copy(), case["states"]
    nv, ns = case["nv"], case["ns"]
    out = {}
    rhs, br = np.empty_like(q), np.empty(nv)
    assert lib.reactive_transport_rhs(h, T.dp(q), T.states_ptr(st), None, None, T.dp(rhs), T.dp(br)) == 0, \
        lib.reactive_transport_error(h)
    out["rhs"], out["br"] = rhs, br.copy()
    dt = C.c_double()
    assert lib.reactive_transport_stable_step(h, T.dp(q), T.states_ptr(st), .23, .1, C.byref(dt)) == 0
    out["dt"] = dt.value
    prim = T.primitives(q, st, ns)
    assert lib.reactive_transport_stable_step_primitives(h, prim, T.states_ptr(st), .23, .1, C.byref(dt)) == 0
    out["dt_prim"] = dt.value
    step = .1 * out["dt"]
    b0, b1 = np.empty(nv), np.empty(nv)
    assert lib.reactive_transport_stage(h, T.dp(q), T.states_ptr(st), None, None, step, 0, T.dp(b0)) == 0
    out["q1"] = q.copy()
    st1, _, _ = T.ideal_states(q, ns)
    assert lib.reactive_transport_stage(h, T.dp(q), T.states_ptr(st1), None, None, step, 1, T.dp(b1)) == 0
    out["qn"], out["b0"], out["b1"] = q.copy(), b0, b1
    return out


@pytest.mark.parametrize("spec", BOXES, ids=lambda s: "x".join(map(str, s["dims"])) + f"-ns{s['ns']}")
def test_host_entries_on_the_structured_box_match_the_face_graph(spec):
    """The host-array entries use the structured FP64 HLL stencils on a
    canonical box (whatever precision and flux the device entries use): RHS,
    CFL steps and stages bitwise equal to the face graph's, ledgers within the
    operator tolerance."""
    L = _lib.load()
    lib = T.bind(L)
    kinds = mixed_kinds(spec["dims"], 17) if spec["kinds"] == "mixed" else spec["kinds"]
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    cw = spec.get("wale")
    results = []
    for structured in (1, 0):
        h = T.create(lib, 1, case, wale_cw=cw)
        try:
            assert L.reactive_transport_structured_v3(h, structured, None) == 0
            if structured:  # device-entry settings do not reach the host entries
                assert L.reactive_transport_precision_v3(h, 1, None) == 0
                assert L.reactive_transport_flux_v3(h, 1, None) == 0
            results.append(_host_walk(lib, h, case))
        finally:
            lib.reactive_transport_destroy(h)
    box, graph = results
    for key in ("rhs", "q1", "qn"):
        assert np.array_equal(box[key], graph[key]), key
    assert box["dt"] == graph["dt"] and box["dt_prim"] == graph["dt_prim"]
    for key in ("br", "b0", "b1"):
        assert T.scaled_error(box[key][None], graph[key][None]) <= T.RHS_TOL


@pytest.mark.parametrize("path", ["structured-fp64", "structured-mixed", "structured-hllc", "face-graph"])
@pytest.mark.parametrize("spec", BOXES, ids=lambda s: "x".join(map(str, s["dims"])) + f"-ns{s['ns']}")
def test_cfl_stage_entry_equals_the_two_calls(spec, path):
    """reactive_transport_stage_cfl_device_v3 (the CFL query and the stage in one
    call) gives the CFL step, the staged state and the boundary ledger of
    stable_step_device_v3 followed by stage_device_v3, bit for bit, for both stages."""
    import torch
    L = _lib.load()
    lib = T.bind(L)
    kinds = mixed_kinds(spec["dims"], 17) if spec["kinds"] == "mixed" else spec["kinds"]
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    h = T.create(lib, 1, case, wale_cw=spec.get("wale"))
    try:
        if path == "face-graph":
            assert L.reactive_transport_structured_v3(h, 0, None) == 0
        elif path == "structured-mixed":
            assert L.reactive_transport_precision_v3(h, 1, None) == 0
        elif path == "structured-hllc":
            assert L.reactive_transport_flux_v3(h, 1, None) == 0
        stream = torch.cuda.current_stream().cuda_stream
        nc, nv = case["nc"], case["nv"]
        cells, fixed, nvar, nsp = (C.c_size_t() for _ in range(4))
        assert L.reactive_transport_layout_v3(h, C.byref(cells), C.byref(fixed), C.byref(nvar), C.byref(nsp)) == 0
        all_ = nc + fixed.value
        q0 = torch.zeros((nv, all_), dtype=torch.float64, device="cuda")
        q0[:, :nc] = torch.from_numpy(case["q"].T.copy()).cuda()
        st = torch.zeros((all_, 7), dtype=torch.float64, device="cuda")
        st[:nc] = torch.from_numpy(case["states"].view(np.float64).reshape(nc, 7)).cuda()
        assert L.reactive_transport_fill_fixed_v3(h, q0.data_ptr(), st.data_ptr(), stream) == 0
        dt = torch.zeros(1, dtype=torch.float64, device="cuda")
        assert L.reactive_transport_stable_step_device_v3(h, q0.data_ptr(), st.data_ptr(), .23, .1, dt.data_ptr(),
                                                          stream) == 0
        torch.cuda.synchronize()
        step = .1 * dt.item()
        for stage in (0, 1):
            outs = []
            for combined in (False, True):
                q_out = q0.clone() * 0.75  # stage 1 reads q_out as q^n
                br = torch.zeros(nv, dtype=torch.float64, device="cuda")
                d = torch.zeros(1, dtype=torch.float64, device="cuda")
                if combined:
                    rc = L.reactive_transport_stage_cfl_device_v3(h, q0.data_ptr(), q_out.data_ptr(), st.data_ptr(),
                                                                  step, stage, br.data_ptr(), .23, .1, d.data_ptr(),
                                                                  stream)
                    assert rc == 0, lib.reactive_transport_error(h)
                else:
                    assert L.reactive_transport_stable_step_device_v3(h, q0.data_ptr(), st.data_ptr(), .23, .1,
                                                                      d.data_ptr(), stream) == 0
                    assert L.reactive_transport_stage_device_v3(h, q0.data_ptr(), q_out.data_ptr(), st.data_ptr(),
                                                                step, stage, br.data_ptr(), stream) == 0
                torch.cuda.synchronize()
                outs.append((d.item(), q_out.cpu().numpy(), br.cpu().numpy()))
            (d0, qa, ba), (d1, qb, bb) = outs
            assert d0 == d1 and d0 > 0, (stage, d0, d1)
            assert np.array_equal(qa, qb), stage
            assert np.array_equal(ba, bb), stage
        status = C.c_uint()
        assert L.reactive_transport_status_v3(h, C.byref(status), 1, stream) == 0 and status.value == 0
    finally:
        lib.reactive_transport_destroy(h)


TILE_BOXES = BOXES + [
    dict(dims=(70, 9, 37), ns=1, kinds="mixed", viscous=True, conduction=True, wale=.325),
    dict(dims=(33, 6, 17), ns=2, kinds=(1, 2, 3, 1, 2, 1), viscous=True, conduction=True),
]


@pytest.mark.parametrize("path", ["fp64", "mixed", "hllc"])
@pytest.mark.parametrize("spec", TILE_BOXES, ids=lambda s: "x".join(map(str, s["dims"])) + f"-ns{s['ns']}")
def test_tiled_stage_kernel_equals_per_cell_kernel(spec, path):
    """The shared-memory tiled stage kernel (launch shape 0: each x and y face
    evaluated once per plane into shared memory, z faces carried down the
    column) and the split stage (shape 1: each interior face's flux once, then
    the per-cell sums, in mixed precision the compensated sums continued in the
    same order) give the
    per-cell kernel's stage results bit for bit: both stages, the CFL step and
    the boundary ledger, across tiles and z-chunks."""
    import torch
    L = _lib.load()
    lib = T.bind(L)
    kinds = mixed_kinds(spec["dims"], 17) if spec["kinds"] == "mixed" else spec["kinds"]
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    h = T.create(lib, 1, case, wale_cw=spec.get("wale"))
    try:
        if path == "mixed":
            assert L.reactive_transport_precision_v3(h, 1, None) == 0
        elif path == "hllc":
            assert L.reactive_transport_flux_v3(h, 1, None) == 0
        stream = torch.cuda.current_stream().cuda_stream
        runs = []
        for stage_shape in (0, 1, 128):
            shapes = (C.c_uint * 3)(stage_shape, 256, 256)
            active = (C.c_uint * 3)()
            assert L.reactive_transport_launch_shapes_v3(h, shapes, active) == 0
            assert list(active) == [stage_shape, 256, 256]
            runs.append(_stage_pair(L, h, case, stream, torch))
        per_cell = runs[-1]
        for other in runs[:-1]:
            assert other["status"] == per_cell["status"]
            assert other["dt"] == per_cell["dt"]
            assert np.array_equal(other["q1"], per_cell["q1"])
            assert np.array_equal(other["qn"], per_cell["qn"])
            assert np.array_equal(other["br0"], per_cell["br0"]) and np.array_equal(other["br1"], per_cell["br1"])
            assert other["tail"]
        assert per_cell["tail"]
        bad = (C.c_uint * 3)(32, 256, 256)
        assert L.reactive_transport_launch_shapes_v3(h, bad, None) == 1
    finally:
        lib.reactive_transport_destroy(h)


def _stage_cfl_pair(L, h, case, stream, torch):
    """Both stages through the combined CFL + stage entry (stage_cfl_device_v3)."""
    nc, nv, ns = case["nc"], case["nv"], case["ns"]
    cells, fixed, nvar, nsp = (C.c_size_t() for _ in range(4))
    assert L.reactive_transport_layout_v3(h, C.byref(cells), C.byref(fixed), C.byref(nvar), C.byref(nsp)) == 0
    all_ = nc + fixed.value
    q0 = torch.zeros((nv, all_), dtype=torch.float64, device="cuda")
    q0[:, :nc] = torch.from_numpy(case["q"].T.copy()).cuda()
    st = torch.zeros((all_, 7), dtype=torch.float64, device="cuda")
    st[:nc] = torch.from_numpy(case["states"].view(np.float64).reshape(nc, 7)).cuda()
    assert L.reactive_transport_fill_fixed_v3(h, q0.data_ptr(), st.data_ptr(), stream) == 0
    dt = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert L.reactive_transport_stable_step_device_v3(h, q0.data_ptr(), st.data_ptr(), .23, .1, dt.data_ptr(),
                                                      stream) == 0
    torch.cuda.synchronize()
    step = .1 * dt[0].item()
    q1, qn = q0.clone(), q0.clone()
    br = torch.zeros((2, nv), dtype=torch.float64, device="cuda")
    assert L.reactive_transport_stage_cfl_device_v3(h, q0.data_ptr(), q1.data_ptr(), st.data_ptr(), step, 0,
                                                    br[0].data_ptr(), .23, .1, dt[0:].data_ptr(), stream) == 0
    torch.cuda.synchronize()
    got1 = np.ascontiguousarray(q1[:, :nc].cpu().numpy().T)
    st1, _, _ = T.ideal_states(got1, ns)
    st[:nc] = torch.from_numpy(st1.view(np.float64).reshape(nc, 7)).cuda()
    assert L.reactive_transport_stage_cfl_device_v3(h, q1.data_ptr(), qn.data_ptr(), st.data_ptr(), step, 1,
                                                    br[1].data_ptr(), .23, .1, dt[1:].data_ptr(), stream) == 0
    torch.cuda.synchronize()
    status = C.c_uint()
    assert L.reactive_transport_status_v3(h, C.byref(status), 1, stream) == 0
    return dict(dt=dt.cpu().numpy(), q1=got1, qn=qn[:, :nc].cpu().numpy().T, br=br.cpu().numpy(),
                status=status.value)


@pytest.mark.parametrize("path", ["fp64", "mixed", "hllc"])
@pytest.mark.parametrize("spec", TILE_BOXES, ids=lambda s: "x".join(map(str, s["dims"])) + f"-ns{s['ns']}")
def test_split_stage_with_its_cfl_step_equals_per_cell_kernels(spec, path):
    """The combined CFL + stage entry with the split stage (launch shape 1:
    the CFL step formed from the face speeds the face pass evaluates once,
    beside the fluxes) gives the per-cell kernels' CFL steps, stages and
    boundary ledgers bit for bit, on both stages."""
    import torch
    L = _lib.load()
    lib = T.bind(L)
    kinds = mixed_kinds(spec["dims"], 17) if spec["kinds"] == "mixed" else spec["kinds"]
    case = box_case(spec["dims"], spec["ns"], kinds, spec.get("viscous", False), spec.get("conduction", False))
    h = T.create(lib, 1, case, wale_cw=spec.get("wale"))
    try:
        if path == "mixed":
            assert L.reactive_transport_precision_v3(h, 1, None) == 0
        elif path == "hllc":
            assert L.reactive_transport_flux_v3(h, 1, None) == 0
        stream = torch.cuda.current_stream().cuda_stream
        runs = []
        for stage_shape in (1, 128):
            shapes = (C.c_uint * 3)(stage_shape, 256, 256)
            assert L.reactive_transport_launch_shapes_v3(h, shapes, None) == 0
            runs.append(_stage_cfl_pair(L, h, case, stream, torch))
        split, per_cell = runs
        assert split["status"] == per_cell["status"]
        assert np.array_equal(split["dt"], per_cell["dt"]) and (split["dt"] > 0).all()
        assert np.array_equal(split["q1"], per_cell["q1"]) and np.array_equal(split["qn"], per_cell["qn"])
        assert np.array_equal(split["br"], per_cell["br"])
    finally:
        lib.reactive_transport_destroy(h)
