"""GPU parity of the CUDA transport (libreactive_b200.so, backend 1) through the
reference C ABI: the full RHS / CFL / RK-stage / residency contract on every
validation case, WALE meshes, and the device-resident *_v3 entry points, all
against the CPU oracle (itself pinned to the reference's CPU build)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, _lib
import transport_cases as T

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return T.bind(_lib.load())


@pytest.mark.parametrize("spec", T.CASES, ids=lambda s: "-".join(map(str, s)))
def test_cuda_transport_contract(lib, spec):
    case = T.case_from_tuple(spec)
    summary = T.contract_walk(lib, 1, case, oracle)
    assert summary["rhs_error"] <= T.RHS_TOL


@pytest.mark.parametrize("nc", [65535, 65536, 65537])
def test_cuda_large_cfl(lib, nc):
    T.large_cfl_walk(lib, 1, nc)


def test_backend_zero_is_rejected(lib):
    case = T.case_from_tuple(T.CASES[0])
    with pytest.raises(RuntimeError, match="CUDA only"):
        T.create(lib, 0, case)


@pytest.mark.parametrize("spec", T.WALE_CASES, ids=lambda s: "-".join(map(str, s)))
def test_cuda_wale(lib, spec):
    ns, nc, kind, spatial, viscous, cw = spec
    case = T.make_case(ns, nc, kind, transport=False, spatial=spatial, viscous_only=viscous, seed=5)
    h = T.create(lib, 1, case, wale_cw=cw)
    try:
        q, st = case["q"], case["states"]
        rhs, br = np.empty_like(q), np.empty(case["nv"])
        assert lib.reactive_transport_rhs(h, T.dp(q), T.states_ptr(st), None, None, T.dp(rhs), T.dp(br)) == 0, \
            lib.reactive_transport_error(h)
        exp, exp_br, nut, _, status = oracle.transport_rhs(case, q, st.ctypes.data_as(C.c_void_p),
                                                           wale_cw=cw, want_nut=True)
        assert status == 0
        assert T.scaled_error(rhs, exp) <= T.RHS_TOL
        assert T.scaled_error(br[None], exp_br[None]) <= T.RHS_TOL
        got = np.empty(nc)
        prim = T.primitives(q, st, ns)
        assert lib.reactive_transport_wale_primitives_v1(h, prim, T.states_ptr(st), T.dp(got)) == 0
        assert np.max(np.abs(got - nut) / np.maximum(np.abs(nut), 1e-300)) < 1e-12
        dt = C.c_double()
        assert lib.reactive_transport_stable_step(h, T.dp(q), T.states_ptr(st), .23, .1, C.byref(dt)) == 0
        odt = oracle.transport_stable_dt(case, q, st.ctypes.data_as(C.c_void_p), .23, .1, wale_cw=cw)
        assert abs(dt.value / odt - 1) < T.DT_TOL
    finally:
        lib.reactive_transport_destroy(h)


V3_CASES = [dict(ns=4, nc=7, kind=3, viscous_only=True, conduction=True),
            dict(ns=1, nc=64, kind=2, spatial=True, viscous_only=True, conduction=True),
            dict(ns=2, nc=33, kind=1, spatial=True, extra_boundary=40, viscous_only=True, wale=.325),
            dict(ns=1, nc=40, kind=3, spatial=True, conduction=True, wale=.325)]


@pytest.mark.parametrize("spec", V3_CASES, ids=lambda s: "-".join(f"{k}{v}" for k, v in s.items()))
def test_cuda_device_resident_v3(lib, spec):
    """Both SSPRK2 stages and the CFL step on device pointers against the oracle."""
    import torch
    L = _lib.load()
    spec = dict(spec)
    cw = spec.pop("wale", None)
    case = T.make_case(**spec)
    ns, nc, nv = case["ns"], case["nc"], case["nv"]
    h = T.create(lib, 1, case, wale_cw=cw)
    wale_cw = -1.0 if cw is None else cw
    try:
        cells, fixed, nvar, nsp = (C.c_size_t() for _ in range(4))
        assert L.reactive_transport_layout_v3(h, C.byref(cells), C.byref(fixed), C.byref(nvar), C.byref(nsp)) == 0
        assert (cells.value, nvar.value, nsp.value) == (nc, nv, ns)
        all_ = nc + fixed.value
        stream = torch.cuda.current_stream().cuda_stream
        q0 = torch.zeros((nv, all_), dtype=torch.float64, device="cuda")
        q0[:, :nc] = torch.from_numpy(case["q"].T.copy()).cuda()
        st = torch.zeros((all_, 7), dtype=torch.float64, device="cuda")
        st[:nc] = torch.from_numpy(case["states"].view(np.float64).reshape(nc, 7)).cuda()
        assert L.reactive_transport_fill_fixed_v3(h, q0.data_ptr(), st.data_ptr(), stream) == 0
        q1 = q0.clone()
        br = torch.zeros(nv, dtype=torch.float64, device="cuda")
        dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
        assert L.reactive_transport_stable_step_device_v3(h, q0.data_ptr(), st.data_ptr(), .23, .1,
                                                          dt_dev.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        odt = oracle.transport_stable_dt(case, case["q"], case["states"].ctypes.data_as(C.c_void_p), .23, .1,
                                         wale_cw=wale_cw)
        assert abs(dt_dev.item() / odt - 1) < T.DT_TOL
        step = .1 * odt
        assert L.reactive_transport_stage_device_v3(h, q0.data_ptr(), q1.data_ptr(), st.data_ptr(), step, 0,
                                                    br.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        rhs, exp_br, _, _, _ = oracle.transport_rhs(case, case["q"], case["states"].ctypes.data_as(C.c_void_p),
                                                    case["y"], case["h"], wale_cw=wale_cw)
        got1 = q1[:, :nc].cpu().numpy().T
        assert T.scaled_error(got1, case["q"] + step * rhs) <= T.RHS_TOL
        assert T.scaled_error(br.cpu().numpy()[None], exp_br[None]) <= T.RHS_TOL
        st1, y1, h1 = T.ideal_states(np.ascontiguousarray(got1), ns, case["mechanical"])
        st[:nc] = torch.from_numpy(st1.view(np.float64).reshape(nc, 7)).cuda()
        qn = q0.clone()
        assert L.reactive_transport_stage_device_v3(h, q1.data_ptr(), qn.data_ptr(), st.data_ptr(), step, 1, 0,
                                                    stream) == 0
        torch.cuda.synchronize()
        rhs1, _, _, _, _ = oracle.transport_rhs(case, np.ascontiguousarray(got1), st1.ctypes.data_as(C.c_void_p),
                                                y1, h1, wale_cw=wale_cw)
        assert T.scaled_error(qn[:, :nc].cpu().numpy().T, .5 * case["q"] + .5 * (got1 + step * rhs1)) <= T.RHS_TOL
        assert torch.equal(qn[:, nc:], q0[:, nc:])
        # a diffusive configuration is rejected on the device path
    finally:
        lib.reactive_transport_destroy(h)
