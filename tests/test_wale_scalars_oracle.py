"""CPU: the WALE scalar closure (turbulent Prandtl heat flux and turbulent
Schmidt species mixing, src/reactiveTransport/reactiveTransport.cpp:653-702 and
reactiveTransportKernels.h:150-168, :323-336, :440-477) in the oracle against
the reference CPU build, and the reference's install/upload contract."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A
import transport_cases as T

# (WALE case, Prandtl, Schmidt)
SCALAR_CASES = [(c, pr, sc) for c in T.WALE_CASES for pr, sc in ((.9, .7), (.85, 0.0), (0.0, .6))]


@pytest.fixture(scope="module")
def ref():
    return T.bind(oracle.ref_transport_lib())


def oracle_rhs_dt(case, q, st, cw, pr, sc, fields):
    oracle.set_wale_scalars(pr, sc, **fields)
    try:
        rhs, br, _, _, status = oracle.transport_rhs(case, q, st.ctypes.data_as(C.c_void_p), wale_cw=cw)
        dt = oracle.transport_stable_dt(case, q, st.ctypes.data_as(C.c_void_p), .23, .1, wale_cw=cw)
    finally:
        oracle.set_wale_scalars()
    return rhs, br, status, dt


@pytest.mark.parametrize("spec,pr,sc", SCALAR_CASES, ids=lambda s: "-".join(map(str, s)) if isinstance(s, tuple)
                         else str(s))
def test_wale_scalars_oracle_matches_reference_cpu(ref, spec, pr, sc):
    ns, nc, kind, spatial, viscous, cw = spec
    case = T.make_case(ns, nc, kind, transport=False, spatial=spatial, viscous_only=viscous, seed=5)
    fields = T.scalar_fields(case, seed=nc)
    h = T.create(ref, 0, case, wale_cw=cw, wale_scalars=(pr, sc))
    try:
        q, st = case["q"], case["states"]
        assert T.upload_scalar_fields(ref, h, fields) == 0, ref.reactive_transport_error(h)
        rhs, br = np.empty_like(q), np.empty(case["nv"])
        assert ref.reactive_transport_rhs(h, T.dp(q), T.states_ptr(st), None, None, T.dp(rhs), T.dp(br)) == 0, \
            ref.reactive_transport_error(h)
        dt = C.c_double()
        assert ref.reactive_transport_stable_step(h, T.dp(q), T.states_ptr(st), .23, .1, C.byref(dt)) == 0
        exp, exp_br, status, odt = oracle_rhs_dt(case, q, st, cw, pr, sc, fields)
        assert status == 0
        assert T.scaled_error(rhs, exp) <= T.RHS_TOL
        assert T.scaled_error(br[None], exp_br[None]) <= T.RHS_TOL
        assert abs(dt.value / odt - 1) < T.DT_TOL
        # the closure changes the operator and the step (the fluxes are not trivially zero)
        plain, _, _, pdt = oracle_rhs_dt(case, q, st, cw, 0, 0, fields)
        if kind != 1 or nc > 1:
            assert T.scaled_error(plain, exp) > 1e-9 or (ns == 1 and pr == 0)
        assert pdt >= odt
        prof = A.WaleScalarProfile(1, C.sizeof(A.WaleScalarProfile))
        assert ref.reactive_transport_wale_scalar_profile_v1(h, C.byref(prof)) == 0
        assert prof.fieldUploads == 1
        all_ = nc + case["config"].fixed
        assert prof.workspaceBytes == (all_ * 8 if pr > 0 else 0) + (all_ * ns * 8 if sc > 0 else 0)
    finally:
        ref.reactive_transport_destroy(h)


def test_wale_scalar_contract_on_reference_cpu(ref):
    """Install preconditions, field validation and the stage/CFL preconditions
    (reactiveTransport.cpp:653-702, :1395-1397, :1415-1416)."""
    T.wale_scalar_contract(ref, 0)
