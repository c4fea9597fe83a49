"""CPU: WALE known answers of the reference's unit test (tools/wale_test.cpp:96-133)
on the oracle, and the oracle against the reference CPU build on WALE meshes."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A
import transport_cases as T


def direct_formula(g, delta, cw):
    g = np.asarray(g, dtype=float).reshape(3, 3)
    sq = g @ g
    s = .5 * (g + g.T)
    d = .5 * (sq + sq.T) - np.trace(sq) / 3 * np.eye(3)
    ss, dd = np.sum(s * s), np.sum(d * d)
    if dd == 0:
        return 0.0
    return cw * cw * delta * delta * dd ** 1.5 / (ss ** 2.5 + dd ** 1.25)


def test_wale_known_answers():
    assert oracle.wale_nut(np.zeros(9), .37, .5) == 0.0
    shear = np.zeros(9); shear[1] = 3.0
    assert oracle.wale_nut(shear, .37, .5) == 0.0
    g = [0.7, -1.1, 0.2, 0.4, -0.3, 0.8, -0.6, 0.1, 0.5]
    got, want = oracle.wale_nut(g, .23, .57), direct_formula(g, .23, .57)
    assert abs(got - want) <= 2e-15 * max(1.0, abs(got), abs(want))
    rot = np.zeros(9); rot[1], rot[3] = -2.0, 2.0
    assert oracle.wale_nut(rot, .37, .5) > 0.0
    # Extreme unit scales stay finite through the normalised invariants.
    big = np.array(g) * 1e200
    assert np.isfinite(oracle.wale_nut(big, 1e-3, .5))
    bad = np.array(g); bad[4] = np.nan
    assert oracle.wale_nut(bad, .37, .5) is None


@pytest.fixture(scope="module")
def ref():
    return T.bind(oracle.ref_transport_lib())


@pytest.mark.parametrize("spec", T.WALE_CASES, ids=lambda s: "-".join(map(str, s)))
def test_wale_oracle_matches_reference_cpu(ref, spec):
    ns, nc, kind, spatial, viscous, cw = spec
    case = T.make_case(ns, nc, kind, transport=False, spatial=spatial, viscous_only=viscous, seed=5)
    h = T.create(ref, 0, case, wale_cw=cw)
    try:
        q, st = case["q"], case["states"]
        rhs, br = np.empty_like(q), np.empty(case["nv"])
        assert ref.reactive_transport_rhs(h, T.dp(q), T.states_ptr(st), None, None, T.dp(rhs), T.dp(br)) == 0, \
            ref.reactive_transport_error(h)
        exp, exp_br, nut, _, status = oracle.transport_rhs(case, q, st.ctypes.data_as(C.c_void_p),
                                                           wale_cw=cw, want_nut=True)
        assert status == 0
        assert T.scaled_error(rhs, exp) <= T.RHS_TOL
        assert T.scaled_error(br[None], exp_br[None]) <= T.RHS_TOL
        got_nut = np.empty(nc)
        prim = T.primitives(q, st, ns)
        assert ref.reactive_transport_wale_primitives_v1(h, prim, T.states_ptr(st), T.dp(got_nut)) == 0
        assert np.max(np.abs(got_nut - nut) / np.maximum(np.abs(nut), 1e-300)) < 1e-12
        assert np.any(nut > 0)
        dt = C.c_double()
        assert ref.reactive_transport_stable_step(h, T.dp(q), T.states_ptr(st), .23, .1, C.byref(dt)) == 0
        odt = oracle.transport_stable_dt(case, q, st.ctypes.data_as(C.c_void_p), .23, .1, wale_cw=cw)
        assert abs(dt.value / odt - 1) < T.DT_TOL
    finally:
        ref.reactive_transport_destroy(h)
