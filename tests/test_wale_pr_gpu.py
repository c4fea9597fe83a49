"""GPU: the WALE Peng-Robinson scalar-property pass
(reactive_transport_set_wale_pr_model_v1 / wale_pr_properties_v1/v2 /
wale_pr_profile_v1) on a liquid N2O drop in air (the production model, the
capillary closure converged on its geometry), against a second handle whose
WALE scalar fields are uploaded from the host with the reference's own
property evaluation (ReactiveDeviceWalePr::evaluate compiled for the host):
the CFL step bit for bit, the RK stage within the transport tolerance; and the
reference's install, epoch and failure contract."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, _lib
from spuma_multiphysics_b200.capillary import CapillaryClosure
from spuma_multiphysics_b200.hem import GpuHem
import capillary_cases as K
import transport_cases as T

pytestmark = pytest.mark.gpu
SIGMA = 50.0
PR, SC = .9, .7
CFL_STAGE = 2 ** 64 - 1


def wale_handle(L, case, pr_image=None):
    opts = K.options(sigma=SIGMA, cfl=.5, eps=1e-10, species=2)
    h = K.Handle(L, 1, case, wale_cw=.325, wale_scalars=(PR, SC), opts=opts)
    if pr_image is not None:
        model = A.WalePrModel(1, C.sizeof(A.WalePrModel), C.cast(C.c_char_p(pr_image), C.c_void_p), len(pr_image),
                              K.MODEL_HASH, None, None)
        h.check(L.reactive_transport_set_wale_pr_model_v1(h.h, C.byref(model)))
    return h


def epoch(next_token, geometry, enthalpies, thermo=1):
    return A.WalePrEpoch(1, C.sizeof(A.WalePrEpoch), next_token, thermo, geometry, 1, enthalpies)


@pytest.fixture(scope="module")
def drop():
    """The drop after its capillary closure: q, states, color."""
    case, image, states0 = K.drop_case(10)
    L = K.bind(_lib.load())
    h = wale_handle(L, case)
    hem = GpuHem(model=image, capacity=case["nc"])
    try:
        q, states = case["q"].copy(), states0.copy()
        closure = CapillaryClosure(h.h, hem, case["ns"], SIGMA)
        closure.recover_host(q, states)
        color = closure.color.copy()
    finally:
        hem.close()
        h.close()
    return case, image, q, states, color


def geometry(h, color):
    n = len(color)
    e, k = np.zeros(n), np.zeros(n)
    h.check(h.lib.reactive_transport_capillary_geometry_v1(h.h, A.dptr(color), None, A.dptr(e), A.dptr(k), None))
    return e, k


def builds(h):
    return h.profile()["geometryBuilds"]


def test_wale_pr_properties_match_the_reference_evaluation(drop):
    case, image, q, states, color = drop
    L = K.bind(_lib.load())
    ns, nc, nv = case["ns"], case["nc"], case["nv"]
    ours, ref = wale_handle(L, case, pr_image=image), wale_handle(L, case)
    try:
        _, curvature = geometry(ours, color)
        geometry(ref, color)
        # the reference's per-cell evaluation at the published geometry
        eff, cp, status = oracle.ref_wale_pr_evaluate(image, q[:, :ns], states, color, SIGMA * curvature)
        assert (status == 0).all(), np.bincount(status)
        ref.check(L.reactive_transport_wale_scalar_fields_v1(ref.h, A.dptr(cp), A.dptr(np.ascontiguousarray(eff)),
                                                             None, None))
        # CFL outside an attempt: the state's cp
        st = T.ideal_states(q, ns)[0]   # transport states: the ideal closure's fields are not what is tested
        st["p"], st["T"], st["rho"], st["cv"] = states["p"], states["T"], states["rho"], states["cv"]
        st["sound"], st["gasMass"] = states["soundFrozen"], states["gasMass"]
        ours.check(L.reactive_transport_wale_pr_properties_v1(ours.h, C.byref(epoch(A.Token(0, 0, 0), builds(ours), 0)),
                                                              None, 0, states.ctypes.data_as(C.c_void_p)))
        assert ours.stable_step(q, st) == ref.stable_step(q, st)
        # an RK stage: properties for the exact next conserved input
        out = {}
        for name, h in (("ours", ours), ("ref", ref)):
            qq = q.copy()
            h.check(L.reactive_transport_begin_attempt(h.h, K.MODEL_HASH, 1))
            if name == "ours":
                h.check(L.reactive_transport_wale_pr_properties_v2(
                    h.h, C.byref(epoch(A.Token(1, 0, 5), builds(h), 1, thermo=2)), A.dptr(qq), nv,
                    states.ctypes.data_as(C.c_void_p), 1))
            h.check(L.reactive_transport_upload_conserved(h.h, A.dptr(qq), 5))
            br = np.zeros(nv)
            h.check(L.reactive_transport_advance_resident_v2(h.h, A.Token(1, 0, 5), A.Token(1, 1, 6),
                                                             T.states_ptr(st), None, None, None, 1e-9, A.dptr(br)))
            h.check(L.reactive_transport_download_conserved(h.h, A.Token(1, 1, 6), A.dptr(qq)))
            out[name] = (qq, br)
            if name == "ours":
                # the next stage needs properties of its own input
                br2 = np.zeros(nv)
                assert L.reactive_transport_advance_resident_v2(h.h, A.Token(1, 1, 6), A.Token(1, 2, 7),
                                                                T.states_ptr(st), None, None, None, 1e-9,
                                                                A.dptr(br2)) == 1
                assert b"stale conserved or geometry epoch" in L.reactive_transport_error(h.h)
        assert T.scaled_error(out["ours"][0], out["ref"][0]) <= T.RHS_TOL
        assert T.scaled_error(out["ours"][1][None], out["ref"][1][None]) <= T.RHS_TOL
        prof = A.WalePrProfile(1, C.sizeof(A.WalePrProfile))
        ours.check(L.reactive_transport_wale_pr_profile_v1(ours.h, C.byref(prof)))
        assert prof.builds == 2 and prof.cells == 2 * nc and prof.failures == 0 and prof.kernels == 4
        # the v2 reuse skipped one state upload
        assert prof.inputUploadBytes > 0
    finally:
        ours.close()
        ref.close()


def test_wale_pr_contract(drop):
    case, image, q, states, color = drop
    L = K.bind(_lib.load())
    ns, nv = case["ns"], case["nv"]
    h = wale_handle(L, case)
    try:
        bad = A.WalePrModel(1, C.sizeof(A.WalePrModel), C.cast(C.c_char_p(image), C.c_void_p), len(image),
                            b"b" * 64, None, None)
        assert L.reactive_transport_set_wale_pr_model_v1(h.h, C.byref(bad)) == 1
        assert b"identity differs" in L.reactive_transport_error(h.h)
    finally:
        h.close()
    h = wale_handle(L, case, pr_image=image)
    try:
        model = A.WalePrModel(1, C.sizeof(A.WalePrModel), C.cast(C.c_char_p(image), C.c_void_p), len(image),
                              K.MODEL_HASH, None, None)
        assert L.reactive_transport_set_wale_pr_model_v1(h.h, C.byref(model)) == 1
        assert b"installed on CUDA before stepping" in L.reactive_transport_error(h.h)
        cp = np.full(case["nc"], 1000.0)
        assert L.reactive_transport_wale_scalar_fields_v1(h.h, A.dptr(cp), None, None, None) == 1
        assert b"cannot replace installed PR device properties" in L.reactive_transport_error(h.h)
        sp = states.ctypes.data_as(C.c_void_p)
        # no geometry yet
        assert L.reactive_transport_wale_pr_properties_v1(h.h, C.byref(epoch(A.Token(0, 0, 0), 0, 0)), None, 0,
                                                          sp) == 1
        assert b"current capillary geometry" in L.reactive_transport_error(h.h)
        geometry(h, color)
        g = builds(h)
        cases_ = [(epoch(A.Token(0, 0, 0), g + 1, 0), b"current capillary geometry"),
                  (epoch(A.Token(1, 0, 3), g, 0), b"cannot claim an RK token"),
                  (epoch(A.Token(0, 0, 0), g, 1), b"require an open RK attempt"),
                  (A.WalePrEpoch(1, C.sizeof(A.WalePrEpoch), A.Token(0, 0, 0), 0, g, 1, 0), b"Invalid WALE PR property epoch")]
        for e, msg in cases_:
            assert L.reactive_transport_wale_pr_properties_v1(h.h, C.byref(e), A.dptr(q), nv, sp) == 1
            assert msg in L.reactive_transport_error(h.h), (msg, L.reactive_transport_error(h.h))
        # a state that does not match its phases fails the call and publishes nothing
        broken = states.copy()
        broken["rho"][17] *= 1.001
        assert L.reactive_transport_wale_pr_properties_v1(h.h, C.byref(epoch(A.Token(0, 0, 0), g, 0, thermo=3)),
                                                          None, 0, broken.ctypes.data_as(C.c_void_p)) == 0  # cp only
        h.check(L.reactive_transport_begin_attempt(h.h, K.MODEL_HASH, 1))
        assert L.reactive_transport_wale_pr_properties_v1(
            h.h, C.byref(epoch(A.Token(1, 0, 5), g, 1, thermo=3)), A.dptr(q), nv,
            broken.ctypes.data_as(C.c_void_p)) == 1
        assert b"WALE PR GPU property cell 17 status 7" in L.reactive_transport_error(h.h)
        prof = A.WalePrProfile(1, C.sizeof(A.WalePrProfile))
        h.check(L.reactive_transport_wale_pr_profile_v1(h.h, C.byref(prof)))
        assert prof.failures == 1 and prof.builds == 1
        # thermo versions never decrease
        assert L.reactive_transport_wale_pr_properties_v1(
            h.h, C.byref(epoch(A.Token(1, 2 ** 64 - 1, 0), g, 0, thermo=2)), None, 0, sp) == 1
        assert b"Invalid WALE PR property epoch" in L.reactive_transport_error(h.h)
        # a new geometry retires the properties: the CFL query refuses them
        h.check(L.reactive_transport_wale_pr_properties_v1(
            h.h, C.byref(epoch(A.Token(1, CFL_STAGE, 0), g, 0, thermo=4)), None, 0, sp))
        geometry(h, color * .999)
        st = T.ideal_states(q, ns)[0]
        with pytest.raises(RuntimeError, match="heat capacities were not uploaded"):
            h.stable_step(q, st)
    finally:
        h.close()
