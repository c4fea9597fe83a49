"""GPU: the resident capillary closure (reactive_transport_capillary_resident_*_v1
with reactive_gpu_hem_run_resident_v1 on its device view).

* The reference's resident-buffer contract, restated from its own validation
  (tools/validate_capillary_resident.py): on a 35-cell periodic line (a partial
  warp) with 1, 5 and 16 species and controlled flash outputs, the full dirty
  set at iteration 0 is a permutation of the cells, heavy-first by active
  liquids; publishing the seeds' own states leaves a zero residual and an empty
  dirty set; the committed geometry equals the host geometry entry's bit for
  bit and a later identical host request reuses it; a changed species count is
  refused; a workspace budget failure leaves the handle's memory unchanged and
  can be retried.
* The closure itself: a liquid N2O drop in air and N2O vapour (the production
  model) with a large surface tension, in equilibrium and with the frozen
  partition: the resident path gives the host path's states, color, surface
  energy and curvature bit for bit (the host path runs the capillary HEM
  batches that match the reference's recoverCapillary, and the geometry entry
  that matches the reference's CPU build). Out-of-order calls fail.
"""
import ctypes as C

import numpy as np
import pytest

from spuma_multiphysics_b200 import _abi as A, _lib
from spuma_multiphysics_b200.capillary import CapillaryClosure
from spuma_multiphysics_b200.hem import GpuHem
import capillary_cases as K
import transport_cases as T

pytestmark = pytest.mark.gpu


def _runtime():
    from cuda.bindings import runtime
    return runtime


def memcpy_to_device(dst, src_bytes):
    cudart = _runtime()
    err, = cudart.cudaMemcpy(dst, src_bytes, len(src_bytes), cudart.cudaMemcpyKind.cudaMemcpyHostToDevice)
    assert int(err) == 0


def memcpy_to_host(src, nbytes):
    cudart = _runtime()
    out = bytearray(nbytes)
    err, = cudart.cudaMemcpy(out, src, nbytes, cudart.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0
    return bytes(out)


def line_handle(L, n, ns, limit=1e8):
    faces = (A.Face * n)(*[A.Face(c, (c + 1) % n, -1, (C.c_double * 3)(1, 0, 0), 1, 1, .5, 0) for c in range(n)])
    cfg = A.Config(n, ns, ns + 5, n, 0, 0, 0, 0, 1.1, limit, 0)
    err = C.create_string_buffer(2048)
    h = L.reactive_transport_create(1, C.byref(cfg), A.dptr(np.ones(n)), faces, None, None, None, None, err,
                                    len(err))
    assert h, err.value.decode()
    h = C.c_void_p(h)
    assert L.reactive_transport_set_capillary_v1(h, C.byref(K.options(sigma=.01, cfl=.25, species=0))) == 0
    return h


def allocated(L, h):
    s = A.Stats()
    assert L.reactive_transport_stats(h, C.byref(s)) == 0
    return s.allocatedBytes


@pytest.mark.parametrize("ns", [1, 5, 16])
def test_resident_buffer_contract(ns):
    L = _lib.load()
    n = 35
    t, ref = line_handle(L, n, ns), line_handle(L, n, ns)
    fallback = C.c_int()
    try:
        base = allocated(L, t)
        color = np.linspace(.1, .8, n)
        masses = np.zeros((n, ns))
        state = np.zeros(n, dtype=A.THERMO_DTYPE)
        for c in range(n):
            masses[c, 0] = 1
            masses[c, c % ns] += 2
        state["rho"], state["p"], state["T"] = 1, 1e5, 290
        state["liquidMass"][:, 0] = color
        state["rhoLiquid"][:, 0] = 1
        state["gasMass"], state["rhoGas"] = 1 - color, 1
        state["activeLiquids"] = np.arange(n) % 2
        original = state.tobytes()
        liquid, bulk = color.copy(), np.full(n, 1e6)

        def begin(species=ns):
            return L.reactive_transport_capillary_resident_begin_v1(
                t, species, A.dptr(masses), A.dptr(liquid), A.dptr(bulk), state.ctypes.data_as(C.c_void_p), None,
                .01, 1, C.byref(fallback))
        assert begin() == 0 and fallback.value == 0 and state.tobytes() == original
        view = A.CapillaryResidentView(1, C.sizeof(A.CapillaryResidentView))
        assert L.reactive_transport_capillary_resident_select_v1(t, 0, C.byref(view), C.byref(fallback)) == 0
        assert fallback.value == 0 and view.count == n
        order = np.frombuffer(memcpy_to_host(view.order, 4 * n), dtype=np.uint32)
        assert sorted(order.tolist()) == list(range(n))
        active = state["activeLiquids"][order]
        assert (np.diff(active) <= 0).all()     # heavy first
        if ns > 1:
            assert len({int(np.argmax(masses[c])) for c in order}) > 1
        # publish controlled successful outputs: the seeds' own states
        outputs = np.zeros(n, dtype=A.HEM_OUTPUT_DTYPE)
        outputs["state"] = state
        outputs["success"] = 1
        memcpy_to_device(view.output, outputs.tobytes())
        residual = C.c_double()
        assert L.reactive_transport_capillary_resident_update_v1(t, n, C.byref(residual), C.byref(fallback)) == 0
        assert fallback.value == 0 and residual.value == 0
        assert L.reactive_transport_capillary_resident_select_v1(t, 1, C.byref(view), C.byref(fallback)) == 0
        assert view.count == 0
        assert L.reactive_transport_capillary_resident_update_v1(t, 0, C.byref(residual), C.byref(fallback)) == 0
        assert residual.value == 0 and fallback.value == 0
        got = np.zeros(n, dtype=A.THERMO_DTYPE)
        gc, ge, gk, re, rk = (np.zeros(n) for _ in range(5))
        assert L.reactive_transport_capillary_resident_commit_v1(t, got.ctypes.data_as(C.c_void_p), A.dptr(gc),
                                                                 A.dptr(ge), A.dptr(gk)) == 0
        assert L.reactive_transport_capillary_geometry_v1(ref, A.dptr(color), None, A.dptr(re), A.dptr(rk), None) == 0
        assert got.tobytes() == original and gc.tobytes() == color.tobytes()
        assert ge.tobytes() == re.tobytes() and gk.tobytes() == rk.tobytes()
        # the next ordinary request sees the geometry just published, without device work
        prof0 = A.CapillaryProfile(1, C.sizeof(A.CapillaryProfile))
        assert L.reactive_transport_capillary_profile_v1(t, C.byref(prof0)) == 0
        ce, ck = np.zeros(n), np.zeros(n)
        assert L.reactive_transport_capillary_geometry_v1(t, A.dptr(color), None, A.dptr(ce), A.dptr(ck), None) == 0
        prof1 = A.CapillaryProfile(1, C.sizeof(A.CapillaryProfile))
        assert L.reactive_transport_capillary_profile_v1(t, C.byref(prof1)) == 0
        assert ce.tobytes() == ge.tobytes() and ck.tobytes() == gk.tobytes()
        assert prof1.geometryBuilds == prof0.geometryBuilds
        assert begin(ns + 1) != 0
        # out of order after a refusal: select needs a successful begin
        assert L.reactive_transport_capillary_resident_select_v1(t, 0, C.byref(view), C.byref(fallback)) != 0
        assert b"out of order" in L.reactive_transport_error(t)
        assert base > 0
    finally:
        L.reactive_transport_destroy(t)
        L.reactive_transport_destroy(ref)
    # a budget that admits the handle but not the whole workspace: the call fails
    # and leaves the memory as it was, twice in a row
    probe = line_handle(L, n, ns)
    base = allocated(L, probe)
    L.reactive_transport_destroy(probe)
    t = line_handle(L, n, ns, limit=base + n * (ns + 1) * 8 + 1)
    try:
        before = allocated(L, t)
        for _ in range(2):
            rc = L.reactive_transport_capillary_resident_begin_v1(
                t, ns, A.dptr(masses), A.dptr(liquid), A.dptr(bulk), state.ctypes.data_as(C.c_void_p), None, .01, 1,
                C.byref(fallback))
            assert rc != 0 and b"workspace budget" in L.reactive_transport_error(t)
            assert allocated(L, t) == before
    finally:
        L.reactive_transport_destroy(t)


def test_resident_entries_refuse_without_the_capillary_model():
    L = _lib.load()
    lib = T.bind(L)
    case = T.make_case(4, 9, 0, frozen=1)
    h = T.create(lib, 1, case)
    try:
        fallback = C.c_int()
        q = np.zeros((9, 4))
        z = np.zeros(9)
        st = np.zeros(9, dtype=A.THERMO_DTYPE)
        assert L.reactive_transport_capillary_resident_begin_v1(h, 4, A.dptr(q), A.dptr(z), A.dptr(z),
                                                                st.ctypes.data_as(C.c_void_p), None, .01, 1,
                                                                C.byref(fallback)) == 1
        assert b"needs CUDA diffuse geometry" in L.reactive_transport_error(h)
        view = A.CapillaryResidentView(1, C.sizeof(A.CapillaryResidentView))
        assert L.reactive_transport_capillary_resident_select_v1(h, 0, C.byref(view), C.byref(fallback)) == 1
        assert L.reactive_transport_capillary_resident_relax_v1(h) == 1
        assert b"out of order" in L.reactive_transport_error(h)
    finally:
        lib.reactive_transport_destroy(h)


@pytest.mark.parametrize("frozen", [False, True])
def test_resident_closure_equals_host_closure(frozen):
    case, image, states0 = K.drop_case(10)
    sigma = 50.0
    L = K.bind(_lib.load())
    paths = {}
    for path in ("host", "resident"):
        opts = K.options(sigma=sigma, cfl=.5, eps=1e-10, species=2)
        h = K.Handle(L, 1, case, opts=opts)
        hem = GpuHem(model=image, capacity=case["nc"], resident=path == "resident")
        try:
            q, states = case["q"].copy(), states0.copy()
            closure = CapillaryClosure(h.h, hem, case["ns"], sigma, frozen=frozen)
            if path == "host":
                closure.recover_host(q, states)
            else:
                assert closure.recover_resident(q, states)
            paths[path] = (q, states, closure.color.copy(), closure.surface_energy.copy(), closure.curvature.copy(),
                           closure.iterations, closure.residual)
        finally:
            hem.close()
            h.close()
    hq, hs, hc, he, hk, hit, hres = paths["host"]
    rq, rs, rc, re, rk, rit, rres = paths["resident"]
    assert hit == rit and hit >= 2, (hit, rit)
    assert hres == rres and hres <= 1e-9
    assert rs.tobytes() == hs.tobytes()
    assert rc.tobytes() == hc.tobytes() and re.tobytes() == he.tobytes() and rk.tobytes() == hk.tobytes()
    assert rq.tobytes() == hq.tobytes()
    # the interface moved the cells' pressures: the jump reached the flash
    assert np.max(np.abs(hs["p"] - states0["p"]) / states0["p"]) > 1e-6
    assert np.max(np.abs(hk)) > 0
