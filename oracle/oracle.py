"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracles and to the
reference's own CPU builds in oracle/_ref/. Imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the product.
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"
# the reference checkout (its sources feed the _ref/ builds and the fixture
# scripts): $REFERENCE, by default the directory `reference` beside this repository
REFERENCE = Path(os.environ.get("REFERENCE", HERE.parent.parent / "reference"))
ORACLE_LIB = HERE / "liboracle.so"
REF_TRANSPORT = REF / "libreactiveTransport_ref.so"
REF_FLASH = REF / "libref_flash.so"

_d = C.POINTER(C.c_double)
_v = C.c_void_p


def build():
    """Compile liboracle.so and, when the reference sources are present, _ref/."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def _load(path):
    if not path.exists():
        build()
    return C.CDLL(str(path))


_oracle = None
_ref_transport = None
_ref_flash = None
_ref_hllc = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = _load(ORACLE_LIB)
        _oracle.oracle_transport_rhs.argtypes = [_v, _d, _v, _d, _v, _d, _d, C.c_double, _d, _v, _d, _d,
                                                 _d, _d, _d, _d]
        _oracle.oracle_transport_rhs.restype = C.c_int
        _oracle.oracle_transport_stable_dt.argtypes = [_v, _d, _v, _d, _v, C.c_double, _d, _v, C.c_double,
                                                       C.c_double]
        _oracle.oracle_transport_stable_dt.restype = C.c_double
        _oracle.oracle_wale_nut.argtypes = [_d, C.c_double, C.c_double, _d]
        _oracle.oracle_wale_nut.restype = C.c_int
        _oracle.oracle_set_wale_scalars.argtypes = [C.c_double, C.c_double, _d, _d, _d, _d]
        _oracle.oracle_set_wale_scalars.restype = None
        _oracle.oracle_set_flux_scheme.argtypes = [C.c_int]
        _oracle.oracle_set_flux_scheme.restype = None
        _oracle.oracle_hllc_face.argtypes = [C.c_double, _d, C.c_double, C.c_double, C.c_double, C.c_double, _d,
                                             C.c_double, C.c_double, C.c_double, _d, _d]
        _oracle.oracle_hllc_face.restype = C.c_int
        if hasattr(_oracle, "oracle_flash_recover"):
            _oracle.oracle_flash_recover.argtypes = [C.c_char_p, C.c_size_t, _d, _d, _v, _v, C.POINTER(C.c_int),
                                                     C.POINTER(C.c_uint64), C.c_int]
            _oracle.oracle_flash_recover.restype = C.c_int
    return _oracle


def ref_transport_lib():
    """The reference's transport compiled for CPU (backend 0, serial)."""
    global _ref_transport
    if _ref_transport is None:
        if not REF_TRANSPORT.exists():
            build()
        _ref_transport = C.CDLL(str(REF_TRANSPORT))
    return _ref_transport


def ref_hllc_lib():
    """The reference's HLLC face core compiled for the host."""
    global _ref_hllc
    if _ref_hllc is None:
        path = HERE / "_ref" / "libref_hllc.so"
        if not path.exists():
            build()
        _ref_hllc = C.CDLL(str(path))
        _ref_hllc.ref_hllc_face.argtypes = [C.c_double, _d, C.c_double, C.c_double, C.c_double, C.c_double, _d,
                                            C.c_double, C.c_double, C.c_double, _d, _d]
        _ref_hllc.ref_hllc_face.restype = C.c_int
    return _ref_hllc


def hllc_face(lib_fn, L, R, normal):
    """(ok, [contact, advectLeft, advectRight, pressureMomentum, pressureEnergy]) of one face;
    L, R = (rho, u[3], p, a, E)."""
    out = np.zeros(5)
    a = lambda x: np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(_d)
    ok = lib_fn(L[0], a(L[1]), L[2], L[3], L[4], R[0], a(R[1]), R[2], R[3], R[4], a(normal), out.ctypes.data_as(_d))
    return ok, out


_scalar_fields = None


def set_wale_scalars(pr=0.0, sc=0.0, cell_cp=None, fixed_cp=None, cell_h=None, fixed_h=None):
    """WALE scalar closure of transport_rhs / transport_stable_dt (0 disables a
    flux; the arrays are held here while the closure is set)."""
    global _scalar_fields
    arrays = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
              for a in (cell_cp, fixed_cp, cell_h, fixed_h)]
    _scalar_fields = arrays
    oracle_lib().oracle_set_wale_scalars(float(pr), float(sc), *[_p(a) for a in arrays])


def set_flux_scheme(scheme):
    """Flux scheme of transport_rhs / transport_stable_dt: 0 HLL, 1 HLLC."""
    oracle_lib().oracle_set_flux_scheme(int(scheme))


def ref_flash_lib():
    """The reference's device flash compiled for the host."""
    global _ref_flash
    if _ref_flash is None:
        if not REF_FLASH.exists():
            build()
        lib = C.CDLL(str(REF_FLASH))
        lib.ref_flash_recover.argtypes = [C.c_char_p, C.c_size_t, _d, _d, _v, _v, C.POINTER(C.c_int),
                                          C.POINTER(C.c_uint64), C.c_int, C.c_int]
        lib.ref_flash_recover.restype = C.c_int
        lib.ref_flash_recover_capillary.argtypes = [C.c_char_p, C.c_size_t, _d, _d, _v, _d, _d,
                                                    C.POINTER(C.c_int), _v, C.POINTER(C.c_int),
                                                    C.POINTER(C.c_int), C.POINTER(C.c_uint64), C.c_int]
        lib.ref_flash_recover_capillary.restype = C.c_int
        lib.ref_flash_initialize_tp.argtypes = [C.c_char_p, C.c_size_t, _d, _d, _v, _d, _d, _v,
                                                C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.ref_flash_initialize_tp.restype = C.c_int
        lib.ref_wale_pr_evaluate.argtypes = [C.c_char_p, C.c_size_t, _d, _v, _d, _d, C.c_int, _d, _d,
                                             C.POINTER(C.c_int)]
        lib.ref_wale_pr_evaluate.restype = C.c_int
        lib.ref_pr_evaluate_tp.argtypes = [C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _d,
                                           C.POINTER(C.c_int)]
        lib.ref_pr_evaluate_trho.argtypes = [C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_int, _d,
                                             C.POINTER(C.c_int)]
        _ref_flash = lib
    return _ref_flash


def _p(a):
    return None if a is None else a.ctypes.data_as(_d)


def transport_rhs(case, q, states, gy=None, gh=None, wale_cw=-1.0, want_nut=False, want_denominator=False):
    """Oracle RHS (cell-major), boundary ledger, nu_t, CFL denominators, status."""
    cfg = case["config"]
    nc, nv = cfg.cells, cfg.variables
    rhs = np.zeros((nc, nv))
    boundary = np.zeros(nv)
    nut = np.zeros(nc) if want_nut else None
    den = np.zeros(nc) if want_denominator else None
    status = oracle_lib().oracle_transport_rhs(
        C.byref(cfg), _p(case["volume"]), case["faces"], _p(case["fixed_q"]), case["fixed_states_ptr"],
        _p(case.get("fixed_y")), _p(case.get("fixed_h")), wale_cw, _p(np.ascontiguousarray(q)),
        C.cast(states, _v), _p(gy), _p(gh), _p(rhs), _p(boundary), _p(nut), _p(den))
    return rhs, boundary, nut, den, status


def wale_nut(g, delta, cw):
    g = np.ascontiguousarray(g, dtype=np.float64).reshape(9)
    out = C.c_double()
    ok = oracle_lib().oracle_wale_nut(_p(g), delta, cw, C.byref(out))
    return out.value if ok else None


def transport_stable_dt(case, q, states, cfl, maximum, wale_cw=-1.0):
    cfg = case["config"]
    return oracle_lib().oracle_transport_stable_dt(
        C.byref(cfg), _p(case["volume"]), case["faces"], _p(case["fixed_q"]), case["fixed_states_ptr"], wale_cw,
        _p(np.ascontiguousarray(q)), C.cast(states, _v), cfl, maximum)


def ref_flash_recover(model_image, q, energy, guess, threads=1, use_cache=True):
    """Reference flash on the host: (states, success, counters[count,7])."""
    from_dtype = guess.dtype
    count = len(energy)
    out = np.zeros(count, dtype=from_dtype)
    success = np.zeros(count, dtype=np.int32)
    counters = np.zeros((count, 7), dtype=np.uint64)
    rc = ref_flash_lib().ref_flash_recover(
        model_image, count, _p(np.ascontiguousarray(q, dtype=np.float64)),
        _p(np.ascontiguousarray(energy, dtype=np.float64)), guess.ctypes.data_as(_v), out.ctypes.data_as(_v),
        success.ctypes.data_as(C.POINTER(C.c_int)), counters.ctypes.data_as(C.POINTER(C.c_uint64)),
        int(use_cache), int(threads))
    if rc:
        raise RuntimeError("reference flash rejected the model image")
    return out, success, counters


def ref_flash_recover_capillary(model_image, q, energy, guess, color, jump, equilibrium, threads=1):
    """The reference's capillary recovery (recoverCapillary) on the host:
    (states, success, status, counters[count,7]); a failed cell keeps its seed."""
    count = len(energy)
    out = np.zeros(count, dtype=guess.dtype)
    success = np.zeros(count, dtype=np.int32)
    status = np.zeros(count, dtype=np.int32)
    counters = np.zeros((count, 7), dtype=np.uint64)
    eq = np.ascontiguousarray(equilibrium, dtype=np.int32)
    rc = ref_flash_lib().ref_flash_recover_capillary(
        model_image, count, _p(np.ascontiguousarray(q, dtype=np.float64)),
        _p(np.ascontiguousarray(energy, dtype=np.float64)), guess.ctypes.data_as(_v),
        _p(np.ascontiguousarray(color, dtype=np.float64)), _p(np.ascontiguousarray(jump, dtype=np.float64)),
        eq.ctypes.data_as(C.POINTER(C.c_int)), out.ctypes.data_as(_v), success.ctypes.data_as(C.POINTER(C.c_int)),
        status.ctypes.data_as(C.POINTER(C.c_int)), counters.ctypes.data_as(C.POINTER(C.c_uint64)), int(threads))
    if rc:
        raise RuntimeError("reference flash rejected the model image")
    return out, success, status, counters


def ref_flash_initialize_tp(model_image, q, energy, guess, color, jump):
    """The reference's capillary primitive initialisation on the host, per cell:
    (normalised q, normalised energy, states, success, status); q and energy
    keep their inputs where a cell fails."""
    q = np.array(q, dtype=np.float64, order="C")
    energy = np.array(energy, dtype=np.float64, order="C")
    count = len(energy)
    out = np.zeros(count, dtype=guess.dtype)
    success = np.zeros(count, dtype=np.int32)
    status = np.zeros(count, dtype=np.int32)
    rc = ref_flash_lib().ref_flash_initialize_tp(
        model_image, count, _p(q), _p(energy), guess.ctypes.data_as(_v),
        _p(np.ascontiguousarray(color, dtype=np.float64)), _p(np.ascontiguousarray(jump, dtype=np.float64)),
        out.ctypes.data_as(_v), success.ctypes.data_as(C.POINTER(C.c_int)), status.ctypes.data_as(C.POINTER(C.c_int)))
    if rc:
        raise RuntimeError("reference flash rejected the model image")
    return q, energy, out, success, status


def ref_wale_pr_evaluate(model_image, q, states, color, jump, enthalpies=True):
    """The reference's WALE PR scalar properties per cell on the host:
    (effective species enthalpies [count, ns], cp, status)."""
    count = len(states)
    q = np.ascontiguousarray(q, dtype=np.float64)
    ns = q.shape[1]
    effective = np.zeros((count, ns))
    cp = np.zeros(count)
    status = np.zeros(count, dtype=np.int32)
    rc = ref_flash_lib().ref_wale_pr_evaluate(
        model_image, count, _p(q), states.ctypes.data_as(_v), _p(np.ascontiguousarray(color, dtype=np.float64)),
        _p(np.ascontiguousarray(jump, dtype=np.float64)), int(enthalpies), _p(effective), _p(cp),
        status.ctypes.data_as(C.POINTER(C.c_int)))
    if rc:
        raise RuntimeError("reference flash rejected the model image")
    return effective, cp, status


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---- the reference's CUDA scalar closure (oracle/_ref/libref_closure.so)
CLOSURE_IN_DTYPE = np.dtype([("coeff", "<f8", (8,)), ("mix", "<f8", (3,)), ("W", "<f8"), ("b", "<f8"),
                             ("r", "<f8"), ("rho", "<f8"), ("energy", "<f8"), ("T", "<f8"), ("lower", "<f8"),
                             ("upper", "<f8"), ("tolerance", "<f8"), ("pmin", "<f8"), ("pmax", "<f8"),
                             ("pr", "<i4"), ("enabled", "<i4")])
CLOSURE_OUT_DTYPE = np.dtype([("p", "<f8"), ("T", "<f8"), ("energy", "<f8"), ("cv", "<f8"), ("success", "<i4"),
                              ("iterations", "<i4")])
_ref_closure = None


def ref_closure_lib():
    """The reference's scalar closure built for sm_100a (needs a GPU to run)."""
    global _ref_closure
    if _ref_closure is None:
        path = REF / "libref_closure.so"
        if not path.exists():
            build()
        lib = C.CDLL(str(path))
        lib.reactive_closure_scalar_create_v1.argtypes = [C.c_size_t, C.c_char_p, C.c_size_t]
        lib.reactive_closure_scalar_create_v1.restype = C.c_void_p
        lib.reactive_closure_scalar_destroy_v1.argtypes = [C.c_void_p]
        lib.reactive_closure_scalar_run_v1.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                                       C.c_char_p, C.c_size_t]
        lib.reactive_closure_scalar_run_v1.restype = C.c_int
        _ref_closure = lib
    return _ref_closure


def ref_closure_run(inputs):
    """Run the reference's scalar closure kernel on CLOSURE_IN_DTYPE records (in
    batches of its 65,536-record capacity); returns CLOSURE_OUT_DTYPE records."""
    lib = ref_closure_lib()
    err = C.create_string_buffer(1024)
    cap = 65536
    h = lib.reactive_closure_scalar_create_v1(cap, err, len(err))
    if not h:
        raise RuntimeError(err.value.decode())
    inputs = np.ascontiguousarray(inputs, dtype=CLOSURE_IN_DTYPE)
    out = np.zeros(len(inputs), dtype=CLOSURE_OUT_DTYPE)
    profile = (C.c_char * 48)()
    try:
        for begin in range(0, len(inputs), cap):
            chunk = inputs[begin:begin + cap]
            res = out[begin:begin + cap]
            rc = lib.reactive_closure_scalar_run_v1(h, chunk.ctypes.data, len(chunk), res.ctypes.data, profile, err,
                                                    len(err))
            if rc:
                raise RuntimeError(err.value.decode())
    finally:
        lib.reactive_closure_scalar_destroy_v1(h)
    return out
