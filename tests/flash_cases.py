"""Flash parity helpers: seeded pure-N2O batches and comparison metrics."""
import ctypes as C

import numpy as np

from spuma_multiphysics_b200 import _abi as A, cases, thermo_data as td

P_T_TOL = 1e-9      # relative p and T agreement of converged states
STATE_TOL = 1e-7    # relative agreement of derived state fields (rho_g, rho_l, liquid mass, sound)


def model_image(**kw):
    return td.model_bytes(td.pure_model(**kw))


def oracle_flash(oracle, image, q, e, guess):
    n = len(e)
    out = np.zeros(n, dtype=A.THERMO_DTYPE)
    ok = np.zeros(n, dtype=np.int32)
    cnt = np.zeros((n, 7), dtype=np.uint64)
    rc = oracle.oracle_lib().oracle_flash_recover(
        image, n, q.ctypes.data_as(C.POINTER(C.c_double)), e.ctypes.data_as(C.POINTER(C.c_double)),
        guess.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p), ok.ctypes.data_as(C.POINTER(C.c_int)),
        cnt.ctypes.data_as(C.POINTER(C.c_uint64)), 1)
    assert rc == 0
    return out, ok, cnt


def compare(a, ok_a, b, ok_b):
    """Summary of two flash results over cells both solved."""
    both = (ok_a != 0) & (ok_b != 0)
    la, lb = cases.phase_label(a), cases.phase_label(b)
    rel = lambda x, y: np.abs(x - y) / np.maximum(np.abs(y), 1e-300)
    out = dict(cells=len(a), success_equal=bool(np.array_equal(ok_a != 0, ok_b != 0)),
               label_mismatch=int(np.sum(la[both] != lb[both])),
               p_rel=float(rel(a["p"][both], b["p"][both]).max(initial=0)),
               T_rel=float(rel(a["T"][both], b["T"][both]).max(initial=0)),
               ml_rel=float((np.abs(a["liquidMass"][both, 0] - b["liquidMass"][both, 0])
                             / np.maximum(a["rho"][both], 1e-300)).max(initial=0)),
               c_rel=float(rel(a["soundFrozen"][both], b["soundFrozen"][both]).max(initial=0)),
               labels=np.bincount(lb[both], minlength=3).tolist())
    return out
