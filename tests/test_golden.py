"""CPU: the oracles against golden outputs of the reference's own code
(tests/golden/*.npz, written by tests/golden/make_golden.py from the reference
builds in oracle/_ref/), and the seeded case generators reproduce the fixture
inputs bit for bit."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, cases, thermo_data as td
import flash_cases as F
import transport_cases as T

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_flash():
    z = np.load(GOLDEN / "flash_ref.npz")
    return z["q"], z["e"], z["guess"].view(A.THERMO_DTYPE), z


def test_golden_flash_inputs_reproduce():
    q, e, guess, _ = load_flash()
    q1, e1, g1 = cases.flash_batch(256, seed=424242)
    assert np.array_equal(q[:256], q1) and np.array_equal(e[:256], e1)
    assert np.array_equal(guess[:256].view(np.uint8), g1.view(np.uint8))


def test_oracle_flash_matches_golden():
    q, e, guess, z = load_flash()
    out, ok, _ = F.oracle_flash(oracle, td.model_bytes(td.pure_model()), q, e, guess)
    assert np.array_equal(ok, z["success"])
    both = ok != 0
    assert np.array_equal(cases.phase_label(out)[both], z["label"][both])
    for k in ("p", "T"):
        assert np.max(np.abs(out[k][both] / z[f"out_{k}"][both] - 1)) <= F.P_T_TOL
    assert np.max(np.abs(out["soundEquilibrium"][both] / z["out_soundEquilibrium"][both] - 1)) <= F.STATE_TOL


@pytest.mark.parametrize("index", range(4))
def test_oracle_transport_matches_golden(index):
    import sys
    sys.path.insert(0, str(GOLDEN))
    import make_golden
    spec, cw = make_golden.TRANSPORT_CASES[index]
    ns, nc, kind, tr, mech, sp, extra, frozen = spec
    case = T.make_case(ns, nc, kind, tr and cw is None, mech, sp, extra, frozen, seed=3, viscous_only=cw is not None)
    z = np.load(GOLDEN / "transport_ref.npz")
    assert np.array_equal(case["q"], z[f"c{index}_q"])
    rhs, br, _, _, status = oracle.transport_rhs(case, case["q"], case["states"].ctypes.data_as(C.c_void_p),
                                                 case["y"], case["h"], wale_cw=-1.0 if cw is None else cw)
    assert status == 0
    assert T.scaled_error(rhs, z[f"c{index}_rhs"]) <= T.RHS_TOL
    assert T.scaled_error(br[None], z[f"c{index}_boundary"][None]) <= T.RHS_TOL
    dt = oracle.transport_stable_dt(case, case["q"], case["states"].ctypes.data_as(C.c_void_p), .23, .1,
                                    wale_cw=-1.0 if cw is None else cw)
    assert abs(dt / float(z[f"c{index}_dt"]) - 1) < T.DT_TOL
