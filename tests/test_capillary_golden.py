"""CPU: the capillary recovery fixture (tests/golden/capillary_ref.npz, written
by make_capillary_golden.py) still is what the reference's own capillary
recovery (recoverCapillary, compiled for the host) gives on the reference's 656
captured inputs with the production model image, bit for bit."""
import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, cases, thermo_data as td

GOLDEN = oracle.HERE.parent / "tests" / "golden" / "capillary_ref.npz"


def test_fixture_holds_the_captured_trace_liquid_cells():
    d = np.load(GOLDEN)
    out = d["out"].view(A.THERMO_DTYPE)
    assert len(d["energy"]) == 656 and d["success"].all() and (d["status"] == 0).all()
    assert (d["jump"] > 0).all() and (d["equilibrium"] == 1).all()
    # nearly all liquid beside a trace of gas: the capillary boundary search's case
    assert (cases.phase_label(out) == 2).all()
    assert (out["liquidMass"][:, 0] / d["q"][:, 2] > 1 - 1e-4).all()


def test_reference_reproduces_the_capillary_fixture():
    if not oracle.REF_FLASH.exists():
        pytest.skip("oracle/_ref not built")
    d = np.load(GOLDEN)
    guess = d["guess"].view(A.THERMO_DTYPE)
    out, ok, status, _ = oracle.ref_flash_recover_capillary(
        td.model_bytes(td.production_model(analytic_jacobian=0)), d["q"], d["energy"], guess.copy(), d["color"],
        d["jump"], d["equilibrium"], threads=oracle.cpu_threads())
    assert np.array_equal(ok, d["success"]) and np.array_equal(status, d["status"])
    assert out.tobytes() == d["out"].tobytes()
