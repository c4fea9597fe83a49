"""CPU: the mixture flash fixture (tests/golden/mixture_ref.npz, written by
make_mixture_golden.py) still is what the reference's device flash compiled for
the host gives on the reference's 256 captured recovery inputs with the
two-liquid model image, bit for bit."""
import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, cases, thermo_data as td

GOLDEN = oracle.HERE.parent / "tests" / "golden" / "mixture_ref.npz"


def test_two_liquid_image_is_valid_for_the_reference():
    if not oracle.REF_FLASH.exists():
        pytest.skip("oracle/_ref not built")
    image = td.model_bytes(td.two_liquid_model())
    assert len(image) == 47448 and oracle.ref_flash_lib().ref_flash_valid_model(image) == 1


def test_reference_reproduces_the_mixture_fixture():
    if not oracle.REF_FLASH.exists():
        pytest.skip("oracle/_ref not built")
    d = np.load(GOLDEN)
    guess = d["guess"].view(A.THERMO_DTYPE)
    out, ok, _ = oracle.ref_flash_recover(td.model_bytes(td.two_liquid_model()), d["q"], d["energy"], guess.copy(),
                                          threads=oracle.cpu_threads())
    assert np.array_equal(ok, d["success"])
    assert out.tobytes() == d["out"].tobytes()
    assert d["success"].all() and (cases.phase_label(out) == 2).all()
