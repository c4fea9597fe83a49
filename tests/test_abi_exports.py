"""CPU: the C-ABI library loads and exports every function include/*.h declares
(no compute calls: there is no GPU here)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from spuma_multiphysics_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**\s*((?:reactive|rb200)_[A-Za-z0-9_]+)\s*\(",
                  re.M)


def declared():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        names.update(DECL.findall(header.read_text()))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared()
    assert "reactive_transport_create" in names and "reactive_gpu_hem_run_v1" in names


@pytest.mark.parametrize("name", declared())
def test_library_exports(name):
    lib = C.CDLL(str(_lib.LIB_PATH))
    assert hasattr(lib, name), f"{name} is declared in include/ but not exported"
