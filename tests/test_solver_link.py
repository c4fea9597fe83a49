"""CPU: a C translation unit that references every reactive_transport_* and
reactive_gpu_hem_* name the reference solver's sources name
(tests/golden/solver_symbols.txt, written by make_solver_symbols.py) links
against libreactive_b200.so with no undefined reference and loads; the
capillary-only stubs return -1 for a null handle like every other entry.
GPU: on a real handle each stub returns 1 with a message."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

from spuma_multiphysics_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
SYMBOLS = (ROOT / "tests" / "golden" / "solver_symbols.txt").read_text().split()
CAPILLARY_ONLY = ["reactive_transport_install_cartesian_v1", "reactive_transport_cartesian_info_v1",
                  "reactive_transport_set_implicit_v1", "reactive_transport_implicit_coefficients_v1",
                  "reactive_transport_set_wale_pr_model_v1", "reactive_transport_wale_pr_properties_v1",
                  "reactive_transport_wale_pr_properties_v2", "reactive_transport_wale_pr_profile_v1",
                  "reactive_transport_capillary_resident_begin_v1", "reactive_transport_capillary_resident_select_v1",
                  "reactive_transport_capillary_resident_update_v1", "reactive_transport_capillary_resident_relax_v1",
                  "reactive_transport_capillary_resident_commit_v1"]
# argument types after the handle (all passed as null / zero: the stubs refuse
# before reading any)
_v, _d, _z, _i = C.c_void_p, C.c_double, C.c_size_t, C.c_int
EXTRA_ARGS = {"reactive_transport_install_cartesian_v1": [_v], "reactive_transport_cartesian_info_v1": [_v],
              "reactive_transport_set_implicit_v1": [_v],
              "reactive_transport_implicit_coefficients_v1": [_v, _v, _z, _v],
              "reactive_transport_set_wale_pr_model_v1": [_v],
              "reactive_transport_wale_pr_properties_v1": [_v, _v, _z, _v],
              "reactive_transport_wale_pr_properties_v2": [_v, _v, _z, _v, _i],
              "reactive_transport_wale_pr_profile_v1": [_v],
              "reactive_transport_capillary_resident_begin_v1": [_z, _v, _v, _v, _v, _v, _d, _i, _v],
              "reactive_transport_capillary_resident_select_v1": [_i, _v, _v],
              "reactive_transport_capillary_resident_update_v1": [_z, _v, _v],
              "reactive_transport_capillary_resident_relax_v1": [],
              "reactive_transport_capillary_resident_commit_v1": [_v, _v, _v, _v]}


def _bind(lib, name):
    fn = getattr(lib, name)
    fn.restype = C.c_int
    fn.argtypes = [_v] + EXTRA_ARGS[name]
    return fn, [0 if t in (_z, _i, _d) else None for t in EXTRA_ARGS[name]]


def test_fixture_lists_the_solver_names():
    assert len(SYMBOLS) >= 40
    assert "reactive_transport_advance_resident_v2" in SYMBOLS and "reactive_gpu_hem_run_v2" in SYMBOLS
    assert set(CAPILLARY_ONLY) - {"reactive_transport_wale_pr_properties_v1"} <= set(SYMBOLS)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_solver_names_link_against_the_library(tmp_path):
    lib = Path(_lib.LIB_PATH)
    src = tmp_path / "link.c"
    decls = "".join(f"extern void {n}(void);\n" for n in SYMBOLS)
    table = ",\n".join(f"    (void (*)(void)){n}" for n in SYMBOLS)
    src.write_text(f'#include <stdio.h>\n{decls}\nstatic void (*const names[])(void) = {{\n{table}\n}};\n'
                   'int main(void) {\n    int n = 0;\n'
                   '    for (unsigned i = 0; i < sizeof(names) / sizeof(names[0]); ++i) n += names[i] != 0;\n'
                   '    printf("%d\\n", n);\n    return 0;\n}\n')
    exe = tmp_path / "link"
    res = subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe), f"-L{lib.parent}", f"-l:{lib.name}",
                          f"-Wl,-rpath,{lib.parent}", "-Wl,--no-undefined"], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    assert int(run.stdout) == len(SYMBOLS)


@pytest.mark.parametrize("name", CAPILLARY_ONLY)
def test_capillary_stub_rejects_null_handle(name):
    fn, args = _bind(C.CDLL(str(_lib.LIB_PATH)), name)
    assert fn(None, *args) == -1


@pytest.mark.gpu
def test_capillary_stubs_refuse_with_a_message():
    import numpy as np
    import transport_cases as T
    lib = T.bind(_lib.load())
    case = T.make_case(4, 64, 3, viscous_only=True, conduction=True, spatial=True)
    h = T.create(lib, 1, case)
    raw = C.CDLL(str(_lib.LIB_PATH))
    raw.reactive_transport_error.restype = C.c_char_p
    raw.reactive_transport_error.argtypes = [C.c_void_p]
    try:
        for name in CAPILLARY_ONLY:
            fn, args = _bind(raw, name)
            assert fn(h, *args) == 1, name
            if "capillary_resident" in name or "wale_pr" in name:
                # implemented: with null arguments, on a handle without the
                # capillary model, they refuse with their own message
                assert raw.reactive_transport_error(h), name
            else:
                assert b"is not part of this B200 transport build" in raw.reactive_transport_error(h), name
        # the handle still works after the refusals
        qq = case["q"].copy()
        br = np.zeros(case["nv"])
        assert lib.reactive_transport_stage(h, T.dp(qq), T.states_ptr(case["states"]), None, None, 1e-7, 0,
                                            T.dp(br)) == 0
    finally:
        lib.reactive_transport_destroy(h)
