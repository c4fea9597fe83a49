"""CPU: the WALE Peng-Robinson scalar properties (csrc/wale_pr.cuh, compiled for
the host) against the reference's own ReactiveDeviceWalePr::evaluate compiled
for the host, on accepted states of the capillary flash: the captured
trace-liquid cells (tests/golden/capillary_ref.npz) with their colors and jumps,
and the same states with other jumps; the statuses, the heat capacities
bit for bit, the effective species enthalpies to round-off; and the rejections
of states that do not match their phases."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, thermo_data as td

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden" / "capillary_ref.npz"
D = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    if not oracle.REF_FLASH.exists():
        pytest.skip("oracle/_ref not built (make -C oracle)")
    out = tmp_path_factory.mktemp("walepr") / "libmixture_host.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                    "-I", str(ROOT / "spuma-multiphysics_b200" / "csrc"),
                    str(ROOT / "tests" / "native" / "mixture_host_shim.cpp"), "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    lib.wale_pr_properties.argtypes = [C.c_void_p, C.c_size_t, D, C.c_void_p, D, D, C.c_int, D, D,
                                       C.POINTER(C.c_int)]
    return lib


def ours(lib, model, q, states, color, jump, enthalpies=True):
    n, ns = q.shape
    eff, cp, status = np.zeros((n, ns)), np.zeros(n), np.zeros(n, dtype=np.int32)
    lib.wale_pr_properties(C.byref(model), n, np.ascontiguousarray(q).ctypes.data_as(D),
                           states.ctypes.data_as(C.c_void_p), np.ascontiguousarray(color).ctypes.data_as(D),
                           np.ascontiguousarray(jump).ctypes.data_as(D), int(enthalpies), eff.ctypes.data_as(D),
                           cp.ctypes.data_as(D), status.ctypes.data_as(C.POINTER(C.c_int)))
    return eff, cp, status


def compare(lib, model, image, q, states, color, jump):
    eff, cp, status = ours(lib, model, q, states, color, jump)
    reff, rcp, rstatus = oracle.ref_wale_pr_evaluate(image, q, states, color, jump)
    assert np.array_equal(status, rstatus), (np.bincount(status), np.bincount(rstatus))
    ok = status == 0
    assert np.array_equal(cp[ok], rcp[ok])
    scale = np.maximum(np.abs(reff[ok]).max(axis=1, keepdims=True), 1.0)
    assert np.max(np.abs(eff[ok] - reff[ok]) / scale, initial=0) <= 1e-11
    return status


def test_trace_liquid_states_match_the_reference(host):
    d = np.load(GOLDEN)
    states = d["out"].view(A.THERMO_DTYPE).copy()
    model = td.production_model(analytic_jacobian=0)
    image = td.model_bytes(model)
    status = compare(host, model, image, d["q"], states, d["color"], d["jump"])
    assert (status == 0).all()
    # the cp-only request reads the state alone
    _, cp, st = ours(host, model, d["q"], states, d["color"], d["jump"], enthalpies=False)
    assert (st == 0).all() and np.array_equal(cp, states["cp"])


def test_other_jumps_and_colors_match_the_reference(host):
    """The same states read with other interface colors and jumps: where the
    state no longer matches its phases (its energy or liquid density was solved
    for another jump) both report the same status."""
    d = np.load(GOLDEN)
    states = d["out"].view(A.THERMO_DTYPE).copy()
    model = td.production_model(analytic_jacobian=0)
    image = td.model_bytes(model)
    rng = np.random.default_rng(3)
    n = len(states)
    color = rng.choice([0.0, .5, 1.0], n)
    jump = d["jump"] * rng.choice([0.0, 1.0, 1e2, 1e5], n)
    status = compare(host, model, image, d["q"], states, color, jump)
    assert (status == 0).any() and (status != 0).any(), np.bincount(status)


def test_rejections_match_the_reference(host):
    d = np.load(GOLDEN)
    model = td.production_model(analytic_jacobian=0)
    image = td.model_bytes(model)
    n = 64
    states = d["out"].view(A.THERMO_DTYPE)[:n].copy()
    q = d["q"][:n].copy()
    color, jump = d["color"][:n].copy(), d["jump"][:n].copy()
    states["rho"][0] *= 1.001            # density off its species
    states["rhoLiquid"][1] *= 1.01       # liquid density off its EOS
    states["e"][2] *= 1.01               # energy off the phases' enthalpy
    q[3, 0] = -1.0                       # negative inventory
    color[4] = 1.5                       # color outside [0, 1]
    jump[5] = 1e12                       # a liquid pressure outside the model's range
    states["cp"][6] = -1.0               # no heat capacity
    states["liquidMass"][7, 0] = q[7, 2] * 2  # more liquid than species
    status = compare(host, model, image, q, states, color, jump)
    assert set(status[:8].tolist()) >= {2, 3, 7, 8}, status[:8]
    assert (status[8:] == 0).all()
