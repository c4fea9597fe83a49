"""CPU: the library's Peng-Robinson mixture evaluator (csrc/pr_mixture.cuh, the
building block of the air / N2O / isopropanol flash) against the reference's own
mixture evaluator (src/reactiveThermo/reactiveDevicePR.h, compiled for the host
by oracle/Makefile) on the production gas's four species. The library's header
is compiled for the host here (it is host and device code from one source), so
the comparison is of the arithmetic: the same status on every input, the same
reported phase, and properties and chemical potentials to round-off."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from spuma_multiphysics_b200 import thermo_data as td
from spuma_multiphysics_b200._abi import Table

ROOT = Path(__file__).resolve().parents[1]
REF = ROOT / "oracle" / "_ref" / "libref_flash.so"
NS = 4
D = C.POINTER(C.c_double)


def build_libs(directory):
    """(host build of the library's evaluator, the reference's, the model image,
    its gas table as a ReactiveB200Table)."""
    if not REF.exists():
        pytest.skip("oracle/_ref not built (make -C oracle)")
    out = Path(directory) / "libmixture_host.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fno-fast-math",
                    "-I", str(ROOT / "spuma-multiphysics_b200" / "csrc"),
                    str(ROOT / "tests" / "native" / "mixture_host_shim.cpp"), "-o", str(out)], check=True)
    ours, ref = C.CDLL(str(out)), C.CDLL(str(REF))
    model = td.mixture_model()
    image = td.model_bytes(model)
    table = Table()
    C.memmove(C.addressof(table), C.addressof(model.phase[0]), C.sizeof(Table))
    return ours, ref, image, table


@pytest.fixture(scope="module")
def libs(tmp_path_factory):
    return build_libs(tmp_path_factory.mktemp("mix"))


def evaluate(libs, T, value, Y, tp, choice=0, chem=1):
    ours, ref, image, table = libs
    y = (C.c_double * NS)(*Y)
    a, b = (C.c_double * (15 + NS))(), (C.c_double * (15 + NS))()
    pa, pb = C.c_int(9), C.c_int(9)
    if tp:
        sa = ours.mix_tp(C.byref(table), C.c_double(T), C.c_double(value), y, choice, chem, a, C.byref(pa))
        sb = ref.ref_pr_mix_tp(image, 0, C.c_double(T), C.c_double(value), y, choice, chem, b, C.byref(pb))
    else:
        sa = ours.mix_trho(C.byref(table), C.c_double(T), C.c_double(value), y, chem, a, C.byref(pa))
        sb = ref.ref_pr_mix_trho(image, 0, C.c_double(T), C.c_double(value), y, chem, b, C.byref(pb))
    return sa, sb, np.array(a[:]), np.array(b[:]), pa.value, pb.value


def compositions(rng, n):
    """Random four-species mass fractions (some with absent species), plus the
    air, pure N2O and pure isopropanol corners."""
    ys = [np.array([.767, .233, 0, 0]), np.array([0, 0, 1., 0]), np.array([0, 0, 0, 1.])]
    for _ in range(n):
        y = rng.dirichlet(np.ones(NS) * .7)
        y[rng.random(NS) < .25] = 0
        if y.sum() == 0:
            y[2] = 1
        ys.append(y / y.sum())
    for y in ys:
        y[-1] = 1 - y[:-1].sum()  # sum exactly one in the last place
    return [y for y in ys if y[-1] >= 0]


def close(a, b, rtol):
    scale = np.maximum(np.abs(b), 1.0)
    return np.max(np.abs(a - b) / scale) <= rtol



def mu_close(a, b, rt):
    """Chemical potentials (J/kmol) to 1e-12 of their size or of RT."""
    return np.all(np.abs(a - b) <= 1e-12 * np.maximum(np.abs(b), rt))


def test_mixture_tp_and_trho_match_the_reference(libs):
    rng = np.random.default_rng(20261203)
    checked = {"tp": 0, "trho": 0, "failures_equal": 0}
    RT = lambda T: 8314.46261815324 * T
    for y in compositions(rng, 40):
        for T in (160.0, 220.0, 293.15, 350.0, 520.0, 900.0):
            for p in (1e4, 1e5, 2e6, 4e6, 8e6, 3e7):
                for choice in (0, 1, 2):
                    sa, sb, a, b, pa, pb = evaluate(libs, T, p, y, True, choice)
                    assert sa == sb, (y, T, p, choice, sa, sb)
                    if sa:
                        checked["failures_equal"] += 1
                        continue
                    assert pa == pb, (y, T, p, choice)
                    # properties (the roots are formed and polished in each code's own
                    # arithmetic: agreement to round-off, about 3e-14 relative)
                    assert close(a[:15], b[:15], 1e-12), (y, T, p, choice, np.abs(a[:15] - b[:15]))
                    assert mu_close(a[15:], b[15:], RT(T)), (y, T, p, choice)
                    checked["tp"] += 1
                    # the same density through (T, rho): the same arithmetic
                    sa, sb, a2, b2, pa2, pb2 = evaluate(libs, T, b[4], y, False)
                    assert sa == sb and (sa or pa2 == pb2)
                    if not sa:
                        assert close(a2[:15], b2[:15], 1e-12), (y, T, b[4], np.abs(a2[:15] - b2[:15]))
                        assert mu_close(a2[15:], b2[15:], RT(T))
                        checked["trho"] += 1
    # every kind of outcome occurred
    assert checked["tp"] > 1000 and checked["trho"] > 1000 and checked["failures_equal"] > 100, checked


def test_mixture_status_on_bad_inputs_matches_the_reference(libs):
    y = np.array([.25, .25, .25, .25])
    for T, v, tp in [(-1.0, 1e5, True), (300.0, -1.0, True), (300.0, 0.0, False), (300.0, 1e9, False)]:
        sa, sb, *_ = evaluate(libs, T, v, y, tp)
        assert sa == sb and sa != 0
    bad = np.array([.5, .5, .5, -.5])  # a negative mass fraction
    sa, sb, *_ = evaluate(libs, 300.0, 1e5, bad, True)
    assert sa == sb == 3
    off = np.array([.3, .3, .3, .3])  # sums to 1.2
    sa, sb, *_ = evaluate(libs, 300.0, 1e5, off, True)
    assert sa == sb == 3
