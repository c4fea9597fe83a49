"""Regenerates the golden fixtures from the REFERENCE's own code, built by
oracle/Makefile into oracle/_ref/ from the reference sources:

  flash_ref.npz      reference device flash (host build) on 320 seeded pure-N2O
                     states (256 with the generating state as seed, 64 with a
                     fixed 40 bar / 293.15 K gas seed)
  transport_ref.npz  reference CPU transport (backend 0) RHS, boundary ledger and
                     CFL step on three validation configurations and one WALE mesh

Run from the repository root:  python tests/golden/make_golden.py
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]
import conftest  # noqa: F401,E402  (registers the package)
from oracle import oracle  # noqa: E402
from spuma_multiphysics_b200 import cases, thermo_data as td  # noqa: E402
import transport_cases as T  # noqa: E402

OUT = Path(__file__).resolve().parent
FLASH_FIELDS = ("p", "T", "rhoGas", "liquidMass", "soundFrozen", "soundEquilibrium", "gasMass", "activeLiquids")
TRANSPORT_CASES = [((4, 7, 1, True, False, False, 0, 0), None), ((4, 257, 3, True, False, True, 4097, 0), None),
                   ((8, 7, 0, False, True, False, 0, 0), None), ((2, 33, 3, True, False, True, 0, 0), 0.325)]


def flash():
    image = td.model_bytes(td.pure_model())
    parts = [cases.flash_batch(256, seed=424242), cases.flash_batch(64, seed=515151, seed_policy="fixed")]
    q = np.concatenate([p[0] for p in parts])
    e = np.concatenate([p[1] for p in parts])
    guess = np.concatenate([p[2] for p in parts])
    out, ok, _ = oracle.ref_flash_recover(image, q, e, guess)
    fields = {f"out_{k}": (out[k][:, 0] if k == "liquidMass" else out[k]) for k in FLASH_FIELDS}
    np.savez_compressed(OUT / "flash_ref.npz", q=q, e=e, guess=guess.view(np.uint8), success=ok,
                        label=cases.phase_label(out), **fields)


def transport():
    lib = T.bind(oracle.ref_transport_lib())
    store = {}
    for i, (spec, cw) in enumerate(TRANSPORT_CASES):
        ns, nc, kind, tr, mech, sp, extra, frozen = spec
        case = T.make_case(ns, nc, kind, tr and cw is None, mech, sp, extra, frozen, seed=3,
                           viscous_only=cw is not None)
        h = T.create(lib, 0, case, wale_cw=cw)
        rhs, br, dt = np.empty_like(case["q"]), np.empty(case["nv"]), C.c_double()
        assert lib.reactive_transport_rhs(h, T.dp(case["q"]), T.states_ptr(case["states"]), T.dp(case["y"]),
                                          T.dp(case["h"]), T.dp(rhs), T.dp(br)) == 0
        assert lib.reactive_transport_stable_step(h, T.dp(case["q"]), T.states_ptr(case["states"]), .23, .1,
                                                  C.byref(dt)) == 0
        lib.reactive_transport_destroy(h)
        store[f"c{i}_rhs"], store[f"c{i}_boundary"], store[f"c{i}_dt"] = rhs, br, np.array(dt.value)
        store[f"c{i}_q"] = case["q"]
    np.savez_compressed(OUT / "transport_ref.npz", **store)


if __name__ == "__main__":
    flash()
    transport()
    print("golden fixtures written to", OUT)
