"""Regenerates capillary_ref.npz: the reference's captured capillary recovery
inputs (tests/data/capillary-trace-air.jsonl.gz of the reference: 656 cells of
the four-species air / N2O / isopropanol model with liquid N2O, each with its
interface color, pressure jump sigma*kappa, bulk energy and seed state) and the
outputs of the reference's own capillary recovery (recoverCapillary, compiled
for the host into oracle/_ref/libref_flash.so) on them, with the production
model image thermo_data.production_model(analytic_jacobian=0) (the capture's
finite-difference closure Jacobian).

Run from the repository root:  python tests/golden/make_capillary_golden.py
(the reference checkout is $REFERENCE, by default `reference` beside the repository)
"""
import gzip
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]
import conftest  # noqa: F401,E402  (registers the package)
from oracle import oracle  # noqa: E402
from spuma_multiphysics_b200 import _abi as A, thermo_data as td  # noqa: E402

OUT = Path(__file__).resolve().parent / "capillary_ref.npz"


def main():
    path = oracle.REFERENCE / "tests" / "data" / "capillary-trace-air.jsonl.gz"
    rows = [json.loads(line) for line in gzip.open(path, "rt").read().splitlines()]
    n = len(rows)
    q = np.array([r["q"] for r in rows], dtype=np.float64)
    # the flash's input is the bulk energy: kinetic and surface energy removed
    energy = np.array([r["search"]["bulkEnergy"] for r in rows], dtype=np.float64)
    color = np.array([r["search"]["color"] for r in rows], dtype=np.float64)
    jump = np.array([r["search"]["pressureJump"] for r in rows], dtype=np.float64)
    equilibrium = np.array([1 if r["equilibrium"] else 0 for r in rows], dtype=np.int32)
    guess = np.zeros(n, dtype=A.THERMO_DTYPE)
    for c, r in enumerate(rows):
        for name in A.THERMO_DTYPE.names:
            if name in r["guess"]:
                guess[name][c] = r["guess"][name]
    image = td.model_bytes(td.production_model(analytic_jacobian=0))
    out, ok, status, _ = oracle.ref_flash_recover_capillary(image, q, energy, guess.copy(), color, jump, equilibrium,
                                                            threads=oracle.cpu_threads())
    np.savez_compressed(OUT, q=q, energy=energy, color=color, jump=jump, equilibrium=equilibrium,
                        guess=guess.view(np.uint8), out=out.view(np.uint8), success=ok, status=status)
    print(f"{n} inputs ({int(equilibrium.sum())} equilibrium, {int((jump != 0).sum())} with a jump), "
          f"{int(ok.sum())} recovered by the reference -> {OUT}")


if __name__ == "__main__":
    main()
