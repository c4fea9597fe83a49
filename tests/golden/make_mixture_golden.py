"""Regenerates mixture_ref.npz: the reference's captured recovery inputs
(tests/fixtures/r04-recovery.jsonl of the reference: 256 cells of the
four-species air / N2O / isopropanol model, nearly pure liquid isopropanol with
traces of air, with the seed states they were captured with) and the outputs of
the reference's own device flash compiled for the host (oracle/_ref/libref_flash.so)
on them, with the two-liquid model image thermo_data.two_liquid_model().

Run from the repository root:  python tests/golden/make_mixture_golden.py
(the reference checkout is $REFERENCE, by default `reference` beside the repository)
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]
import conftest  # noqa: F401,E402  (registers the package)
from oracle import oracle  # noqa: E402
from spuma_multiphysics_b200 import _abi as A, thermo_data as td  # noqa: E402

OUT = Path(__file__).resolve().parent / "mixture_ref.npz"


def main():
    rows = [json.loads(line) for line in
            (oracle.REFERENCE / "tests" / "fixtures" / "r04-recovery.jsonl").read_text().splitlines()]
    n = len(rows)
    q = np.array([r["q"] for r in rows], dtype=np.float64)
    energy = np.array([r["energy"] for r in rows], dtype=np.float64)
    # the seed state of a row: its `guess` record, or the row itself; fields the
    # row does not give stay zero (the reference replay's guess_of)
    guess = np.zeros(n, dtype=A.THERMO_DTYPE)
    for c, r in enumerate(rows):
        values = r.get("guess", r)
        for name in A.THERMO_DTYPE.names:
            if name in values:
                guess[name][c] = values[name]
    image = td.model_bytes(td.two_liquid_model())
    out, ok, _ = oracle.ref_flash_recover(image, q, energy, guess.copy(), threads=oracle.cpu_threads())
    np.savez_compressed(OUT, q=q, energy=energy, guess=guess.view(np.uint8), out=out.view(np.uint8), success=ok)
    print(f"{n} inputs, {int(ok.sum())} recovered by the reference -> {OUT}")


if __name__ == "__main__":
    main()
