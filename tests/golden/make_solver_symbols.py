"""Regenerates solver_symbols.txt: every reactive_transport_* and
reactive_gpu_hem_* name that the reference solver's sources reference
(src/reactiveFoam/*.C, *.H, *.inc: direct calls, and the dlsym names of its
flash worker pool). A solver linked against this library must resolve each one.

Run from the repository root:  python tests/golden/make_solver_symbols.py
(the reference checkout is $REFERENCE, by default `reference` beside the repository)
"""
import re
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle  # noqa: E402

NAME = re.compile(r"\breactive_(?:transport|gpu_hem)_[a-z0-9_]+")


def main():
    src = oracle.REFERENCE / "src" / "reactiveFoam"
    names = set()
    for path in sorted(src.iterdir()):
        if path.suffix in (".C", ".H", ".inc"):
            names.update(NAME.findall(path.read_text(errors="replace")))
    out = Path(__file__).resolve().parent / "solver_symbols.txt"
    out.write_text("".join(f"{n}\n" for n in sorted(names)))
    print(f"{len(names)} names -> {out}")


if __name__ == "__main__":
    main()
