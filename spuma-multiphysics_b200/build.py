"""Builds libreactive_b200.so (transport + HEM C ABI) for sm_100a with nvcc.

The library is built in-tree next to this file so it travels with the working
tree; nothing is installed into site-packages or a JIT cache.
"""
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libreactive_b200.so"
SOURCES = ["transport.cu", "hem.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--shared", "-Xptxas", "-warn-spills",
         "--expt-relaxed-constexpr"]


def nvcc():
    for candidate in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if candidate and (Path(candidate).exists() or candidate == "nvcc"):
            return candidate
    raise RuntimeError("nvcc not found")


def _stale():
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + list((HERE.parent / "include").glob("*.h"))
    return any(p.stat().st_mtime > built for p in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    sources = [str(CSRC / s) for s in SOURCES if (CSRC / s).exists()]
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, *sources, "-o", str(LIB), "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stderr[-6000:]}")
    if verbose and res.stderr:
        print(res.stderr[-4000:], file=sys.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
