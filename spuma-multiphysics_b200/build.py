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
# Per translation unit rounding policy. Transport: separate rounding
# (--fmad=false) so antisymmetric face terms cancel exactly, e.g. the HLL mass and
# energy fluxes through a slip wall are exactly zero as in the reference's CPU and
# CUDA builds. HEM: fused multiply-add (the Newton iteration is insensitive to it).
# The plain per-cell flash (hem_plain.cu) inlines every EOS/flash routine, the
# work-queue flash (hem.cu) keeps them out of line: each form built as it runs best.
SOURCES = {"transport.cu": ["--fmad=false"], "hem.cu": ["--fmad=true"],
           "hem_plain.cu": ["--fmad=true", "-DRB200_EOS_FN=inline", "-DRB200_FLASH_FN=inline"],
           "ideal.cu": ["--fmad=true"], "probe.cu": ["--fmad=true"], "mixture.cu": ["--fmad=true"],
           # the multi-species flash: separate rounding, as the reference's host build it is compared with
           "hem_mixture.cu": ["--fmad=false"],
           # host-only helpers (no device code)
           "host_tools.cpp": []}
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
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    compile_flags = [f for f in FLAGS if f != "--shared"]
    jobs = []
    for name, policy in SOURCES.items():
        obj = objdir / (name + ".o")
        jobs.append(([nvcc(), *ARCH, *compile_flags, *policy, *extra, "-c", str(CSRC / name), "-o", str(obj)], obj))
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        list(pool.map(lambda job: _run(job[0], verbose), jobs))
    objects = [str(obj) for _, obj in jobs]
    _run([nvcc(), *ARCH, "--shared", *objects, "-o", str(LIB), "-lcudart", "-lpthread"], verbose)
    return LIB


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stderr[-6000:]}")
    if verbose and res.stderr:
        print(res.stderr[-4000:], file=sys.stderr)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
