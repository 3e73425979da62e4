"""Builds kiwi_b200/libkiwi_b200.so in-tree with nvcc for sm_100a.

Each translation unit carries its own floating-point contract:
  * the plain all-FP64 form and the host/binning code: --fmad=false, so that products and sums round
    exactly as the reference's x86-64 build does;
  * the lattice forms (lattice.cu, the adjoint) and the FP32-mixed form: FMA contraction on -- they regroup
    the reference's sum, so rounding each product on its own buys nothing; the quantities integer results
    depend on (bounding boxes, lattice planes, cell centres, the pair counters' support test) use explicitly
    rounded operations in every unit.

Usage: python -m kiwi_b200.build [--verbose]   (or kiwi_b200.build.build())
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkiwi_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr"]

# (source, extra flags)
UNITS = [
    ("capi.cu", ["--fmad=false"]),
    ("kiwi_fp64.cu", ["--fmad=false"]),
    ("lattice.cu", []),
    ("noalloc.cu", ["--fmad=false"]),
    ("voronoi.cu", ["--fmad=false"]),
    ("adjoint.cu", []),
    ("mixed.cu", []),
    ("batch.cu", ["--fmad=false"]),
    ("io.cu", []),
    ("tabulated.cu", ["--fmad=false"]),
    ("cartmap.cu", ["--fmad=false"]),
    ("pointset.cu", ["--fmad=false"]),
    ("lloyd.cu", ["--fmad=false"]),
    # the C++ drop-in of the reference's kernel-integral layer (host code over the C ABI)
    ("kernel_layer.cpp", ["-I" + os.path.join(HERE, "..", "include")]),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, defines: tuple = (), out: str | None = None) -> str:
    """Compiles the library.  `defines` (e.g. ("KIWI_GATHER_MIN_BLOCKS=1",)) and `out` build a variant
    into its own directory (for tuning sweeps); the default is the in-tree kiwi_b200/libkiwi_b200.so."""
    global BUILD, LIB
    if out is not None:
        BUILD = os.path.join(os.path.dirname(os.path.abspath(out)), "_build")
        LIB = os.path.abspath(out)
    extra_defs = [f"-D{d}" for d in defines]
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "kiwi_b200.h"))
    inc_kiwi = os.path.join(HERE, "..", "include", "kiwi")
    headers += [os.path.join(inc_kiwi, f) for f in os.listdir(inc_kiwi) if f.endswith(".hpp")]
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or _stale(o, [s, __file__] + headers):
            cmd = ([nvcc()] + ARCH + COMMON + extra + extra_defs + (["-Xptxas", "-v"] if verbose else []) +
                   ["-c", s, "-o", o])
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if verbose or r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}")
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libkiwi_b200.so failed")
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
