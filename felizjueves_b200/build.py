"""Build libfjb.so in-tree: nvcc for sm_100a (cross-compiles without a GPU).

    python -m felizjueves_b200.build        # or felizjueves_b200.build.build()

The library lands in felizjueves_b200/_lib/libfjb.so, beside the package, so
that it travels with the source tree.  Host C++ is compiled with
-ffp-contract=off: the plan's bounds are reproduced operation for operation,
and a fused multiply-add would change their last bits.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libfjb.so")
REPO = os.path.dirname(HERE)

CU_SOURCES = ["fjb.cu"]
CPP_SOURCES = ["plan.cpp", "hgp_tables.cpp", "boys_table.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libfjb")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(REPO, "include", "fjb.h"))
    if not force and _newer(LIB, deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    cc = nvcc()
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I", CSRC, "-I", os.path.join(REPO, "include")]
    for src in CPP_SOURCES:
        obj = os.path.join(OUT_DIR, src + ".o")
        cmd = [cc, *common, "-x", "c++", "-c", os.path.join(CSRC, src), "-o", obj]
        _run(cmd, verbose)
        objs.append(obj)
    for src in CU_SOURCES:
        obj = os.path.join(OUT_DIR, src + ".o")
        cmd = [cc, *common, *ARCH, "-lineinfo", "--fmad=true", "-Xptxas", "-v" if verbose else "-O3",
               "-c", os.path.join(CSRC, src), "-o", obj]
        _run(cmd, verbose)
        objs.append(obj)
    tmp = LIB + ".tmp"
    _run([cc, "-shared", *ARCH, "-o", tmp, *objs, "-lcudart"], verbose)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode:
        raise RuntimeError(f"build step failed: {' '.join(cmd[:4])} ...")


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
