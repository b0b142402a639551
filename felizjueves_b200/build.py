"""Build libfjb.so in-tree: nvcc for sm_100a (cross-compiles without a GPU).

    python -m felizjueves_b200.build        # or felizjueves_b200.build.build()

Steps: (1) compile and run the generator csrc/gen_hgp.cpp, which writes the
straight-line VRR/HRR bodies of the register-path classes into
csrc/_gen/hgp_classes.cuh from the same recurrence programs
(csrc/hgp_tables.cpp) the interpreter kernel runs; (2) compile every source
in parallel; (3) link felizjueves_b200/_lib/libfjb.so, beside the package, so
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
GEN = os.path.join(CSRC, "_gen")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libfjb.so")
REPO = os.path.dirname(HERE)

CU_SOURCES = ["fjb.cu", "fock_compiled.cu", "router.cu", "jengine.cu", "onee.cu", "rys_fock.cu",
              "rys_fock64.cu", "rys_fock32.cu", "df_mm.cu", "df_eri3.cu"]
CPP_SOURCES = ["plan.cpp", "hgp_tables.cpp", "boys_table.cpp", "scatter.cpp", "rys_table.cpp", "hjk_plan.cpp"]
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


def _sources() -> list[str]:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if os.path.isfile(os.path.join(CSRC, f))]


def generate(verbose: bool = False) -> str:
    """Run the generator; returns the generated header's path."""
    os.makedirs(GEN, exist_ok=True)
    out = os.path.join(GEN, "hgp_classes.cuh")
    gen_src = [os.path.join(CSRC, "gen_hgp.cpp"), os.path.join(CSRC, "hgp_tables.cpp"),
               os.path.join(CSRC, "hgp_tables.h"), os.path.join(CSRC, "fjb_internal.h")]
    if _newer(out, gen_src):
        return out
    exe = os.path.join(GEN, "gen_hgp")
    cxx = shutil.which("g++") or "g++"
    _run([cxx, "-O2", "-std=c++17", "-I", CSRC, "-o", exe, gen_src[0], gen_src[1]], verbose)
    _run([exe, out + ".tmp"], verbose)
    os.replace(out + ".tmp", out)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    deps = _sources() + [os.path.join(REPO, "include", "fjb.h")]
    if not force and _newer(LIB, deps) and os.path.exists(os.path.join(GEN, "hgp_classes.cuh")):
        return LIB
    generate(verbose)
    os.makedirs(OUT_DIR, exist_ok=True)
    cc = nvcc()
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I", CSRC, "-I", os.path.join(REPO, "include")]
    jobs = []
    for src in CPP_SOURCES:
        obj = os.path.join(OUT_DIR, src + ".o")
        jobs.append(([cc, *common, "-x", "c++", "-c", os.path.join(CSRC, src), "-o", obj], obj))
    for src in CU_SOURCES:
        obj = os.path.join(OUT_DIR, src + ".o")
        jobs.append(([cc, *common, *ARCH, "-lineinfo", "--fmad=true", "-c",
                      os.path.join(CSRC, src), "-o", obj], obj))
    procs = []
    for cmd, obj in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                       text=True), cmd, obj))
    failed = None
    for p, cmd, obj in procs:
        out, err = p.communicate()
        if verbose or p.returncode:
            sys.stdout.write(out)
            sys.stderr.write(err)
        if p.returncode and failed is None:
            failed = cmd
    if failed:
        raise RuntimeError(f"build step failed: {' '.join(failed[:4])} ...")
    objs = [obj for _, obj in jobs]
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
