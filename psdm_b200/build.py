"""Build the CUDA engine library libpsdm_rtm.so in-tree for sm_100a.

    python -m psdm_b200.build [--verbose]

Uses nvcc directly (no JIT cache): the shared library lands in
psdm_b200/lib/ next to the sources, so it travels with the repository.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libpsdm_rtm.so")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")

SOURCES = ["rtm_step.cu", "rtm_pair.cu", "rtm_resident.cu", "rtm_fp64.cu", "rtm_engine.cu", "rtm_host.cpp", "rtm_noalloc.cu", "rtm_condition.cu", "su_io.cpp", "rtm_filter.cu", "nav.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the engine has no CPU fallback and must be built with CUDA")


def flags(verbose_ptxas: bool = False) -> list[str]:
    f = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler",
         "-ffp-contract=off", "-I", INCLUDE, "-I", CSRC, *ARCH]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in os.listdir(CSRC)] + [os.path.join(INCLUDE, "psdm_rtm.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    tmp = os.path.join(LIBDIR, "_obj")
    os.makedirs(tmp, exist_ok=True)
    for s in SOURCES:
        o = os.path.join(tmp, os.path.splitext(s)[0] + ".o")
        cmd = [nvcc(), *flags(verbose), "-c", os.path.join(CSRC, s), "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0 or verbose:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}")
        objs.append(o)
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart", "-lcufft"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))
