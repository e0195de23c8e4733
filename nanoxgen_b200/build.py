"""Builds libnxg_b200.so in-tree for sm_100a (nvcc for the CUDA units, g++
for the host unit, static cudart) and, on request, the test-only checkers
under oracle/ (see oracle/Makefile).

    python -m nanoxgen_b200.build          # product library
    python -m nanoxgen_b200.build --all    # plus oracle checkers
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libnxg_b200.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", shutil.which("g++") or "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE,
                     "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra", "-I" + INCLUDE]

CUDA_SOURCES = ["generate.cu", "batched.cu", "classic.cu", "surrogate.cu", "stencil.cu"]
HOST_SOURCES = ["host.cpp", "expression.cpp"]
HEADERS = ["nxg_internal.h", "strand_math.cuh", "generator_core.cuh", "seexpr_gradients.inc", "expression.h",
           "seexpr_permutation.inc", "classic_eval.cuh", "umma.cuh", "walk.cuh"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_library(verbose: bool = False, force: bool = False) -> str:
    """Compiles and links libnxg_b200.so when any source is newer than it."""
    os.makedirs(OBJ, exist_ok=True)
    common = [os.path.join(INCLUDE, "nxg.h"), os.path.join(INCLUDE, "nxg_classic.h")] + [os.path.join(CSRC, h) for h in HEADERS]
    objects = []
    for src in CUDA_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        if force or _stale(obj, [path] + common):
            _run([NVCC] + NVCC_FLAGS + ["-c", path, "-o", obj], verbose)
        objects.append(obj)
    for src in HOST_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        if force or _stale(obj, [path] + common):
            _run([CXX] + CXX_FLAGS + ["-c", path, "-o", obj], verbose)
        objects.append(obj)
    if force or _stale(LIB, objects):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objects + ["-lpthread"], verbose)
    return LIB


def build_oracle(verbose: bool = False) -> None:
    """Builds oracle/liboracle.so, and oracle/_ref/libnxg_ref.so where the
    reference checkout exists (test-only checkers, never product code)."""
    targets = ["oracle"]
    ref = os.environ.get("NXG_REFERENCE_ROOT", "/root/reference")
    if os.path.isfile(os.path.join(ref, "src", "asset.cpp")):
        targets.append("ref")
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "REF=" + ref] + targets, verbose)


if __name__ == "__main__":
    verbose = "-v" in sys.argv
    build_library(verbose=verbose, force="--force" in sys.argv)
    if "--all" in sys.argv:
        build_oracle(verbose=verbose)
    print(LIB)
