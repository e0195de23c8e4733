"""Builds libnxg_b200.so in-tree for sm_100a (nvcc for the CUDA units, g++
for the host unit, static cudart) and, on request, the test-only checkers
under oracle/ (see oracle/Makefile).

    python -m nanoxgen_b200.build          # product library
    python -m nanoxgen_b200.build --all    # plus oracle checkers
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

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

CUDA_SOURCES = ["generate.cu", "batched.cu", "classic.cu", "surrogate.cu", "stencil.cu", "fx.cu", "curve_cache.cu", "payload.cu"]
HOST_SOURCES = ["host.cpp", "expression.cpp"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _includes(path: str, seen: set) -> list[str]:
    """`path` and every header it includes by a quoted name, found next to it
    or under include/, recursively."""
    if path in seen:
        return []
    seen.add(path)
    out = [path]
    with open(path) as fh:
        for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', fh.read(), re.M):
            for d in (os.path.dirname(path), INCLUDE):
                cand = os.path.join(d, name)
                if os.path.exists(cand):
                    out += _includes(cand, seen)
                    break
    return out


def build_library(verbose: bool = False, force: bool = False) -> str:
    """Compiles (in parallel) the translation units whose source or included
    headers are newer than their object, then links libnxg_b200.so."""
    os.makedirs(OBJ, exist_ok=True)
    jobs, objects = [], []
    for src in CUDA_SOURCES + HOST_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objects.append(obj)
        if force or _stale(obj, _includes(path, set())):
            tool = [NVCC] + NVCC_FLAGS if src.endswith(".cu") else [CXX] + CXX_FLAGS
            jobs.append(tool + ["-c", path, "-o", obj])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as pool:
            for f in [pool.submit(_run, cmd, verbose) for cmd in jobs]:
                f.result()
    if force or _stale(LIB, objects):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objects + ["-lpthread"], verbose)
    return LIB


def reference_root() -> str:
    """The reference checkout: $NXG_REFERENCE_ROOT, else a `reference`
    directory beside this repository."""
    return os.environ.get("NXG_REFERENCE_ROOT", os.path.join(os.path.dirname(ROOT), "reference"))


def build_oracle(verbose: bool = False) -> None:
    """Builds oracle/liboracle.so, and oracle/_ref/libnxg_ref.so where the
    reference checkout exists (test-only checkers, never product code)."""
    targets = ["oracle"]
    ref = reference_root()
    if os.path.isfile(os.path.join(ref, "src", "asset.cpp")):
        targets.append("ref")
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "REF=" + ref] + targets, verbose)


if __name__ == "__main__":
    verbose = "-v" in sys.argv
    build_library(verbose=verbose, force="--force" in sys.argv)
    if "--all" in sys.argv:
        build_oracle(verbose=verbose)
    print(LIB)
