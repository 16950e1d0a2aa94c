"""Builds libbfgt_b200.so in-tree (CUDA for sm_100a, host code with g++/OpenMP).

The library is written to heat2d_per_box_b200/lib/ and loaded from there, so
that the same file ships with the source tree and is the one every caller
loads.  Rebuilds only when a source is newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
BUILD = PKG / "_build"
LIB = LIBDIR / "libbfgt_b200.so"
INCLUDE = PKG.parent / "include"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["fgt_device.cu", "split_kernels.cu", "split_fix.cu", "near_tc.cu", "noalloc.cu"]
CPP_SOURCES = ["host_plan.cpp", "tree_build.cpp", "capi.cpp"]


def _sources():
    return [CSRC / s for s in CU_SOURCES + CPP_SOURCES] + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [
        INCLUDE / "bfgt.h"
    ]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(str(c) for c in cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compile every CUDA and host source and link the shared library."""
    if not force and not _stale(LIB, _sources()):
        return LIB
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    cmds, objs = [], []
    for s in CU_SOURCES:
        o = BUILD / (s + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
               "--expt-relaxed-constexpr", "-c", CSRC / s, "-o", o]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(o)
    for s in CPP_SOURCES:
        o = BUILD / (s + ".o")
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
               "-I", os.path.join(CUDA_HOME, "include"), "-I", INCLUDE, "-c", CSRC / s, "-o", o]
        cmds.append(cmd)
        objs.append(o)
    # the translation units compile independently: in parallel
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for f in [ex.submit(_run, c, verbose or ptxas_verbose) for c in cmds]:
            f.result()
    tmp = LIB.with_suffix(".so.tmp")
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-Xcompiler", "-fopenmp", "-lgomp"],
         verbose)
    os.replace(tmp, LIB)
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    if LIB.exists():
        LIB.unlink()


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
