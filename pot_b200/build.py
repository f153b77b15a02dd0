"""Build the sm_100a CUDA library ``pot_b200/libpotgpu.so`` (in-tree).

nvcc compiles every ``csrc/*.cu`` for ``arch=compute_100a,code=sm_100a`` (no
PTX fallback, no other architecture) and links them into one shared library
exporting the C ABI declared in ``include/pot_gpu.h``.  It cross-compiles on
a machine without a GPU.

Usage: ``python -m pot_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libpotgpu.so")
BUILD_DIR = os.path.join(PKG, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: a multiply and an add written separately stay two roundings
# (fused multiply-adds are written as fma() where they are meant), so no
# result depends on how the compiler contracts one kernel or another: a run
# stepped by its own kernels and by a packed batch's gives the same bits.
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-fmad=false", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall", "-Xcudafe", "--diag_suppress=177"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + \
        sorted(glob.glob(os.path.join(CSRC, "*.h"))) + [os.path.join(INCLUDE, "pot_gpu.h"), __file__]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in _deps())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ["-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, p.stdout, p.stderr))
        if verbose or ptxas_info:
            sys.stdout.write(p.stdout + p.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (p.stdout, p.stderr))
    os.replace(tmp, LIB)
    return LIB


HOST_PROGRAMS = {"potgpu": os.path.join(PKG, "host", "potgpu.c"),      # pot's command line and files
                 "potserve": os.path.join(PKG, "host", "potserve.c")}  # batched sweep and serving loop
HOST_BIN = os.path.join(PKG, "potgpu")
SERVE_BIN = os.path.join(PKG, "potserve")


def build_host(force: bool = False) -> str:
    """The C host programs, linked to libpotgpu.so with an $ORIGIN run path;
    returns the path of potgpu."""
    lib = build()
    cc = shutil.which("gcc") or "gcc"
    for name, src in HOST_PROGRAMS.items():
        out = os.path.join(PKG, name)
        deps = [src, lib, os.path.join(INCLUDE, "pot_gpu.h")]
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
            continue
        tmp = out + ".tmp%d" % os.getpid()
        cmd = [cc, "-O2", "-std=c99", "-Wall", "-Wextra", "-Wno-unused-parameter", "-I", INCLUDE, src, "-o", tmp,
               "-L", PKG, "-lpotgpu", "-Wl,-rpath,$ORIGIN", "-lm"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("gcc failed for %s:\n%s%s" % (src, p.stdout, p.stderr))
        os.replace(tmp, out)
    return HOST_BIN


def main(argv=None):
    ap = argparse.ArgumentParser(description="build libpotgpu.so for sm_100a")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info))
    print(build_host(force=a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
