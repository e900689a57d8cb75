"""Builds libmfixdem.so for sm_100a with nvcc (no GPU needed).

    python mfix-cfd-dem_b200/build.py [--force] [--verbose]

Objects go to mfix-cfd-dem_b200/_build/, the library to
mfix-cfd-dem_b200/lib/libmfixdem.so.  The FP64 parity kernels are compiled
with -fmad=false so that every expression rounds like the Fortran reference;
the split-precision kernels keep FMA contraction.
"""
import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libmfixdem.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", str(INCLUDE), "-I", str(CSRC)]

# per-source extra flags
SOURCES = {
    "capi.cu": ["-fmad=false"],
    "scan.cu": [],
    "desgrid.cu": ["-fmad=false"],
    "neighbor.cu": ["-fmad=false"],
    "force.cu": ["-fmad=false"],
    "force_split.cu": ["-fmad=true", "-use_fast_math"],
    "walls.cu": ["-fmad=false"],
    "coupling.cu": ["-fmad=false"],
    "batch.cu": ["-fmad=false"],
    "tune.cu": [],
    "res_des.cu": [],
    "vtp.cu": [],
    "outflow.cu": ["-fmad=false"],
    "inflow.cu": ["-fmad=false"],
}
HEADERS = ["dem_internal.cuh"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(force=False, verbose=False):
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    hdr_mtime = max((CSRC / h).stat().st_mtime for h in HEADERS)
    hdr_mtime = max(hdr_mtime, (INCLUDE / "dem_b200.h").stat().st_mtime)
    objs = []
    changed = force
    for src, extra in SOURCES.items():
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if (not force and o.exists() and o.stat().st_mtime >= s.stat().st_mtime
                and o.stat().st_mtime >= hdr_mtime and o.stat().st_mtime >= Path(__file__).stat().st_mtime):
            continue
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", str(s), "-o", str(o)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        changed = True
    if changed or not LIB.exists():
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
