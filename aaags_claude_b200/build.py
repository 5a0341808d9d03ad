"""Builds libgs3d_cuda.so (the sm_100a kernels + the gs3dc_* C ABI) in-tree.

    python -m aaags_claude_b200.build [--force] [--verbose]

nvcc cross-compiles for sm_100a without a GPU.  plain.cu is compiled with
-fmad=false (no FMA contraction) and IEEE division / square root, the
floating-point contract of the reference's -ffp-contract=off build; host code
gets -ffp-contract=off for the same reason.  The static CUDA runtime is linked
in, so the library needs only the driver at run time.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libgs3d_cuda.so")
HOST = os.path.join(PKG, "host")
ADAPTERS_OBJ = os.path.join(BUILD, "gs3d_stages_cuda.o")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", f"-I{INCLUDE}"]
# per-source extra flags
SOURCES = {
    "plain.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"],
    "raster_bwd.cu": [],   # gradients: FMA contraction allowed
    "chosen.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],   # reduced-storage form: fast math
    "density.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"],   # density control: reference rounding
    "sort.cu": [],
    "sort_static.cu": [],
    "capi.cu": [],
    "io.cpp": [],   # file formats (host code, -ffp-contract=off like the reference)
}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _newest(paths) -> float:
    return max((os.path.getmtime(p) for p in paths if os.path.exists(p)), default=0.0)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    hdr_time = _newest(headers)
    objs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    # C++ stage adapters (host/): compiled here so that a broken adapter fails the build; callers
    # compile gs3d_stages_cuda.cpp into their own program and link libgs3d_cuda.so
    src = os.path.join(HOST, "gs3d_stages_cuda.cpp")
    deps = [src] + glob.glob(os.path.join(HOST, "*.hpp")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    if force or not os.path.exists(ADAPTERS_OBJ) or os.path.getmtime(ADAPTERS_OBJ) < _newest(deps):
        cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", "-fPIC", f"-I{INCLUDE}", f"-I{HOST}",
               "-c", src, "-o", ADAPTERS_OBJ]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
