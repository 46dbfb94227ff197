"""Build libhh_cuda.so in-tree for sm_100a with nvcc (no JIT, no torch extension).

The library is plain C ABI (include/hh_cuda.h); this module only drives nvcc.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libhh_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --split-compile=0: nvcc optimises the unit's kernels on every host core in parallel
# (the register allocation of the trajectory kernels is the same as a serial build's)
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-O3", "--split-compile=0"]

# translation units and their extra flags; the sampler keeps the reference's
# arithmetic order (no FMA contraction) so initial conditions match it closely
UNITS = [
    ("hh_api.cu", []),
    ("hh_sampler.cu", ["-fmad=false"]),
]
# host-only units (the host compiler sees the generated tables as plain arrays)
HOST_UNITS = ["hh_n2ar_host.cpp", "hh_ch4co2_host.cpp", "hh_writers.cpp"]
CXX = os.environ.get("CXX", "g++")


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh", ".h", ".cpp")):
            out.append(os.path.join(CSRC, f))
    out.append(os.path.join(os.path.dirname(PKG), "include", "hh_cuda.h"))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    for src, flags in UNITS:
        obj = os.path.join(LIBDIR, src.replace(".cu", ".o"))
        # whole-program compilation per unit (no relocatable device code: the units
        # share no device functions), so ptxas allocates the registers of the
        # out-of-line device functions within their callers' limits
        cmd = [NVCC, *ARCH, *COMMON, *flags, *(extra or []), "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    for src in HOST_UNITS:
        obj = os.path.join(LIBDIR, src.replace(".cpp", ".o"))
        cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
