"""Build ``pyftle_b200/libpyftle_b200.so`` with nvcc for sm_100a (in-tree).

Each CUDA source is compiled on its own so it can carry its own FP flags:
``plain_f64.cu`` is built with ``-fmad=false`` (no FMA contraction: the FP64
path reproduces pyFTLE's rounding step by step), and so is ``mixed.cu``: every
FMA it intends is written as ``fmaf``/``fma``, so its results do not depend on
where the compiler would otherwise fuse a product into a sum.  The CUDA runtime is linked
statically so the library has no dependency beyond the driver.

Usage: ``python -m pyftle_b200.build [--force] [--verbose]``.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(REPO, "_build")
LIB = os.path.join(HERE, "libpyftle_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", INCLUDE, "-I", CSRC]
SOURCES = {
    "api.cu": [],
    "plain_f64.cu": ["-fmad=false"],
    "mixed.cu": ["-fmad=false"],
    "no_alloc.cu": [],
    "mlp.cu": [],
    "mlp_fused.cu": [],
    "probe.cu": [],
}
HEADERS = ["common.cuh", "umma.cuh"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pyftle_b200")


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "pyftle_b200.h"),
                                                       __file__]
    dep_time = max(_mtime(d) for d in deps)
    objs = []
    rebuilt = False
    for src, flags in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _mtime(o) < max(_mtime(s), dep_time):
            cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
            rebuilt = True
    if rebuilt or force or not os.path.exists(LIB) or _mtime(LIB) < max(_mtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
