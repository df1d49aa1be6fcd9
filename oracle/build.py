"""Build recipe for the oracle (test infrastructure only).

Two artefacts:

* ``oracle/liboracle.so`` -- the C restatement in ``ftle_oracle.c``
  (gcc, ``-ffp-contract=off`` so no FMA contraction changes rounding, OpenMP
  over particles).
* ``oracle/_ref/ginterp<EXT_SUFFIX>`` -- the reference's own native
  interpolator, ``src/pyftle/grid_interp/GridInterp.cpp`` of pyFTLE,
  compiled straight from the read-only reference tree with the flags of the
  reference's CMakeLists.txt (``-O3``, C++17, pybind11, no ``-march``).
  Only built where the reference tree is present (``$PYFTLE_REFERENCE_ROOT``,
  else a checkout named ``reference`` beside this repository); the built module
  travels with the repository snapshot (``oracle/_ref/`` is git-ignored).

Usage: ``python oracle/build.py [--force]``.
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
# the pyFTLE source tree: $PYFTLE_REFERENCE_ROOT, else a checkout named `reference`
# beside this repository
REF_ROOT = os.environ.get("PYFTLE_REFERENCE_ROOT") or os.path.join(
    os.path.dirname(os.path.dirname(HERE)), "reference")
REF_CPP = os.path.join(REF_ROOT, "src", "pyftle", "grid_interp", "GridInterp.cpp")
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_MOD = os.path.join(REF_DIR, "ginterp" + sysconfig.get_config_var("EXT_SUFFIX"))


def _stale(target: str, *sources: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "ftle_oracle.c")
    if force or _stale(LIB, src, __file__):
        cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
               "-fno-fast-math", src, "-o", LIB + ".tmp", "-lm"]
        subprocess.check_call(cmd)
        os.replace(LIB + ".tmp", LIB)
    return LIB


def build_reference(force: bool = False) -> str | None:
    """Compile the reference GridInterp.cpp into oracle/_ref (if the tree exists)."""
    if not os.path.exists(REF_CPP):
        return REF_MOD if os.path.exists(REF_MOD) else None
    if not (force or _stale(REF_MOD, REF_CPP, __file__)):
        return REF_MOD
    import pybind11

    os.makedirs(REF_DIR, exist_ok=True)
    cmd = ["g++", "-O3", "-std=gnu++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I" + sysconfig.get_paths()["include"], "-I" + pybind11.get_include(),
           REF_CPP, "-o", REF_MOD + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(REF_MOD + ".tmp", REF_MOD)
    return REF_MOD


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_reference(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(LIB)
    print(REF_MOD if os.path.exists(REF_MOD) else "reference module not built (no reference tree)")
