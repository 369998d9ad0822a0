"""Build recipe of the CPU oracle (test infrastructure only).

Compiles oracle/tbpm_oracle.cpp with g++ -O3 -march=native -fopenmp (the flags
of the reference's GNU build, pyproject.toml / config/gnu.cfg) into
oracle/libtbpm_oracle.so.  The reference Fortran itself is not built: no
Fortran compiler is available, so there is no oracle/_ref.
"""

import os
import subprocess
import sys

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(ORACLE_DIR, "tbpm_oracle.cpp")
LIB = os.path.join(ORACLE_DIR, "libtbpm_oracle.so")


NATIVE_LIB = os.path.join(ORACLE_DIR, "libtbpm_oracle_native.so")


def build(force: bool = False, native: bool = False) -> str:
    """Build the oracle library.  The default build targets the portable
    x86-64-v2 baseline (it is built here and runs on other hosts); native=True
    builds with -march=native for timing on the machine that runs it."""
    lib = NATIVE_LIB if native else LIB
    if not force and os.path.exists(lib) and os.path.getmtime(lib) >= os.path.getmtime(SRC):
        return lib
    tmp = lib + ".tmp"
    march = "-march=native" if native else "-march=x86-64-v2"
    cmd = ["g++", "-O3", march, "-fopenmp", "-fPIC", "-shared", "-std=c++17",
           "-fno-fast-math", "-ffp-contract=off", SRC, "-o", tmp]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
