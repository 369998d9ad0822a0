"""Build recipe of libtbpm_b200.so (the CUDA extension of tbplas_b200).

The library is compiled in-tree for sm_100a only, with nvcc, from the sources
under tbplas_b200/csrc, and placed next to this file so that it travels with
the package.  Usage::

    python -m tbplas_b200.build          # build if out of date
    python -m tbplas_b200.build --force  # rebuild
"""

import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
INCLUDE = os.path.join(ROOT_DIR, "include")
LIB_PATH = os.path.join(PKG_DIR, "libtbpm_b200.so")

SOURCES = ["tbpm_engine.cu", "tbpm_capi.cu", "tbpm_noalloc.cu", "tbpm_nn.cu",
           "tbpm_supercell.cu", "tbpm_nn_tc.cu", "tbpm_analysis.cu"]
HEADERS = ["tbpm_common.cuh", "tbpm_kernels.cuh", "tbpm_ring_kernels.cuh", "tbpm_pq_gemm.cuh",
           "tbpm_pair_kernels.cuh",
           "tbpm_dc_kernels.cuh",
           "tbpm_seg_kernels.cuh",
           "tbpm_more_kernels.cuh", "tbpm_scan.cuh",
           "tbpm_engine.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
    "-shared",
]


def nvcc_path() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "tbpm_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB_PATH):
        return False
    t_lib = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(f) <= t_lib for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile libtbpm_b200.so for sm_100a; return its path."""
    if not force and up_to_date():
        return LIB_PATH
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc_path()] + NVCC_FLAGS + ["-I" + INCLUDE, "-I" + CSRC, "-o", tmp]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
