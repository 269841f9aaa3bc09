"""Build recipe for the CUDA library of difftetvr_b200 (sm_100a).

Compiles the kernels and the C ABI into ``difftetvr_b200/libdifftetvr_b200.so``
in-tree with nvcc.  The library has no torch dependency; Python binds it with
ctypes (``difftetvr_b200._lib``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_NAME = "libdifftetvr_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)

SOURCES = ["dtv_api.cu", "dtv_kernels.cu", "dtv_mesh.cpp", "dtv_noalloc.cu", "dtv_batch.cu", "dtv_raytet.cu", "dtv_regularizer.cu", "dtv_io.cpp", "dtv_cells.cu", "dtv_split.cpp"]
HEADERS = ["dtv_types.h", "dtv_device.cuh", "dtv_segment.cuh", "dtv_internal.h", "dtv_host.h", "dtv_path.cuh"]

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC,-fopenmp,-O3",
    "-shared",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(ROOT, "include", "difftetvr_b200.h"))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if any source is newer than it; return its path."""
    if not force and up_to_date():
        return LIB_PATH
    env = dict(os.environ)
    # nvcc's host compiler: the system g++ (an OpenMP-capable toolchain).
    env.pop("CC", None)
    env.pop("CXX", None)
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    cmd += ["-o", LIB_PATH + ".tmp", "-lgomp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose and (res.stdout or res.stderr):
        print(res.stdout, res.stderr, file=sys.stderr)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
