"""Compiles tests/cpp/cabi_classes.cpp (the check program of the C++ classes in
include/difftetvr_b200.hpp) against the public headers and the in-tree
libdifftetvr_b200.so, into tests/cpp/_build/cabi_classes."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SRC = os.path.join(HERE, "cabi_classes.cpp")
OUT = os.path.join(HERE, "_build", "cabi_classes")
HEADERS = [os.path.join(ROOT, "include", h) for h in ("difftetvr_b200.h", "difftetvr_b200.hpp")]
LIB = os.path.join(ROOT, "difftetvr_b200", "libdifftetvr_b200.so")


def build() -> str:
    inputs = [SRC, LIB] + HEADERS
    if os.path.exists(OUT) and all(os.path.getmtime(f) <= os.path.getmtime(OUT) for f in inputs):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    nvcc = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    cmd = [nvcc, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", os.path.dirname(LIB), "-ldifftetvr_b200",
           "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../../../difftetvr_b200", "-o", OUT + ".tmp"]
    res = subprocess.run(cmd, env=env, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"building the C++ check program failed:\n{res.stdout}\n{res.stderr}")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build())
