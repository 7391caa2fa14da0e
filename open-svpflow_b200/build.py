"""Builds libsvpflow_b200.so (sm_100a) in-tree: open-svpflow_b200/lib/.

    python open-svpflow_b200/build.py [--verbose]

nvcc compiles the CUDA kernels and the host C++ (options, C ABI) into one shared
library with the CUDA runtime linked statically, so the library has no dependency
beyond the driver. `-Xptxas -v` output (registers, spills, shared memory) goes to
lib/ptxas.log.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
CORE = os.path.join(LIB_DIR, "libsvpflow_b200.so")
SOURCES = ["analyse.cu", "super.cu", "opts.cpp", "capi.cpp", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-v", "-cudart", "static",
         "--diag-suppress", "177"]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "svpflow_b200.h")]
    if force or _stale(CORE, deps):
        cmd = ["nvcc", *ARCH, *FLAGS, "-shared", "-o", CORE] + [os.path.join(CSRC, s) for s in SOURCES]
        r = subprocess.run(cmd, capture_output=True, text=True)
        with open(os.path.join(LIB_DIR, "ptxas.log"), "w") as f:
            f.write(r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed building libsvpflow_b200.so")
        if verbose:
            print(r.stdout + r.stderr)
    return CORE


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(CORE)
