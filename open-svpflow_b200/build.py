"""Builds libsvpflow_b200.so (sm_100a) in-tree: open-svpflow_b200/lib/.

    python open-svpflow_b200/build.py [--verbose]

nvcc compiles each CUDA / C++ source to an object (in parallel) and links them into one
shared library with the CUDA runtime linked statically, so the library has no
dependency beyond the driver. `-Xptxas -v` output (registers, spills, shared memory)
goes to lib/ptxas.log.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
CORE = os.path.join(LIB_DIR, "libsvpflow_b200.so")
SOURCES = ["analyse_nt128.cu", "analyse_nt64.cu", "analyse_nt32.cu", "analyse_nt128b3.cu", "analyse_nt64b6.cu",
           "analyse_nt128p16.cu", "variants.cpp", "params.cpp", "super.cu", "opts.cpp", "capi.cpp", "noalloc.cu",
           "batch.cpp", "serve.cpp", "vectors.cu", "render.cu"]
OBJ_DIR = os.path.join(LIB_DIR, "obj")
# the VapourSynth plugin: the reference plugin's exports over the same objects
VS_PLUGIN = os.path.join(LIB_DIR, "libsvpflow1_vs.so")
VS_SOURCES = ["vs_plugin.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-v", "-cudart", "static",
         "--diag-suppress", "177"]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str):
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    cmd = ["nvcc", *ARCH, *FLAGS, "-c", "-o", obj, src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return obj, r.returncode, r.stdout + r.stderr


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "svpflow_b200.h")]
    if force or _stale(CORE, deps) or _stale(VS_PLUGIN, deps):
        srcs = [os.path.join(CSRC, s) for s in SOURCES + VS_SOURCES]
        with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
            results = list(ex.map(_compile, srcs))
        log = "".join(f"==== {os.path.basename(o)}\n{out}" for o, _, out in results)
        bad = [o for o, rc, _ in results if rc != 0]
        core_objs = [o for o, _, _ in results[:len(SOURCES)]]
        vs_objs = [o for o, _, _ in results[len(SOURCES):]]
        for target, objs in ((CORE, core_objs), (VS_PLUGIN, core_objs + vs_objs)):
            if bad:
                break
            cmd = ["nvcc", *ARCH, "-shared", "-cudart", "static", "-o", target] + objs
            r = subprocess.run(cmd, capture_output=True, text=True)
            log += f"==== link {os.path.basename(target)}\n" + r.stdout + r.stderr
            if r.returncode != 0:
                bad = ["link " + os.path.basename(target)]
        with open(os.path.join(LIB_DIR, "ptxas.log"), "w") as f:
            f.write(log)
        if bad:
            sys.stderr.write(log)
            raise RuntimeError(f"nvcc failed building libsvpflow_b200.so: {bad}")
        if verbose:
            print(log)
    return CORE


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(CORE)
