"""Build libedgpu.so (the sm_100a engine) in-tree with nvcc.

Usage: python ed_lattice_b200/build.py [--force]   (by path: the package import needs the library)

The library is written next to this file so that it travels with the source tree;
ed_lattice_b200/_edgpu_lib.py loads it from there and fails loudly when it is missing.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libedgpu.so")
BUILD_DIR = os.path.join(HERE, "_build")

SOURCES = ["basis.cu", "hxv.cu", "vecops.cu", "lanczos.cu", "excite.cu", "capi.cu", "noalloc.cu", "lowest.cu", "evalgrid.cu", "chains.cu", "tridiag_host.cpp"]
HEADERS = ["common.cuh", "reduce.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "edgpu.h")]
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", path, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [nvcc(), "-x", "cu", *ARCH, *NVCC_FLAGS, "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        # export only the edg_* C ABI: the version script hides everything else
        vs = os.path.join(BUILD_DIR, "exports.map")
        with open(vs, "w") as f:
            f.write("{ global: edg_*; local: *; };\n")
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-Xlinker", "--version-script=" + vs, "-lcudart_static",
               "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
