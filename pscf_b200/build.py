"""Build the engine library libpscfgpu.so with nvcc for sm_100a.

The library is built in-tree (pscf_b200/_lib/) so that it travels with the
working tree.  Usage: python -m pscf_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libpscfgpu.so")
SOURCES = ["engine.cu", "noalloc.cu"]
# compiled on their own, with extra flags: the graph-driven Anderson control
# kernels round as the host iteration does only without multiply-add
# contraction
SEPARATE = {"am_graph.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, extra=()) -> str:
    import tempfile
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    common = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC"]
    with tempfile.TemporaryDirectory() as tmp:
        objs = []
        for name, flags in SEPARATE.items():
            obj = os.path.join(tmp, name.replace(".cu", ".o"))
            cmd = [nvcc(), *common, *flags, "-c", "-o", obj, os.path.join(CSRC, name), *extra]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            objs.append(obj)
        cmd = [nvcc(), *common, "-shared", "-o", LIB, *srcs, *objs, *extra]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
