"""Builds libarepo_gpugrav.so in-tree for sm_100a (B200).

The parity translation units (domain, tree, walk64, direct) are compiled with
-fmad=false so that every double operation rounds like the reference's plain
C; the FP32 walk keeps fused multiply-adds.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libarepo_gpugrav.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_LIB = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")  # cuFFT (PM long-range force)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-I", INCLUDE, "-I", CSRC]

# (source, exact-double?)
SOURCES = [
    ("domain.cu", True),
    ("tree.cu", True),
    ("walk64.cu", True),
    ("direct.cu", True),
    ("direct_noalloc.cu", True),
    ("walk32.cu", False),
    ("targets.cu", False),
    ("timestep.cu", True),
    ("peak.cu", False),
    ("serve.cu", False),
    ("pm.cu", False),
    ("ewald.cu", True),
    ("gpugrav.cu", True),
]


def _needs(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "gpugrav.h"))
    objs = []
    for src, exact in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _needs(o, [s] + headers):
            cmd = [NVCC] + ARCH + COMMON + (["-fmad=false"] if exact else []) + (extra or []) + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.check_call(cmd)
    if force or _needs(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-L" + CUDA_LIB, "-lcufft",
                                                              "-Xlinker", "-rpath," + CUDA_LIB]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
