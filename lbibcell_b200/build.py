"""Builds liblbibcuda.so in-tree with nvcc for sm_100a.

The FP64 (parity) translation units are compiled with --fmad=false so that no
multiply-add contraction changes a rounding relative to the reference's
double-precision build; the FP32-shifted lattice kernels keep FMA.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblbibcuda.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(os.path.dirname(HERE), "include")]
UNITS = [
    ("k_lattice64.cu", ["--fmad=false"]),
    ("k_membrane.cu", ["--fmad=false"]),
    ("k_topology.cu", ["--fmad=false"]),
    ("k_forces.cu", ["--fmad=false"]),
    ("lbib_host.cu", ["--fmad=false"]),
    ("k_lattice32.cu", []),
    ("k_adjoint.cu", []),
    ("vtk_io.cu", []),
]


def sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(os.path.dirname(HERE), "include", "lbibcell.h"), __file__]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src, flags in UNITS:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [NVCC] + ARCH + COMMON + flags + list(extra) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
        "-Xcompiler", "-static-libstdc++", "-Xlinker", "--exclude-libs,ALL", "-Xlinker", "-Bsymbolic", "-Xlinker", "--no-undefined",
        "-cudart", "static"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a.startswith("-X")])
