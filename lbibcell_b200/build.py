"""Builds liblbibcuda.so in-tree with nvcc for sm_100a.

The FP64 (parity) translation units are compiled with --fmad=false so that no
multiply-add contraction changes a rounding relative to the reference's
double-precision build; the FP32-shifted lattice kernels keep FMA.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblbibcuda.so")
# LBIBCell's C++ application API (SimulationRunner, GeometryHandler, plugin
# registries, reporters) over the C ABI: apps written against the reference
# compile against dropin/include and link this library
DROPIN_LIB = os.path.join(HERE, "libLbmLib.so")
DROPIN = os.path.join(HERE, "dropin")
CXX = os.environ.get("CXX", "g++")
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


def dropin_sources():
    out = []
    for root, _, files in os.walk(DROPIN):
        out += [os.path.join(root, f) for f in files if f.endswith((".cpp", ".hpp"))]
    return out


def build_dropin(force: bool = False) -> str:
    """libLbmLib.so: the drop-in C++ host layer, linked against liblbibcuda.so
    (found next to it at run time)."""
    deps = dropin_sources() + [LIB, os.path.join(os.path.dirname(HERE), "include", "lbibcell.h"), __file__]
    if not force and os.path.exists(DROPIN_LIB) and all(os.path.getmtime(d) <= os.path.getmtime(DROPIN_LIB)
                                                         for d in deps):
        return DROPIN_LIB
    srcs = sorted(f for f in dropin_sources() if f.endswith(".cpp"))
    cmd = [CXX, "-std=gnu++11", "-O2", "-fPIC", "-shared", "-Wall", "-I" + os.path.join(DROPIN, "include"),
           "-I" + os.path.join(os.path.dirname(HERE), "include")] + srcs + [
        "-L" + HERE, "-llbibcuda", "-Wl,-rpath,$ORIGIN", "-o", DROPIN_LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(DROPIN_LIB + ".tmp", DROPIN_LIB)
    return DROPIN_LIB


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and up_to_date():
        build_dropin()
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    jobs = []
    for src, flags in UNITS:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [NVCC] + ARCH + COMMON + flags + list(extra) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        jobs.append((cmd, obj))
    # the translation units compile independently: one nvcc per unit at a time
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for r in [pool.submit(subprocess.run, cmd, check=True) for cmd, _ in jobs]:
            r.result()
    objs = [obj for _, obj in jobs]
    # linked beside the library and renamed over it: a process that has the
    # old one loaded keeps its mapping, and no reader sees a partial file
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + [
        "-Xcompiler", "-static-libstdc++", "-Xlinker", "--exclude-libs,ALL", "-Xlinker", "-Bsymbolic", "-Xlinker", "--no-undefined",
        "-cudart", "static"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_dropin(force=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a.startswith(("-X", "-D"))])
