"""ctypes wrapper of the CPU oracle (liboracle.so) and reader of the reference
build's dumps (oracle/_ref/ref_driver).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
``bench.py``'s cpu_baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")
REF_DRIVER_FAST = os.path.join(HERE, "_ref", "ref_driver_fast")
# the reference built with GuoZhengShi2002ForceModel as FluidSolver's base class
REF_DRIVER_GUO = os.path.join(HERE, "_ref", "ref_driver_guo")
# apps/tutorial_01.cpp and tutorial_02.cpp of the reference, unmodified, built
# against lbibcell_b200's drop-in libLbmLib
REF_APPS = os.path.join(HERE, "_ref", "apps")
# Root of the reference's source tree (read only by the build recipe and by
# tests that use its files where they are present): one environment variable.
REFERENCE = os.environ.get("LBIB_REFERENCE", "/root/reference")


def reference_present() -> bool:
    return os.path.isdir(os.path.join(REFERENCE, "libs"))

_lib = None


def build(ref: bool = False) -> None:
    """Compile the oracle (and, with ``ref``, the reference build and the
    reference's applications against the drop-in library) via oracle/Makefile."""
    targets = ["oracle"] + (["ref", "apps"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE, "-j8", "REF=" + REFERENCE] + targets, check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        c_p, c_d, c_i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        L.orc_create.restype = c_p
        L.orc_create.argtypes = [ctypes.c_char_p] * 4
        L.orc_destroy.argtypes = [c_p]
        L.orc_error.restype = c_i
        L.orc_error.argtypes = [c_p, ctypes.c_char_p, c_i]
        L.orc_step.restype = c_i
        L.orc_step.argtypes = [c_p, c_i]
        L.orc_sizes.argtypes = [c_p, ctypes.c_void_p]
        L.orc_get_lattice.argtypes = [c_p] + [ctypes.c_void_p] * 7
        L.orc_get_membrane.argtypes = [c_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_get_connections.argtypes = [c_p, ctypes.c_void_p]
        L.orc_areas.restype = c_i
        L.orc_areas.argtypes = [c_p, ctypes.c_void_p, ctypes.c_void_p, c_i]
        L.orc_set_lattice.argtypes = [c_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_lattice_step.restype = c_i
        L.orc_lattice_step.argtypes = [c_p, c_i, c_i]
        L.orc_fastcos.restype = c_d
        L.orc_fastcos.argtypes = [c_d]
        L.orc_delta.restype = c_d
        L.orc_delta.argtypes = [c_d, c_d]
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class State:
    """One snapshot of the simulation, in the reference's layout."""

    t: int
    nx: int
    ny: int
    S: int
    current_iteration: int
    f: np.ndarray        # (L, 9) slot convention
    g: np.ndarray        # (S, L, 5)
    vel: np.ndarray      # (L, 2)
    force: np.ndarray    # (L, 2)
    dom: np.ndarray      # (L,) uint32
    ctype: np.ndarray    # (L,) uint32
    ids: np.ndarray      # (M,) uint32
    node: np.ndarray     # (M, 6) x, y, vx, vy, fx, fy
    conn: np.ndarray     # (C, 3) id1, id2, domain
    counters: Optional[np.ndarray] = None


class Oracle:
    """The CPU restatement of the reference time loop."""

    def __init__(self, paths: Dict[str, str]):
        self.L = lib()
        self.h = self.L.orc_create(paths["parameters"].encode(), paths["geometry"].encode(),
                                   paths.get("force", "").encode(), paths.get("plugins", "").encode())
        self.check()

    def check(self) -> None:
        buf = ctypes.create_string_buffer(512)
        err = self.L.orc_error(self.h, buf, 512)
        if err:
            raise RuntimeError(f"oracle error {err}: {buf.value.decode()}")

    def error(self):
        buf = ctypes.create_string_buffer(512)
        return self.L.orc_error(self.h, buf, 512), buf.value.decode()

    def close(self) -> None:
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1, check: bool = True) -> int:
        rc = self.L.orc_step(self.h, n)
        if check and rc:
            self.check()
        return rc

    def lattice_step(self, n: int = 1, outlet: bool = True) -> None:
        self.L.orc_lattice_step(self.h, n, 1 if outlet else 0)

    def sizes(self):
        s = np.zeros(8, dtype=np.int64)
        self.L.orc_sizes(self.h, _ptr(s))
        return s

    def state(self) -> State:
        nx, ny, S, M, C, it, _, _ = (int(v) for v in self.sizes())
        L = nx * ny
        f = np.zeros((L, 9)); g = np.zeros((S, L, 5)); vel = np.zeros((L, 2)); force = np.zeros((L, 2))
        dom = np.zeros(L, np.uint32); ctype = np.zeros(L, np.uint32); rta = np.zeros(L)
        self.L.orc_get_lattice(self.h, _ptr(f), _ptr(g), _ptr(vel), _ptr(force), _ptr(dom), _ptr(ctype), _ptr(rta))
        ids = np.zeros(M, np.uint32); node = np.zeros((M, 6))
        self.L.orc_get_membrane(self.h, _ptr(ids), _ptr(node))
        conn = np.zeros((C, 3), np.uint32)
        self.L.orc_get_connections(self.h, _ptr(conn))
        st = State(it, nx, ny, S, it, f, g, vel, force, dom, ctype, ids, node, conn)
        st.rho_to_add = rta
        return st

    def set_lattice(self, f=None, g=None, force=None) -> None:
        self.L.orc_set_lattice(self.h, _ptr(None if f is None else np.ascontiguousarray(f, np.float64)),
                               _ptr(None if g is None else np.ascontiguousarray(g, np.float64)),
                               _ptr(None if force is None else np.ascontiguousarray(force, np.float64)))

    def areas(self) -> Dict[int, float]:
        cap = 1 << 16
        d = np.zeros(cap, np.uint32); a = np.zeros(cap)
        n = self.L.orc_areas(self.h, _ptr(d), _ptr(a), cap)
        return {int(d[i]): float(a[i]) for i in range(n)}


def read_dump(path: str) -> State:
    """Read one dump written by oracle/_ref/ref_driver."""
    raw = open(path, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a.copy()

    hdr = take(np.int64, 8)
    assert hdr[0] == 0x4C424942, "not a reference dump"
    t, nx, ny, S, M, C, it = (int(v) for v in hdr[1:])
    L = nx * ny
    f = take(np.float64, L * 9).reshape(L, 9)
    g = take(np.float64, S * L * 5).reshape(S, L, 5)
    vel = take(np.float64, L * 2).reshape(L, 2)
    force = take(np.float64, L * 2).reshape(L, 2)
    dom = take(np.uint32, L)
    ctype = take(np.uint32, L)
    ids = take(np.uint32, M)
    node = take(np.float64, M * 6).reshape(M, 6)
    conn = take(np.uint32, C * 3).reshape(C, 3)
    counters = take(np.int64, 2)
    return State(t, nx, ny, S, it, f, g, vel, force, dom, ctype, ids, node, conn, counters)


def run_reference(paths: Dict[str, str], outdir: str, driver: str = REF_DRIVER, timeout: float = 3600,
                  extra=()) -> Dict[int, State]:
    """Run the reference build on a configuration; returns its dumps by time.
    ``extra``: further driver arguments ("restart", solver file; "write", prefix)."""
    os.makedirs(outdir, exist_ok=True)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run([driver, paths["parameters"], paths["geometry"], paths["force"], paths["plugins"], outdir]
                       + [str(a) for a in extra],
                       cwd=outdir, env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed: {r.stderr}{r.stdout}")
    out = {}
    for fn in os.listdir(outdir):
        if fn.startswith("dump_") and fn.endswith(".bin"):
            st = read_dump(os.path.join(outdir, fn))
            out[st.t] = st
    out["stdout"] = r.stdout
    return out
