"""Host-side mirror of LBIBCell's simulation interface over the C ABI.

``Simulation`` stands for the objects a reference application builds
(apps/tutorial_01.cpp:59-143): the global ``Parameters``, ``Geometry`` +
``GeometryHandler`` and ``SimulationRunner`` with its mass and bio solvers.  It
is created from the same files the reference reads, plus the plugin file of
lbibcell_b200/configs.py.  Every call goes to liblbibcuda.so; state lives on
the GPU.

Method map (reference -> here):
    SimulationRunner::runSimulation loop body   -> step(n)
    SimulationRunner::writeSimulation solvers   -> lattice() (same slot layout)
    SimulationRunner::initSolvers(file)         -> set_lattice()
    Geometry::getGeometryNodes                  -> membrane()
    Geometry::getConnections                    -> connections()
    GeometryHandler::computeAreas               -> areas()
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, Optional, Tuple

import numpy as np

from ._lib import LbibError, load

FP64 = 0
FP32_SHIFTED = 1


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class LatticeState:
    f: np.ndarray       # (L, 9) reference slot convention
    g: np.ndarray       # (S, L, 5)
    vel: np.ndarray     # (L, 2)
    force: np.ndarray   # (L, 2)
    dom: np.ndarray     # (L,) uint32
    ctype: np.ndarray   # (L,) uint32


class Simulation:
    """One GPU-resident LBIBCell simulation."""

    def __init__(self, paths: Dict[str, str], precision: int = FP64, device: int = 0):
        self._L = load()
        h = ctypes.c_void_p()
        rc = self._L.lbib_create_from_files(paths["parameters"].encode(), paths["geometry"].encode(),
                                            paths.get("force", "").encode(), paths.get("plugins", "").encode(),
                                            int(precision), int(device), ctypes.byref(h))
        self._h = h
        # the arrays of the last per-step calls and their data pointers: a call
        # with the same array (its contents rewritten in place) skips the
        # checks and the pointer lookup
        self._src = (None, None, 0, None)
        self._areas = (None, None, 0, 0, 0)
        if rc:
            err = self._error()
            self.close()
            raise err
        self.precision = precision

    # -- lifetime -------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.lbib_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _error(self) -> LbibError:
        buf = ctypes.create_string_buffer(512)
        idx = ctypes.c_longlong(-1)
        code = self._L.lbib_last_error(self._h, buf, 512, ctypes.byref(idx))
        return LbibError(code, buf.value.decode(), idx.value)

    def _check(self, rc: int) -> None:
        if rc:
            raise self._error()

    # -- stepping -------------------------------------------------------------
    def step(self, n: int = 1) -> None:
        """n iterations of SimulationRunner::runSimulation's loop body."""
        self._check(self._L.lbib_step(self._h, int(n)))

    def lattice_step(self, n: int = 1, outlet: bool = True) -> None:
        """n stream-collide steps with the geometry, forces and domains fixed."""
        self._check(self._L.lbib_lattice_step(self._h, int(n), 1 if outlet else 0))

    def set_species_source(self, k: int, rates: np.ndarray) -> None:
        """Per-domain production rate of species k (index = domain id)."""
        r = np.ascontiguousarray(rates, np.float64)
        self._check(self._L.lbib_set_species_source(self._h, int(k), _p(r), int(r.size)))

    def set_species_sources(self, rates: np.ndarray) -> None:
        """Every species' per-domain production rate at once ((S, n_domains)),
        one host-to-device copy; pinned host memory makes it asynchronous."""
        ref, ptr, n, shape = self._src
        if rates is not ref or rates.shape != shape:
            r = np.ascontiguousarray(rates, np.float64)
            n = int(r.shape[-1]) if r.ndim else 0
            ptr = r.ctypes.data
            if r is rates:
                self._src = (r, ptr, n, r.shape)
        self._check(self._L.lbib_set_species_sources(self._h, ptr, n))

    def set_profiling(self, on: bool) -> None:
        self._check(self._L.lbib_set_profiling(self._h, 1 if on else 0))

    def last_timing(self) -> Dict[str, float]:
        out = np.zeros(4)
        self._check(self._L.lbib_last_timing(self._h, _p(out)))
        return {"total_ms": float(out[0]), "collide_ms": float(out[1]), "collide_launches": int(out[2]),
                "launches": int(out[3])}

    # -- state ----------------------------------------------------------------
    def sizes(self) -> Dict[str, int]:
        s = np.zeros(10, np.int64)
        self._check(self._L.lbib_get_sizes(self._h, _p(s)))
        keys = ("nx", "ny", "S", "M", "C", "iteration", "precision", "host_events", "steps", "cells")
        return {k: int(v) for k, v in zip(keys, s)}

    def lattice(self) -> LatticeState:
        z = self.sizes()
        L, S = z["nx"] * z["ny"], z["S"]
        f = np.zeros((L, 9)); g = np.zeros((S, L, 5)); vel = np.zeros((L, 2)); force = np.zeros((L, 2))
        dom = np.zeros(L, np.uint32); ctype = np.zeros(L, np.uint32)
        self._check(self._L.lbib_download_lattice(self._h, _p(f), _p(g), _p(vel), _p(force), _p(dom), _p(ctype)))
        return LatticeState(f, g, vel, force, dom, ctype)

    def set_lattice(self, f=None, g=None, force=None) -> None:
        args = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (f, g, force)]
        self._check(self._L.lbib_upload_lattice(self._h, *[_p(a) for a in args]))

    def init_velocity(self, ux: float, uy: float) -> None:
        """SimulationRunner::initSolvers(Field<double>): the lattice at the
        equilibrium of the uniform velocity (ux, uy)."""
        self._check(self._L.lbib_init_velocity(self._h, float(ux), float(uy)))

    def membrane(self):
        """(ids[M], state[M, 6]) with state = x, y, vx, vy, fx, fy, in id order."""
        M = self.sizes()["M"]
        ids = np.zeros(M, np.uint32); st = np.zeros((M, 6))
        self._check(self._L.lbib_download_membrane(self._h, _p(ids), _p(st)))
        return ids, st

    def connections(self) -> np.ndarray:
        C = self.sizes()["C"]
        c = np.zeros((C, 3), np.uint32)
        self._check(self._L.lbib_download_connections(self._h, _p(c)))
        return c

    def areas(self) -> Dict[int, float]:
        """GeometryHandler::computeAreas: {domain: area}."""
        dom, area = self.areas_array()
        return dict(zip(dom.tolist(), area.tolist()))

    def areas_array(self) -> Tuple[np.ndarray, np.ndarray]:
        """The same as two arrays (domain ids, areas) in the handle's cell
        order, views of buffers kept between calls (sized for the cell count
        plus room for divisions): valid until the next call.  Right after
        step() with an area regulator registered the areas are already on
        the host; otherwise the call is one round trip to the device."""
        for _ in range(2):
            cap = len(getattr(self, "_area_d", ()))
            if cap == 0:
                cap = max(1, self.sizes()["cells"]) + 64
                self._area_d = np.zeros(cap, np.uint32)
                self._area_a = np.zeros(cap)
            n = self.areas_into(self._area_d, self._area_a)
            if n <= cap:
                return self._area_d[:n], self._area_a[:n]
            self._area_d = np.zeros(n + 64, np.uint32)
            self._area_a = np.zeros(n + 64)
        raise RuntimeError("lbib_areas: the cell count keeps changing")

    def areas_into(self, dom: np.ndarray, area: np.ndarray) -> int:
        """lbib_areas into caller-owned contiguous uint32 / float64 arrays
        (pinned or not): fills min(count, len) entries, returns the count."""
        rd, ra, pd, pa, cap = self._areas
        if dom is not rd or area is not ra or cap != min(len(dom), len(area)):
            if dom.dtype != np.uint32 or area.dtype != np.float64 or not (dom.flags.c_contiguous and
                                                                         area.flags.c_contiguous):
                raise ValueError("areas_into needs contiguous uint32 and float64 arrays")
            pd, pa, cap = dom.ctypes.data, area.ctypes.data, min(len(dom), len(area))
            self._areas = (dom, area, pd, pa, cap)
        n = self._L.lbib_areas(self._h, pd, pa, cap)
        if n < 0:
            raise self._error()
        return n

    def accumulated_concentrations(self, species: str) -> Dict[int, float]:
        """GeometryHandler::computeAccumulatedDomainConcentrations(species)."""
        cap = max(1, self.domain_count())
        d = np.zeros(cap, np.uint32); a = np.zeros(cap)
        n = self._L.lbib_accumulated_concentrations(self._h, species.encode(), _p(d), _p(a), cap)
        if n < 0:
            raise self._error()
        return {int(d[i]): float(a[i]) for i in range(n)}

    def set_cell_types(self, types: Dict[int, int]) -> None:
        """getCellTypeTrackerMap()[d] = t for each entry, then copyCellTypeToPhysicalNodes."""
        d = np.array(sorted(types), np.uint32)
        t = np.array([types[int(k)] for k in d], np.uint32)
        self._check(self._L.lbib_set_cell_types(self._h, _p(d), _p(t), len(d)))

    def cell_types(self) -> Dict[int, int]:
        """GeometryHandler::getCellTypeTrackerMap."""
        cap = max(1, self.domain_count())
        d = np.zeros(cap, np.uint32); t = np.zeros(cap, np.uint32)
        n = self._L.lbib_get_cell_types(self._h, _p(d), _p(t), cap)
        if n < 0:
            raise self._error()
        return {int(d[i]): int(t[i]) for i in range(n)}

    # -- topology edits by host bio solvers -----------------------------------------
    def upload_membrane(self, ids, xy, conns) -> None:
        """The membrane after a host plugin's edits (see lbib_upload_membrane):
        ids (M,) ascending, xy (M, 2), conns (C, 3) = id1, id2, domain."""
        i = np.ascontiguousarray(ids, np.uint32)
        p = np.ascontiguousarray(xy, np.float64).reshape(-1, 2)
        c = np.ascontiguousarray(conns, np.uint32).reshape(-1, 3)
        if len(i) != len(p):
            raise ValueError("upload_membrane: ids and xy of different lengths")
        self._check(self._L.lbib_upload_membrane(self._h, _p(i), _p(p), len(i), _p(c), len(c)))

    def cure_lattice(self) -> None:
        """GeometryHandler::cureLattice after topology edits (see lbib_cure_lattice)."""
        self._check(self._L.lbib_cure_lattice(self._h))

    # -- force list and range queries (host bio solvers) -----------------------
    def add_forces(self, types, id1, id2, par) -> None:
        """ForceSolver::addForce for a batch of records (see lbib_add_forces):
        types (n,), id1 (n,), id2 (n,) (ignored where the type has no partner),
        par (n, 4)."""
        t = np.ascontiguousarray(types, np.int32)
        a = np.ascontiguousarray(id1, np.uint32)
        b = np.ascontiguousarray(id2, np.uint32)
        p = np.ascontiguousarray(par, np.float64).reshape(-1, 4)
        if not (len(t) == len(a) == len(b) == len(p)):
            raise ValueError("add_forces: arrays of different lengths")
        self._check(self._L.lbib_add_forces(self._h, _p(t), _p(a), _p(b), _p(p), len(t)))

    def delete_force_type(self, t: int) -> None:
        self._check(self._L.lbib_delete_force_type(self._h, int(t)))

    def delete_all_forces(self) -> None:
        self._check(self._L.lbib_delete_all_forces(self._h))

    def nodes_within_radius(self, x: float, y: float, radius: float, avoid_domain: int = -1) -> np.ndarray:
        """Geometry::getGeometryNodesWithinRadius[WithAvoidance]: node ids, in the
        reference's cell-list order."""
        cap = 64
        while True:
            ids = np.zeros(cap, np.uint32)
            n = self._L.lbib_nodes_within_radius(self._h, float(x), float(y), float(radius), int(avoid_domain),
                                                 _p(ids), cap)
            if n < 0:
                raise self._error()
            if n <= cap:
                return ids[:n].copy()
            cap = n

    def closest_nodes(self, x, y, radius: float, avoid_domain=None) -> np.ndarray:
        """Geometry::getGeometryNodesWithinRadiusWithAvoidanceClosest for each
        query point: node id or -1."""
        qx = np.ascontiguousarray(x, np.float64)
        qy = np.ascontiguousarray(y, np.float64)
        av = None if avoid_domain is None else np.ascontiguousarray(avoid_domain, np.int64)
        out = np.zeros(len(qx), np.int64)
        self._check(self._L.lbib_closest_nodes(self._h, _p(qx), _p(qy), _p(av), len(qx), float(radius), _p(out)))
        return out

    # -- VTK reporters ---------------------------------------------------------------
    VTK_CELLS, VTK_FORCES, VTK_CDE, VTK_FLUID, VTK_CELL_PNG = 1, 2, 3, 4, 5

    def write_vtk(self, prefix: str, time: int, kind: int, coarsening: int = 1) -> str:
        """Appends the block of one vtk*Reporter to prefix_time.vtm; returns the
        .vtm path."""
        self._check(self._L.lbib_write_vtk(self._h, prefix.encode(), int(time), int(kind), int(coarsening)))
        return f"{prefix}_{int(time)}.vtm"

    # -- checkpoint files (the reference's formats) ------------------------------
    def write_simulation(self, prefix: str) -> Dict[str, str]:
        """SimulationRunner::writeSimulation into prefix_{force,geometry,parameters,solver}.txt;
        returns the paths (keys as the configuration files)."""
        paths = {k: f"{prefix}_{k}.txt" for k in ("force", "geometry", "parameters", "solver")}
        self._check(self._L.lbib_write_simulation(self._h, *[paths[k].encode() for k in
                                                                ("force", "geometry", "parameters", "solver")]))
        return paths

    def load_solvers(self, solver_file: str) -> None:
        """SimulationRunner::initSolvers(file): the distributions of a solver dump."""
        self._check(self._L.lbib_load_solvers(self._h, solver_file.encode()))

    # -- differentiated runs (frozen geometry, FP64) -----------------------------
    def domain_count(self) -> int:
        n = ctypes.c_int(0)
        self._check(self._L.lbib_get_domain_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def diff_begin(self, T: int, K: int = 0) -> None:
        """Snapshot the lattice as the initial state of a T-step differentiated
        run with a checkpoint every K steps (K <= 0: ceil(sqrt(T)))."""
        self._check(self._L.lbib_diff_begin(self._h, int(T), int(K)))

    def diff_forward(self, forces=None, tau=None, rates=None, outlet: bool = True) -> None:
        """T forward steps from the snapshot.  forces (M, 2) membrane node
        forces, tau (1 + S,) relaxation times, rates (S, n_domains) source rates;
        None keeps the current values."""
        args = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (forces, tau, rates)]
        self._check(self._L.lbib_diff_forward(self._h, *[_p(a) for a in args], 1 if outlet else 0))

    def diff_backward(self, dLdC) -> Dict[str, np.ndarray]:
        """Gradients of L from dL/dC (S, Nx*Ny) at the final step:
        {"force": (M, 2), "tau": (1 + S,), "rates": (S, n_domains)}."""
        z = self.sizes()
        S, M = z["S"], z["M"]
        seed = np.ascontiguousarray(np.asarray(dLdC, np.float64).reshape(S, z["nx"] * z["ny"]))
        gF = np.zeros((M, 2)); gT = np.zeros(1 + S); gR = np.zeros((S, self.domain_count()))
        self._check(self._L.lbib_diff_backward(self._h, _p(seed), _p(gF), _p(gT), _p(gR)))
        return {"force": gF, "tau": gT, "rates": gR}

    def diff_mass(self, mass=None) -> np.ndarray:
        """Sets the run's per-domain mass source (when given) and returns dL/d
        mass of the last backward pass."""
        n = self.domain_count()
        m = None if mass is None else np.ascontiguousarray(mass, np.float64)
        g = np.zeros(n)
        self._check(self._L.lbib_diff_mass(self._h, _p(m), _p(g), n))
        return g

    def diff_fluid_seed(self, dLdf=None) -> None:
        """dL/d of the final fluid distributions ((L, 9), lattice() layout) for
        the next backward passes; None removes it."""
        a = None if dLdf is None else np.ascontiguousarray(dLdf, np.float64)
        self._check(self._L.lbib_diff_fluid_seed(self._h, _p(a)))

    def diff_force_params(self) -> np.ndarray:
        """dL/d of every force record's four parameters ((n, 4), the order of
        forces()) from the last backward pass's membrane-force gradient."""
        n = self._L.lbib_diff_force_params(self._h, None, 0)
        if n < 0:
            raise self._error()
        g = np.zeros((n, 4))
        got = self._L.lbib_diff_force_params(self._h, _p(g), n)
        if got < 0:
            raise self._error()
        return g

    def diff_motion(self, on: bool = True, dLdX=None) -> None:
        """Moving membrane nodes in the next forward passes (the motion and its
        adjoint); dLdX (M, 2) is dL/d of the final positions, or None."""
        a = None if dLdX is None else np.ascontiguousarray(dLdX, np.float64)
        self._check(self._L.lbib_diff_motion(self._h, 1 if on else 0, _p(a)))

    def diff_positions(self, grad: bool = False):
        """Final positions (M, 2) of the last forward pass; with grad, also
        dL/dX (M, 2) of the starting positions from the last backward pass."""
        M = self.sizes()["M"]
        xT = np.zeros((M, 2))
        g0 = np.zeros((M, 2)) if grad else None
        self._check(self._L.lbib_diff_positions(self._h, _p(xT), _p(g0), M))
        return (xT, g0) if grad else xT

    def forces(self) -> Dict[str, np.ndarray]:
        """The ForceSolver's records in device order (by node, then insertion):
        type, id1, id2 (partner id or 0) and par (n, 4)."""
        n = self._L.lbib_download_forces(self._h, None, None, None, None, 0)
        if n < 0:
            raise self._error()
        t = np.zeros(n, np.int32); a = np.zeros(n, np.uint32); b = np.zeros(n, np.uint32); par = np.zeros((n, 4))
        got = self._L.lbib_download_forces(self._h, _p(t), _p(a), _p(b), _p(par), n)
        if got < 0:
            raise self._error()
        return {"type": t, "id1": a, "id2": b, "par": par}

    def diff_end(self) -> None:
        """Restore the snapshot and free the run's checkpoints."""
        self._check(self._L.lbib_diff_end(self._h))

    def concentrations(self) -> np.ndarray:
        """C_k(x) = sum of species k's distributions, shape (S, Nx*Ny)."""
        return self.lattice().g.sum(axis=2)


def read_vtm_geometry(path: str):
    """Geometry::loadGeometryVTK on the host (no GPU): (ids[n], xy[n, 2] before
    the perturbation of new nodes, connections[c, 3] = id1, id2, domain)."""
    L = load()
    counts = np.zeros(2, np.int32)
    rc = L.lbib_read_vtm_geometry(path.encode(), None, None, 0, None, 0, _p(counts))
    if rc:
        raise LbibError(rc, f"cannot read {path}", -1)
    n, c = int(counts[0]), int(counts[1])
    ids = np.zeros(n, np.uint32); xy = np.zeros((n, 2)); conns = np.zeros((c, 3), np.uint32)
    rc = L.lbib_read_vtm_geometry(path.encode(), _p(ids), _p(xy), n, _p(conns), c, _p(counts))
    if rc:
        raise LbibError(rc, f"cannot read {path}", -1)
    return ids, xy, conns
