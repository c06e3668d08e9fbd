#!/usr/bin/env python
"""Benchmark of the LBIBCell hot path on B200.

Workload: the 1024x1024 tissue (400 cells on a hexagonal grid, ~100k membrane
nodes growing to ~150k after the first remesh, 2 D2Q5 species, tension, area
regulator, cell junctions, box outlet) in lbibcell_b200/configs.py:config2.  A step is one full
iteration of SimulationRunner::runSimulation's loop body on the GPU.  The metric
is MLUPS (lattice node updates per second / 1e6, all species included) of the
FP32-shifted path; the FP64 path's MLUPS and the FP32-vs-FP64 field errors are
reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs N independent replicas (one simulation per GPU, no data exchange;
value = all ranks' lattice updates / max time).  ``--impl reference`` times the
reference's own CPU code (oracle/_ref/ref_driver_fast, built from the
reference sources) on the host cores for the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS FP32-shifted vs FP64 on 1 B200 @ rel.err≤1e-5; adjoint/forward time"
WORKLOAD = ("tissue_1024: 1024x1024 D2Q9 + 2 D2Q5 species, 400 cells (hex grid, spacing 44, r=20+U(-2,2), "
            "250 nodes/cell), tension, area regulator (hold area), cell junctions (radius 1 lu, k 0.02, "
            "rest length 2 lu), box outlet")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiated-run timing")
    ap.add_argument("--adjoint-steps", type=int, default=2000, help="T of the differentiated run")
    ap.add_argument("--no-large", action="store_true", help="skip the tissue_4096 block")
    ap.add_argument("--large-steps", type=int, default=30, help="timed steps of the tissue_4096 block")
    ap.add_argument("--no-adjoint-large", action="store_true", help="skip the adjoint_2048 block")
    ap.add_argument("--large-cpu", action="store_true",
                    help="time the reference CPU build on tissue_4096 too (its set-up alone takes minutes)")
    ap.add_argument("--adjoint-large-steps", type=int, default=10000, help="T of the adjoint_2048 block")
    return ap.parse_args()


def workload_config(cfg):
    """The workload both arms run (the same dict in both JSON lines)."""
    return {"workload": WORKLOAD, "lattice": [cfg.nx, cfg.ny], "species": len(cfg.species), "cells": len(cfg.cells),
            "membrane_nodes_initial": cfg.membrane_nodes,
            "l2": "inputs larger than L2 (lattice state ~170 MB per copy set)"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n):
    """One process per GPU (replicas: the ranks share only the barrier around
    the timed region and the max of the timings).  NCCL on GPUs, gloo without."""
    rank, world, local = 0, 1, 0
    if n > 1 or int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import datetime
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def ref_cpu_time(paths, warm, steps, threads):
    """Wall time of the reference's runSimulation() for `steps` iterations after
    `warm`, on `threads` OpenMP threads (oracle/_ref/ref_driver_fast)."""
    from oracle import oracle as O
    drv = O.REF_DRIVER_FAST
    if not os.path.exists(drv):
        return None
    out = tempfile.mkdtemp(prefix="lbib_ref_")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([drv, paths["parameters"], paths["geometry"], paths["force"], paths["plugins"], out,
                        "timing", str(warm), str(steps)], env=env, capture_output=True, text=True, timeout=1800,
                       cwd=out)
    if r.returncode != 0:
        raise RuntimeError("reference run failed: " + r.stderr[-2000:])
    line = [l for l in r.stderr.splitlines() if l.startswith("{")][-1]
    return json.loads(line)


def port_cpu_time(paths, steps):
    """Fallback CPU baseline: the oracle's C++ restatement, single thread."""
    from oracle import oracle as O
    o = O.Oracle(paths)
    o.step(1)
    t0 = time.perf_counter()
    o.step(steps)
    return {"seconds": time.perf_counter() - t0, "iterations": steps, "threads": 1}


def reference_arm(args, cfg, paths):
    threads = os.cpu_count() or 1
    warm, steps = min(args.warmup, 3), max(1, min(args.steps, 20))
    L = cfg.nx * cfg.ny
    res = ref_cpu_time(paths, warm, steps, threads)
    kind = "reference"
    if res is None:
        res = port_cpu_time(paths, min(steps, 3))
        kind, threads = "port", 1
    mlups = L * res["iterations"] / res["seconds"] / 1e6
    sample = f"{res['iterations']} steps after {warm if kind == 'reference' else 1} warm-up steps of {cfg.name}"
    line = {
        "impl": "reference", "metric": METRIC, "value": mlups, "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * res["seconds"] / res["iterations"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(cfg),
        "precision": "FP64 (reference CPU build, -O3 -march=x86-64-v3 -fopenmp)",
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": kind, "sample": sample,
                         "cpu_model": cpu_model()},
        "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _rel(x, y):
    ok = np.isfinite(x) & np.isfinite(y)
    if not ok.any():
        return None
    d = np.abs(x[ok] - y[ok]).max()
    s = np.abs(x[ok]).max()
    return float(d / s) if s > 0 else float(d)


def rel_errors(a, b):
    """Max-norm errors of b against a: rho-1 by max|rho-1|, u by max|u|, c_k by
    max c_k (finite entries), plus counts of non-finite values and of domain ids
    that differ."""
    ra, rb = a.f.sum(1) - 1.0, b.f.sum(1) - 1.0
    out = {"rho_minus_1": _rel(ra, rb), "rho_abs": float(np.nanmax(np.abs(ra - rb))), "u": _rel(a.vel, b.vel)}
    for k in range(a.g.shape[0]):
        out[f"c{k}"] = _rel(a.g[k].sum(1), b.g[k].sum(1))
    out["nonfinite"] = int((~np.isfinite(a.g)).sum() + (~np.isfinite(b.g)).sum())
    out["domain_mismatch"] = int(np.count_nonzero(a.dom != b.dom))
    return out


def fp32_error_at(paths, horizons, local):
    """FP32-shifted vs FP64 errors (rel_errors) after each horizon of full steps,
    with the non-finite counts: the reference's re-initialisation writes NaN
    for nodes trapped between touching membranes (CDESolverD2Q5.cpp:223)."""
    from lbibcell_b200 import runner
    a = runner.Simulation(paths, runner.FP64, device=local)
    b = runner.Simulation(paths, runner.FP32_SHIFTED, device=local)
    out, done = {}, 0
    for h in horizons:
        a.step(h - done)
        b.step(h - done)
        done = h
        la, lb = a.lattice(), b.lattice()
        e = rel_errors(la, lb)
        e["nonfinite_fp64_g"] = int((~np.isfinite(la.g)).sum())
        e["finite_fraction_g"] = float(np.isfinite(la.g).mean())
        out[str(h)] = e
    a.close()
    b.close()
    return out


def large_block(args, tmp, rank, world, local):
    """tissue_4096 (configs.config3: 4096x4096, 6000 cells, ~1M membrane nodes,
    3 species, tension, junctions, growth and division): FP32-shifted and FP64
    step rates, the whole-step and stream-collide roofline fractions, the
    FP32-vs-FP64 error after the same steps, and a truncated CPU baseline."""
    from lbibcell_b200 import configs, runner
    cfg = configs.config3(iterations=10 ** 6)
    paths = cfg.write(os.path.join(tmp, f"large_rank{rank}"))
    L, S = cfg.nx * cfg.ny, len(cfg.species)
    warm, K, prof = 5, args.large_steps, 10
    peak, _ = measured_peaks()
    out = {"workload": f"{cfg.name}: {cfg.nx}x{cfg.ny}, {len(cfg.cells)} cells (Poisson-disk, r U(10,16)), "
                       f"{cfg.membrane_nodes} membrane nodes at t=0, 3 species, tension, junctions, "
                       "growth to 2.5x area, division at 2x", "steps_timed": K}
    runs = {}
    for name, prec in (("fp32", runner.FP32_SHIFTED), ("fp64", runner.FP64)):
        sim = runner.Simulation(paths, prec, device=local)
        sim.step(warm)
        barrier(world)
        sim.step(K)
        ms = dist_max(sim.last_timing()["total_ms"], world)
        sim.set_profiling(True)
        sim.step(prof)
        sim.set_profiling(False)
        tp = sim.last_timing()
        avg = tp["collide_ms"] / max(1, tp["collide_launches"])
        bpn = (80 + 48 * S) * (2 if prec == runner.FP64 else 1)
        mlups = world * L * K / (ms / 1e3) / 1e6
        runs[name] = sim
        out[name] = {"mlups": mlups, "ms_per_step": ms / K,
                     "whole_step_roofline_frac": mlups * 1e6 * bpn / (peak * 1e9),
                     "stream_collide_avg_ms": avg,
                     "stream_collide_roofline_frac": bpn * L / (avg / 1e3) / 1e9 / peak,
                     "algorithmic_bytes_per_node": bpn, "membrane_nodes": sim.sizes()["M"],
                     "host_events": sim.sizes()["host_events"]}
    out["fp32_over_fp64"] = out["fp32"]["mlups"] / out["fp64"]["mlups"]
    a, b = runs["fp64"].lattice(), runs["fp32"].lattice()
    # full steps: the trajectories separate where a membrane node's FP32
    # position moves a crossing (a domain flip re-initialises a node), so the
    # pointwise error is the flips'; the frozen-geometry comparison below is
    # the lattice arithmetic's
    out["fp32_vs_fp64_rel_err"] = rel_errors(a, b)
    out["steps_compared"] = warm + K + prof
    force = a.force
    del a, b
    for sim in runs.values():
        sim.close()
    # fresh simulations (same initial state and domain ids), the FP64 run's
    # force field, lattice steps only
    fr = {p: runner.Simulation(paths, p, device=local) for p in (runner.FP64, runner.FP32_SHIFTED)}
    for sim in fr.values():
        sim.set_lattice(force=force)
        sim.lattice_step(K, outlet=True)
    out["fp32_vs_fp64_rel_err_frozen_geometry"] = rel_errors(fr[runner.FP64].lattice(), fr[runner.FP32_SHIFTED].lattice())
    out["frozen_steps"] = K
    for sim in fr.values():
        sim.close()
    runs = {}
    for sim in runs.values():
        sim.close()
    if rank == 0 and args.large_cpu and world == 1:
        try:
            res = ref_cpu_time(paths, 1, 20, os.cpu_count() or 1)
            if res is not None:
                out["cpu_baseline_truncated"] = {
                    "value": L * res["iterations"] / res["seconds"] / 1e6, "unit": "MLUPS",
                    "cores": res.get("threads", 1), "cpu_model": cpu_model(),
                    "sample": f"truncated: {res['iterations']} steps after 1 warm-up step of {cfg.name} "
                              "(set-up excluded), reference CPU build"}
        except Exception as e:
            out["cpu_baseline_truncated"] = {"value": None, "sample": f"failed: {e}"[:300]}
    return out


def adjoint_large_block(args, tmp, rank, world, local):
    """adjoint_2048 (configs.config5): 2048x2048, 1000 cells, fluid + 2 species,
    frozen geometry after 3 full steps.  Parameters: the 1000 per-cell
    area-regulator strengths s_d, entering as the mass source
    m_d = s_d (target_d - A_d) / target_d (LbibAreaRegulator below its clamp,
    areas frozen).  Loss: the kinetic energy of the final distributions in the
    central 256x256 window plus sum (C_k - c_target_k)^2, c_target from a
    forward run with the strengths perturbed by N(0, 0.1) relative.  sqrt(T)
    checkpoints with segment recompute.  FP32-shifted forward and FP32
    checkpoints; the reverse step computes in FP64 and the parameter gradients
    accumulate in FP64.  Reports adjoint/forward time, the device memory in
    use during the run and one central-difference check (step 1e-4 on a
    strength of 0.01: the FP32 forward's rounding rules out smaller steps)."""
    import torch
    from lbibcell_b200 import configs, runner
    cfg = configs.config5()
    paths = cfg.write(os.path.join(tmp, f"adj2048_rank{rank}"))
    T = args.adjoint_large_steps
    sim = runner.Simulation(paths, runner.FP32_SHIFTED, device=local)
    first = sim.areas()          # the regulator's targets: 1.2 x these
    sim.step(3)
    areas = sim.areas()
    nD = sim.domain_count()
    factor, strength0, maxsource = cfg.area
    coef = np.zeros(nD)
    for d, a in areas.items():
        tgt = factor * first[d]
        coef[d] = (tgt - a) / tgt
    strengths = np.full(nD, strength0)
    strengths[0] = 0.0

    def mass_of(s):
        return np.clip(s * coef, -maxsource, maxsource)

    free0, total = torch.cuda.mem_get_info(local)
    sim.diff_begin(T, 0)
    free1, _ = torch.cuda.mem_get_info(local)
    n = cfg.nx
    yy, xx = np.divmod(np.arange(n * n), n)
    window = (abs(xx - n // 2) < 128) & (abs(yy - n // 2) < 128)
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])[[0, 3, 4, 1, 2, 7, 8, 5, 6]]
    ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])[[0, 3, 4, 1, 2, 7, 8, 5, 6]]
    target = strengths * (1.0 + np.random.default_rng(6).normal(0.0, 0.1, nD))
    sim.diff_mass(mass_of(target))
    sim.diff_forward()
    c_target = sim.concentrations().copy()

    def loss(s):
        sim.diff_mass(mass_of(s))
        sim.diff_forward()
        f = sim.lattice().f
        rho = f.sum(1)
        jx, jy = f @ ex, f @ ey
        e = 0.5 * (jx * jx + jy * jy) / rho
        C = sim.concentrations()
        dke = ((np.outer(jx, ex) + np.outer(jy, ey)) / rho[:, None] - (e / rho)[:, None]) * window[:, None]
        return float(e[window].sum() + ((C - c_target) ** 2).sum()), dke, 2.0 * (C - c_target)

    torch.cuda.synchronize()
    L0, dke, dC = loss(strengths)
    fwd_ms = sim.last_timing()["total_ms"]
    sim.diff_fluid_seed(dke)
    g = sim.diff_backward(dC)
    bwd_ms = sim.last_timing()["total_ms"]
    free2, _ = torch.cuda.mem_get_info(local)
    gS = sim.diff_mass() * coef
    d = int(np.argmax(np.abs(gS[1:]))) + 1
    h = 1e-4
    sp, sm = strengths.copy(), strengths.copy()
    sp[d] += h
    sm[d] -= h
    fd = (loss(sp)[0] - loss(sm)[0]) / (2 * h)
    sim.diff_end()
    sim.close()
    return {"workload": f"{cfg.name}: {cfg.nx}x{cfg.ny}, {len(cfg.cells)} cells, fluid + {len(cfg.species)} species, "
                        "frozen geometry, FP32-shifted forward and checkpoints, FP64 reverse arithmetic",
            "T": T, "K": int(math.ceil(math.sqrt(T))), "forward_ms": fwd_ms, "backward_ms": bwd_ms,
            "adjoint_over_forward": bwd_ms / fwd_ms,
            "device_memory_gb": {"before_run": (total - free0) / 1e9, "run_allocated": (total - free1) / 1e9,
                                 "after_backward": (total - free2) / 1e9, "total": total / 1e9},
            "parameters": f"{nD - 1} per-cell area-regulator strengths", "loss": L0,
            "grad_strength_max": float(np.abs(gS).max()),
            "fd_check": {"domain": d, "adjoint": float(gS[d]), "central_difference": fd, "h": h,
                         "rel_err": abs(gS[d] - fd) / max(abs(fd), 1e-300)},
            "grad_finite": bool(np.isfinite(gS).all() and np.isfinite(g["tau"]).all())}


def main():
    args = parse()
    from lbibcell_b200 import configs
    cfg = configs.config2(iterations=args.steps + args.warmup)
    tmp = tempfile.mkdtemp(prefix="lbib_bench_")
    rank, world, local = dist_setup(args.gpus)
    paths = cfg.write(os.path.join(tmp, f"rank{rank}"))

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, cfg, paths)
        return

    import torch
    from lbibcell_b200 import build, runner
    build.build()
    torch.cuda.set_device(local)
    L = cfg.nx * cfg.ny
    S = len(cfg.species)

    # ---- FP32-shifted: the headline ---------------------------------------
    sim = runner.Simulation(paths, runner.FP32_SHIFTED, device=local)
    sim.step(args.warmup)
    M = sim.sizes()["M"]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        sim.step(args.steps)
    torch.cuda.synchronize()
    barrier(world)
    tm = sim.last_timing()
    t_ms = dist_max(tm["total_ms"], world)
    value = world * L * args.steps / (t_ms / 1e3) / 1e6
    host_events = sim.sizes()["host_events"]

    # roofline of the fused stream-collide kernel (algorithmic bytes per lattice
    # update); its launches are timed with CUDA events on the handle's stream
    # over a further stretch of the same run (the timed region above replays
    # CUDA graphs, which carry no per-kernel events)
    prof_steps = min(args.steps, 100)
    sim.set_profiling(True)
    sim.step(prof_steps)
    sim.set_profiling(False)
    tp_ = sim.last_timing()
    bytes_per_node = 80 + 48 * S
    peak, peak_kind = measured_peaks()
    avg_ms = tp_["collide_ms"] / max(1, tp_["collide_launches"])
    achieved = bytes_per_node * L / (avg_ms / 1e3) / 1e9
    # dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of the
    # same kernel on this workload, from its committed summary
    traffic = None
    tp = os.path.join(ROOT, "profiles", "stream_collide32_tissue_1024.md")
    if os.path.exists(tp):
        m = re.search(r"\|\s*traffic_bytes_per_launch\s*\|\s*(\d+)", open(tp).read())
        traffic = int(m.group(1)) if m else None

    # ---- end to end through the public API, host buffers each step ---------
    # every step: H2D of both species' per-domain secretion tables (what a host
    # plugin pushes) from pinned memory in one copy, lbib_step(1), D2H of the
    # per-cell areas into pinned host arrays.  A fresh handle runs the same
    # iterations as the timed region above (the same warm-up, then `steps`
    # steps): the membrane grows over a run, so a later window would be a
    # heavier workload.
    sim.close()
    sim = runner.Simulation(paths, runner.FP32_SHIFTED, device=local)
    sim.step(args.warmup)
    nd = sim.domain_count()
    pinned = torch.zeros((S, nd), dtype=torch.float64).pin_memory()
    for k, sp in enumerate(cfg.species):
        for d, r in sp.source.items():
            pinned[k, d] = r
    src = pinned.numpy()
    # the areas come back into pinned host arrays (the caller's buffers)
    cap = sim.sizes()["cells"] + 64
    area_dom = torch.zeros(cap, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    area_val = torch.zeros(cap, dtype=torch.float64).pin_memory().numpy()
    e2e_steps = args.steps
    host_events_before = sim.sizes()["host_events"]
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nareas = 0
    for _ in range(e2e_steps):
        sim.set_species_sources(src)
        sim.step(1)
        nareas = sim.areas_into(area_dom, area_val)
    torch.cuda.synchronize()
    e2e_s = dist_max(time.perf_counter() - t0, world)
    e2e = {"value": world * L * e2e_steps / e2e_s / 1e6, "unit": "MLUPS",
           "h2d_bytes_per_step": int(S * nd * 8), "d2h_bytes_per_step": int(nareas * 8 + nareas * 4),
           "steps": e2e_steps, "host_events": sim.sizes()["host_events"] - host_events_before}
    sim.close()

    # ---- FP64 path and the FP32-vs-FP64 error --------------------------------
    fp64 = None
    if not args.no_fp64:
        a = runner.Simulation(paths, runner.FP64, device=local)
        b = runner.Simulation(paths, runner.FP32_SHIFTED, device=local)
        a.step(args.warmup)
        b.step(args.warmup)
        torch.cuda.synchronize()
        a.step(args.steps)
        t64 = dist_max(a.last_timing()["total_ms"], world)
        b.step(args.steps)
        err = rel_errors(a.lattice(), b.lattice())
        # the same comparison with the geometry frozen (lattice kernels only):
        # the arithmetic error of the FP32-shifted path, free of the membrane's
        # discrete events (remesh/coarsen/domain flips) that amplify rounding
        force = a.lattice().force
        a.close()
        b.close()
        a = runner.Simulation(paths, runner.FP64, device=local)
        b = runner.Simulation(paths, runner.FP32_SHIFTED, device=local)
        a.set_lattice(force=force)
        b.set_lattice(force=force)
        a.lattice_step(args.steps, outlet=True)
        b.lattice_step(args.steps, outlet=True)
        err_frozen = rel_errors(a.lattice(), b.lattice())
        fp64 = {"mlups": world * L * args.steps / (t64 / 1e3) / 1e6, "ms_per_step": t64 / args.steps,
                "fp32_vs_fp64_rel_err": err, "steps_compared": args.warmup + args.steps,
                "fp32_vs_fp64_rel_err_frozen_geometry": err_frozen, "frozen_steps": args.steps}
        a.close()
        b.close()

    # ---- differentiated run: adjoint/forward time on the adjoint workload ----
    adjoint = None
    if not args.no_adjoint:
        acfg = configs.config4()
        apaths = acfg.write(os.path.join(tmp, f"adj_rank{rank}"))
        T, K = args.adjoint_steps, max(1, args.adjoint_steps // 20)
        d = runner.Simulation(apaths, runner.FP64, device=local)
        d.step(3)  # membrane forces of a force evaluation become the default parameters
        d.diff_begin(T, K)
        seed = np.random.default_rng(0).normal(size=(len(acfg.species), acfg.nx * acfg.ny))
        d.diff_forward()  # untimed: first touch of the checkpoint memory
        d.diff_backward(seed)
        torch.cuda.synchronize()
        d.diff_forward()
        fwd_ms = dist_max(d.last_timing()["total_ms"], world)
        g = d.diff_backward(seed)
        bwd_ms = dist_max(d.last_timing()["total_ms"], world)
        d.diff_end()
        # The same workload with moving membrane nodes (the motion and its
        # adjoint), a loss of the final positions joined to the concentrations'
        # seed.  The node forces stay those of one force evaluation for the
        # whole run, so over long runs they push nodes to the lattice's edge
        # (a refused stencil at T = 2000); 200 steps move them up to 0.65 lu.
        Tm = min(T, 200)
        Km = max(1, Tm // 20)
        d.diff_begin(Tm, Km)
        _, st0 = d.membrane()
        d.diff_motion(True, np.random.default_rng(1).normal(size=(st0.shape[0], 2)))
        d.diff_forward()  # untimed: first touch of the position store
        d.diff_backward(seed)
        torch.cuda.synchronize()
        d.diff_forward()
        fwdm = dist_max(d.last_timing()["total_ms"], world)
        gm = d.diff_backward(seed)
        bwdm = dist_max(d.last_timing()["total_ms"], world)
        xT, gx0 = d.diff_positions(grad=True)
        moving = {"T": Tm, "K": Km, "forward_ms": fwdm, "backward_ms": bwdm, "adjoint_over_forward": bwdm / fwdm,
                  "membrane_nodes": int(st0.shape[0]),
                  "max_displacement_lu": float(np.abs(xT - st0[:, :2]).max()),
                  "grad_finite": bool(np.isfinite(gm["force"]).all() and np.isfinite(gx0).all())}
        d.diff_end()
        d.close()
        # the same run on an FP32-shifted handle (FP32 forward and states)
        d32 = runner.Simulation(apaths, runner.FP32_SHIFTED, device=local)
        d32.step(3)
        d32.diff_begin(T, K)
        d32.diff_forward()
        d32.diff_backward(seed)
        torch.cuda.synchronize()
        d32.diff_forward()
        fwd32 = dist_max(d32.last_timing()["total_ms"], world)
        g32 = d32.diff_backward(seed)
        bwd32 = dist_max(d32.last_timing()["total_ms"], world)
        d32.diff_end()
        d32.close()
        AL = acfg.nx * acfg.ny
        adjoint_fp32 = {"forward_ms": fwd32, "backward_ms": bwd32, "adjoint_over_forward": bwd32 / fwd32,
                        "grad_rel_diff_vs_fp64": {
                            k: float(np.abs(g32[k] - g[k]).max() / max(np.abs(g[k]).max(), 1e-300))
                            for k in ("force", "tau", "rates")}}
        adjoint = {"workload": f"{acfg.name}: {acfg.nx}x{acfg.ny}, {len(acfg.cells)} cells, "
                               f"{len(acfg.species)} species, frozen geometry, FP64",
                   "T": T, "K": K, "forward_ms": fwd_ms, "backward_ms": bwd_ms,
                   "forward_mlups": world * AL * T / (fwd_ms / 1e3) / 1e6,
                   "backward_note": "segment recompute from checkpoints + adjoint steps",
                   "grad_finite": bool(np.isfinite(g["force"]).all() and np.isfinite(g["tau"]).all()),
                   "fp32": adjoint_fp32, "moving_nodes": moving}

    # ---- FP32-shifted error at fixed horizons (independent of --steps) -------
    horizons = None
    if not args.no_fp64:
        horizons = fp32_error_at(configs.config2(iterations=1000).write(os.path.join(tmp, f"hz_rank{rank}")),
                                 (500, 1000), local)

    # ---- adjoint_2048: the large differentiated run -------------------------
    adjoint_large = None
    if not args.no_adjoint_large:
        adjoint_large = adjoint_large_block(args, tmp, rank, world, local)

    # ---- tissue_4096: the large configuration ------------------------------
    large = None
    if not args.no_large:
        large = large_block(args, tmp, rank, world, local)

    if rank != 0:
        return
    cpu = None
    if not args.no_cpu and world == 1:
        try:
            res = ref_cpu_time(paths, 2, 10, os.cpu_count() or 1)
            kind = "reference"
            if res is None:
                res = port_cpu_time(paths, 2)
                kind = "port"
            cpu = {"value": L * res["iterations"] / res["seconds"] / 1e6, "unit": "MLUPS",
                   "cores": res.get("threads", 1), "kind": kind, "cpu_model": cpu_model(),
                   "sample": f"{res['iterations']} steps of {cfg.name} after {res.get('warmup', 1)} warm-up steps"}
            if kind == "reference":
                one = ref_cpu_time(paths, 1, 3, 1)
                cpu["single_thread"] = {"value": L * one["iterations"] / one["seconds"] / 1e6, "unit": "MLUPS",
                                        "cores": 1, "sample": f"{one['iterations']} steps after 1 warm-up step, "
                                                              "OMP_NUM_THREADS=1"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"[:300]}

    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(cfg),
        "precision": "FP32-shifted distributions, FP64 membrane",
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "membrane_nodes": M, "host_events": host_events,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "stream_collide32",
                     "algorithmic_bytes_per_node": bytes_per_node, "avg_launch_ms": avg_ms,
                     "launches_timed": tp_["collide_launches"], "peak_source": peak_kind},
        "fp64": fp64,
        "fp32_over_fp64": (value / fp64["mlups"]) if fp64 else None,
        "fp32_error_at_horizons": horizons,
        "tissue_4096": large,
        "adjoint_over_forward": (adjoint["backward_ms"] / adjoint["forward_ms"]) if adjoint else None,
        "adjoint": adjoint,
        "adjoint_2048": adjoint_large,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(tm["launches"]),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    try:
        main()
    finally:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()
