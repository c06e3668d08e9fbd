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
    return ap.parse_args()


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
        "config": {"workload": WORKLOAD, "lattice": [cfg.nx, cfg.ny], "species": len(cfg.species),
                   "cells": len(cfg.cells), "precision": "FP64 (reference CPU build, -O3 -march=x86-64-v3 -fopenmp)"},
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": kind, "sample": sample},
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
    # plugin pushes) from pinned memory, lbib_step(1), D2H of the per-cell areas.
    nd = max(d for d, _ in cfg.cells) + 1
    pinned = torch.zeros((S, nd), dtype=torch.float64).pin_memory()
    for k, sp in enumerate(cfg.species):
        for d, r in sp.source.items():
            pinned[k, d] = r
    src = pinned.numpy()
    e2e_steps = min(args.steps, 200)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nareas = 0
    for _ in range(e2e_steps):
        for k in range(S):
            sim.set_species_source(k, src[k])
        sim.step(1)
        nareas = len(sim.areas())
    torch.cuda.synchronize()
    e2e_s = dist_max(time.perf_counter() - t0, world)
    e2e = {"value": world * L * e2e_steps / e2e_s / 1e6, "unit": "MLUPS",
           "h2d_bytes_per_step": int(S * nd * 8), "d2h_bytes_per_step": int(nareas * 8 + nareas * 4),
           "steps": e2e_steps}
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
        d.close()
        AL = acfg.nx * acfg.ny
        adjoint = {"workload": f"{acfg.name}: {acfg.nx}x{acfg.ny}, {len(acfg.cells)} cells, "
                               f"{len(acfg.species)} species, frozen geometry, FP64",
                   "T": T, "K": K, "forward_ms": fwd_ms, "backward_ms": bwd_ms,
                   "forward_mlups": world * AL * T / (fwd_ms / 1e3) / 1e6,
                   "backward_note": "segment recompute from checkpoints + adjoint steps",
                   "grad_finite": bool(np.isfinite(g["force"]).all() and np.isfinite(g["tau"]).all())}

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
                   "cores": res.get("threads", 1), "kind": kind,
                   "sample": f"{res['iterations']} steps of {cfg.name} after {res.get('warmup', 1)} warm-up steps"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"[:300]}

    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lattice": [cfg.nx, cfg.ny], "species": S, "cells": len(cfg.cells),
                   "membrane_nodes": M, "precision": "FP32-shifted distributions, FP64 membrane",
                   "l2": "inputs larger than L2 (lattice state ~170 MB per copy set)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "host_events": host_events},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "stream_collide32",
                     "algorithmic_bytes_per_node": bytes_per_node, "avg_launch_ms": avg_ms,
                     "launches_timed": tp_["collide_launches"], "peak_source": peak_kind},
        "fp64": fp64,
        "fp32_over_fp64": (value / fp64["mlups"]) if fp64 else None,
        "adjoint_over_forward": (adjoint["backward_ms"] / adjoint["forward_ms"]) if adjoint else None,
        "adjoint": adjoint,
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
