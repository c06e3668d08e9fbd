"""Checkpoint files in the reference's formats (SimulationRunner::writeSimulation
and initSolvers(file)): a run written by this library restarts in the reference
build, and a run written by the reference build restarts here; both restarted
runs then agree bit for bit (FP64)."""
import os

import numpy as np
import pytest

from lbibcell_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lbib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from lbibcell_b200 import build, runner
    build.build()
    return runner


def _cfg(iterations):
    cfg = configs.toy(n=48, r=8.0, nodes=80, iterations=iterations, report_step=10, species=2)
    cfg.area = None  # the area regulator's targets are plugin state that no file holds
    return cfg


def _same(sim, ref_state, what):
    lat = sim.lattice()
    for name in ("f", "g", "vel", "dom"):
        a, b = getattr(lat, name), getattr(ref_state, name)
        assert np.array_equal(a, b), f"{what}: {name} differs (max {np.abs(a.astype(float) - b.astype(float)).max()})"
    ids, node = sim.membrane()
    assert np.array_equal(ids, ref_state.ids), f"{what}: membrane ids differ"
    assert np.array_equal(node[:, :2], ref_state.node[:, :2]), f"{what}: membrane positions differ"


def _at_iteration(dumps, it):
    """The reference dump taken at global iteration `it` (runSimulation runs
    `Iterations` further steps from CurrentIterations and labels its reports by
    the steps of this run)."""
    for k, st in dumps.items():
        if k != "stdout" and st.current_iteration == it:
            return st
    raise AssertionError(f"no reference dump at iteration {it}")


def _restart_paths(written, plugins):
    return {"parameters": written["parameters"], "geometry": written["geometry"], "force": written["force"],
            "plugins": plugins}


def test_written_files_match_state(lbib, tmp_path):
    paths = _cfg(40).write(str(tmp_path / "cfg"))
    sim = lbib.Simulation(paths, lbib.FP64)
    sim.step(20)
    w = sim.write_simulation(str(tmp_path / "gpu"))
    # parameters: the current iteration and the rest of the file
    par = dict(line.split("\t", 1) for line in open(w["parameters"]).read().splitlines()[1:])
    assert par["CurrentIterations:"].strip() == "20" and par["SizeX:"].strip() == "48"
    # geometry: every node's position to the last bit
    ids, node = sim.membrane()
    rows = [l.split("\t") for l in open(w["geometry"]).read().split("#Connection")[0].splitlines()[1:]]
    assert [int(r[0]) for r in rows] == ids.tolist()
    assert np.array_equal(np.array([[float(r[1]), float(r[2])] for r in rows]), node[:, :2])
    # solver dump: reloading it into a fresh handle gives the same distributions
    other = lbib.Simulation(_restart_paths(w, paths["plugins"]), lbib.FP64)
    other.load_solvers(w["solver"])
    a, b = sim.lattice(), other.lattice()
    assert np.array_equal(a.f, b.f) and np.array_equal(a.g, b.g)


def test_gpu_checkpoint_restarts_in_reference(lbib, oracle_mod, tmp_path):
    """This library writes at iteration 20; the reference build and this library
    both restart from the files and run to iteration 40."""
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    paths = _cfg(40).write(str(tmp_path / "cfg"))
    sim = lbib.Simulation(paths, lbib.FP64)
    sim.step(20)
    w = sim.write_simulation(str(tmp_path / "gpu"))
    rpaths = _restart_paths(w, paths["plugins"])
    dumps = oracle_mod.run_reference(rpaths, str(tmp_path / "ref"), extra=("restart", w["solver"]))
    again = lbib.Simulation(rpaths, lbib.FP64)
    again.load_solvers(w["solver"])
    again.step(20)
    assert again.sizes()["iteration"] == 40
    _same(again, _at_iteration(dumps, 40), "restart from this library's files")


def test_reference_checkpoint_restarts_here(lbib, oracle_mod, tmp_path):
    """The reference build writes at iteration 20 (its own 6-digit text); it
    and this library both restart from those files and run to iteration 40."""
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    paths = _cfg(20).write(str(tmp_path / "cfg"))
    prefix = str(tmp_path / "refw")
    oracle_mod.run_reference(paths, str(tmp_path / "ref0"), extra=("write", prefix))
    w = {k: f"{prefix}_{k}.txt" for k in ("force", "geometry", "parameters", "solver")}
    # the written parameters say CurrentIterations 20, Iterations 20: a restart
    # runs 20 further steps
    rpaths = _restart_paths(w, paths["plugins"])
    dumps = oracle_mod.run_reference(rpaths, str(tmp_path / "ref1"), extra=("restart", w["solver"]))
    sim = lbib.Simulation(rpaths, lbib.FP64)
    sim.load_solvers(w["solver"])
    sim.step(20)
    assert sim.sizes()["iteration"] == 40
    _same(sim, _at_iteration(dumps, 40), "restart from the reference's files")
