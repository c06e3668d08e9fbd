"""The reference's CDE reaction family on the device (CDESolver/*.cpp):
tutorial_02_CDESolverD2Q5_{L,R} (gamma(b - R^2 L), gamma(a - R + R^2 L),
deltaT 1e-4), SchnakenbergD2Q5{u,v} (deltaT 20 / Iterations, diagonal
re-initialisation) and CDESolverD2Q5BMP with CDESolverD2Q5HH, against the
reference build itself (FP64, exact).

The reference seeds the random initial conditions of tutorial_02 and
Schnakenberg from std::random_device, so both runs restart from one solver
file (SimulationRunner::initSolvers(file)) written by this library at
iteration 0."""
import os

import numpy as np
import pytest

from lbibcell_b200 import configs
from lbibcell_b200.configs import Species

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lbib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from lbibcell_b200 import build, runner
    build.build()
    return runner


# species (name, tau); Iterations in the parameter file; iterations run
CASES = {
    "tutorial_02": ([("tutorial_02_CDESolverD2Q5_L", 1.0), ("tutorial_02_CDESolverD2Q5_R", 1.2)], 40, 40),
    # deltaT = 20 / 200000: gamma * deltaT = 0.08, a stable explicit step
    "schnakenberg": ([("SchnakenbergD2Q5u", 1.0), ("SchnakenbergD2Q5v", 0.9)], 200000, 40),
    "bmp_hh": ([("CDESolverD2Q5BMP", 1.0), ("CDESolverD2Q5HH", 0.8)], 40, 40),
    "signal_coupled": ([("tutorial_01_CDESolverD2Q5_SIGNAL", 1.0), ("tutorial_02_CDESolverD2Q5_L", 0.9),
                        ("tutorial_02_CDESolverD2Q5_R", 1.1)], 40, 40),
}


def _cfg(species, iterations):
    # r 12 in a 64^2 lattice: the cell moves under tension, so nodes change
    # domain and the re-initialisation variants run every step
    cfg = configs.toy(n=64, r=12.0, nodes=120, iterations=iterations, report_step=10, species=1)
    cfg.area = None
    cfg.species = [Species(n, t) for n, t in species]
    return cfg


def _compare(sim, ref, t):
    lat = sim.lattice()
    for name in ("f", "g", "vel", "dom"):
        a, b = getattr(lat, name), getattr(ref, name)
        assert np.array_equal(a, b), f"t={t} {name}: max |diff| {np.nanmax(np.abs(a.astype(float) - b.astype(float)))}"
    ids, node = sim.membrane()
    assert np.array_equal(ids, ref.ids) and np.array_equal(node, ref.node), f"t={t}: membrane differs"


@pytest.mark.parametrize("case", sorted(CASES))
def test_reactions_match_reference(lbib, oracle_mod, tmp_path, case):
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    species, iters, run = CASES[case]
    paths = _cfg(species, iters).write(str(tmp_path / "cfg"))
    start = lbib.Simulation(paths, lbib.FP64).write_simulation(str(tmp_path / "start"))
    dumps = oracle_mod.run_reference(paths, str(tmp_path / "ref"), extra=("restart", start["solver"], "run", run))
    sim = lbib.Simulation(paths, lbib.FP64)
    sim.load_solvers(start["solver"])
    done = 0
    for t in range(10, run + 1, 10):
        sim.step(t - done)
        done = t
        _compare(sim, dumps[t], t)
    g = sim.lattice().g
    assert np.isfinite(g).all()
    # the reactions act: the species differ from a run without them
    assert float(np.abs(g).sum()) > 0


def test_reactions_fp32_shifted(lbib, tmp_path):
    """The coupled reactions in the FP32-shifted kernel: the species stay
    within 1e-5 (relative to the largest concentration slot) of the FP64 run
    started from the same solver file."""
    species, iters, _ = CASES["signal_coupled"]
    paths = _cfg(species, iters).write(str(tmp_path / "cfg"))
    start = lbib.Simulation(paths, lbib.FP64).write_simulation(str(tmp_path / "start"))
    a = lbib.Simulation(paths, lbib.FP64)
    b = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    a.load_solvers(start["solver"])
    b.load_solvers(start["solver"])
    a.step(30)
    b.step(30)
    ga, gb = a.lattice().g, b.lattice().g
    assert np.abs(ga - gb).max() <= 1e-5 * np.abs(ga).max()


def test_unsupported_cde_solver_is_refused(lbib, tmp_path):
    """The D2Q4 solvers (CDESolverD2Q4, DiracD2Q4, SchnakenbergD2Q4u/v) are
    not built; a create call that names one fails."""
    paths = _cfg([("CDESolverD2Q4", 1.0)], 20).write(str(tmp_path))
    with pytest.raises(lbib.LbibError) as e:
        lbib.Simulation(paths, lbib.FP64)
    assert e.value.code == 90


def test_missing_partner_is_refused(lbib, tmp_path):
    """PhysicalNode::getCDESolverSlow throws for a solver the node lacks: a
    coupled species without its partner fails the create call."""
    paths = _cfg([("tutorial_02_CDESolverD2Q5_R", 1.0)], 20).write(str(tmp_path))
    with pytest.raises(lbib.LbibError) as e:
        lbib.Simulation(paths, lbib.FP64)
    assert e.value.code == 90
