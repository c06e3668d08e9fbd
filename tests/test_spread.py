"""The immersed-boundary spread (SimulationRunner::distributeForce,
SimulationRunner.cpp:425-453; GeometryNode::distributeForce,
GeometryNode.cpp:228-235) in its two device forms on the same membrane state:
the FP64 ordered gather (identical to the reference build, tests elsewhere)
and the FP32-shifted fixed-point scatter.  The scatter's per-node sums are
exact up to the 2^-44 rounding of each contribution, then rounded once to
FP32, so every lattice node's force agrees within that bound: a missing or
doubled contribution would not.
"""
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


def test_fixed_point_spread_matches_ordered_gather(lbib, tmp_path):
    cells = configs.hex_tissue(320, 320, 44.0, 20.0, 2.0, 250, 0, cols=5, rows=5)
    # a cell centred on a lattice node with its first node on a lattice line:
    # that node's stencil is 5 wide (the last writer holds each slot)
    cells.append((26, configs.circle(40.0, 40.0, 12.0, 120, phase=0.0)))
    cfg = configs.Config(name="spread", nx=320, ny=320, tau_fluid=1.0, iterations=10, report_step=10, cells=cells,
                         species=[configs.Species(configs.SPECIES_NAMES[0], 0.8, source={1: 1e-3})])
    paths = cfg.write(str(tmp_path))
    a = lbib.Simulation(paths, lbib.FP64)
    b = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    # the force list starts empty (the tension records follow the first
    # step's bio stage): a constant force (type 2) on every node, the same
    # in both, so that the first step's spread acts on identical positions
    ids, _ = a.membrane()
    rng = np.random.default_rng(3)
    par = np.zeros((len(ids), 4))
    par[:, :2] = rng.uniform(-2e-3, 2e-3, (len(ids), 2))
    for sim in (a, b):
        sim.add_forces(np.full(len(ids), 2), ids, np.zeros(len(ids)), par)
        sim.step(1)
    fa, fb = a.lattice().force, b.lattice().force
    assert np.abs(fa).max() > 1e-4
    bound = 2.0 ** -23 * np.abs(fa) + 64 * 2.0 ** -44
    bad = np.abs(fb - fa) > bound
    assert not bad.any(), (int(bad.sum()), float(np.abs(fb - fa).max()))
