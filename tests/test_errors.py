"""Failure detection without a GPU fault: errors the reference raises with
lbm_fail / UtilLib::Exception come back as LBIB_ERR_* codes, from the host
(bad files, geometry at the edge) and from the device (a membrane node moving
faster than the lattice allows, SpeedCheck in LagrangianPoint::setVelocity,
LagrangianPoint.cpp:92-103), and the handle then refuses further work."""
import ctypes

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


def test_missing_file(lbib, tmp_path):
    paths = configs.toy(n=48, r=8.0, nodes=80).write(str(tmp_path))
    paths["parameters"] = str(tmp_path / "absent.txt")
    with pytest.raises(lbib.LbibError) as e:
        lbib.Simulation(paths, lbib.FP64)
    assert e.value.code == 90


def test_unknown_plugin(lbib, tmp_path):
    paths = configs.toy(n=48, r=8.0, nodes=80).write(str(tmp_path))
    with open(paths["plugins"], "a") as f:
        f.write("BioSolver\tNoSuchSolver\n")
    with pytest.raises(lbib.LbibError) as e:
        lbib.Simulation(paths, lbib.FP64)
    assert e.value.code == 90


@pytest.mark.parametrize("where, code", [("west", 10), ("south", 11), ("east", 12), ("north", 13)])
def test_geometry_at_the_edge(lbib, tmp_path, where, code):
    """connectGeometryNodesToPhysicalNodes refuses nodes within 2 lu of an edge
    (GeometryHandler.cpp:618-636)."""
    n = 48
    centre = {"west": (9.5, 24.0), "south": (24.0, 9.5), "east": (38.5, 24.0), "north": (24.0, 38.5)}[where]
    cfg = configs.toy(n=n, r=8.0, nodes=80)
    cfg.cells = [(1, configs.circle(centre[0], centre[1], 8.0, 80))]
    with pytest.raises(lbib.LbibError) as e:
        sim = lbib.Simulation(cfg.write(str(tmp_path)), lbib.FP64)
        sim.step(1)
    assert e.value.code == code


def test_device_error_stops_the_run(lbib, tmp_path):
    """A fluid moving at 0.9 lattice units per step carries the membrane
    faster than the lattice allows: the device raises the error inside the
    step, the host reports it with the node, and later calls keep returning it."""
    sim = lbib.Simulation(configs.toy(n=64, r=10.0, nodes=100).write(str(tmp_path)), lbib.FP64)
    c = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]], float)
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    u = np.array([0.9, 0.0])
    cu = c @ u
    feq = w * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * u @ u)
    lat = sim.lattice()
    sim.set_lattice(f=np.tile(feq, (lat.f.shape[0], 1)))
    with pytest.raises(lbib.LbibError) as e:
        sim.step(5)
    assert e.value.code == 20, e.value
    assert 0 <= e.value.index < 100
    with pytest.raises(lbib.LbibError) as e2:
        sim.step(1)
    assert e2.value.code == 20
