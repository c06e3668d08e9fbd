"""The FP32-shifted stream-collide kernel in its two forms: four nodes per
thread (128-bit row loads, the x-shifted pull sources by warp shuffle; the
plain modes on rows of a multiple of 256 nodes; LBIB_COLLIDE_X4=1) and one
node per thread (the default).  Both run the same per-node expressions, so the
states they produce are compared to the last bit: lattice-only steps with a
force field and the box outlet, and full steps with moving membranes, two and
three species, per-domain and per-node mass sources."""
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


def _tissue(tmp_path, species, division=False):
    cells = configs.hex_tissue(512, 256, 44.0, 20.0, 2.0, 250, 1, cols=10, rows=5)
    taus = (0.8, 1.2, 1.0)
    sp = [configs.Species(configs.SPECIES_NAMES[k], taus[k], decay=1e-4 * k, source={1: 1e-3, 7: 2e-3})
          for k in range(species)]
    cfg = configs.Config(name="strip50", nx=512, ny=256, tau_fluid=1.0, iterations=60, report_step=30, cells=cells,
                         species=sp)
    if division:  # the area regulator then writes a per-node mass source
        cfg.bio = ["LbibCellDivision\tfactor\t2.0\tfrequency\t100"]
    return cfg.write(str(tmp_path))


def _run(lbib, paths, monkeypatch, scalar, steps, lattice_only):
    if scalar:
        monkeypatch.delenv("LBIB_COLLIDE_X4", raising=False)
    else:
        monkeypatch.setenv("LBIB_COLLIDE_X4", "1")
    sim = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    sim.step(2)  # forces on the lattice
    if lattice_only:
        sim.lattice_step(steps, outlet=True)
    else:
        sim.step(steps)
    lat = sim.lattice()
    ids, node = sim.membrane()
    sim.close()
    monkeypatch.delenv("LBIB_COLLIDE_X4", raising=False)
    return lat, node


@pytest.mark.parametrize("species,division", [(2, False), (3, False), (2, True)])
@pytest.mark.parametrize("lattice_only", [True, False])
def test_four_nodes_per_thread_equal_one(lbib, tmp_path, monkeypatch, species, division, lattice_only):
    paths = _tissue(tmp_path, species, division)
    a, na = _run(lbib, paths, monkeypatch, False, 25, lattice_only)
    b, nb = _run(lbib, paths, monkeypatch, True, 25, lattice_only)
    for k in ("f", "g", "vel", "force", "dom"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    np.testing.assert_array_equal(na, nb)
