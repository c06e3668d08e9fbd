"""Boundary solvers on the membrane (BoundarySolverNoFlux, BoundarySolverNoFluxD2Q5;
BoundarySolverNoFlux.cpp:36-105, BoundarySolverNoFluxD2Q5.cpp:37-106), named
per connection as in apps/config/tutorial_02_geometry.txt, against the
reference build itself: FP64 results identical, including the reference's
pre-advect loop that serves only the first listed species."""
import os

import numpy as np
import pytest

from lbibcell_b200 import configs

pytestmark = pytest.mark.gpu

A, B = configs.SPECIES_NAMES[0], configs.SPECIES_NAMES[1]


@pytest.fixture(scope="module")
def lbib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from lbibcell_b200 import build, runner
    build.build()
    return runner


@pytest.mark.parametrize("boundary", [
    [("BoundarySolverNoFluxD2Q5", A)],
    [("BoundarySolverNoFluxD2Q5", A), ("BoundarySolverNoFluxD2Q5", B)],
    [("BoundarySolverNoFluxD2Q5", B), ("BoundarySolverNoFlux", A)],
], ids=["d2q5-A", "d2q5-A-B", "both-kinds"])
def test_noflux_matches_reference(lbib, oracle_mod, tmp_path, boundary):
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    cfg = configs.toy(n=48, r=8.0, nodes=80, iterations=60, report_step=30, species=2)
    cfg.boundary = boundary
    paths = cfg.write(str(tmp_path / "cfg"))
    dumps = oracle_mod.run_reference(paths, str(tmp_path / "ref"))
    sim = lbib.Simulation(paths, lbib.FP64)
    done = 0
    for t in (30, 60):
        sim.step(t - done)
        done = t
        ref = dumps[t]
        lat = sim.lattice()
        for name in ("f", "g", "vel", "dom"):
            a, b = getattr(lat, name), getattr(ref, name)
            assert np.array_equal(a, b), f"t={t} {name}: max |diff| {np.abs(a.astype(float) - b.astype(float)).max()}"
        ids, node = sim.membrane()
        assert np.array_equal(node[:, :2], ref.node[:, :2]), f"t={t}: membrane positions differ"


def test_noflux_changes_the_species(lbib, tmp_path):
    """The boundary condition acts: with it the species field differs from the
    run without it, and the FP32-shifted run stays close to the FP64 one."""
    base = configs.toy(n=48, r=8.0, nodes=80, iterations=60, species=2)
    with_nf = configs.toy(n=48, r=8.0, nodes=80, iterations=60, species=2)
    with_nf.boundary = [("BoundarySolverNoFluxD2Q5", A)]
    s0 = lbib.Simulation(base.write(str(tmp_path / "a")), lbib.FP64)
    s1 = lbib.Simulation(with_nf.write(str(tmp_path / "b")), lbib.FP64)
    s2 = lbib.Simulation(with_nf.write(str(tmp_path / "c")), lbib.FP32_SHIFTED)
    for s in (s0, s1, s2):
        s.step(40)
    c0, c1, c2 = s0.concentrations(), s1.concentrations(), s2.concentrations()
    assert np.abs(c1[0] - c0[0]).max() > 1e-6
    assert np.abs(c2 - c1).max() <= 1e-5 * np.abs(c1).max()


def test_differentiated_runs_refuse_boundary_solvers(lbib, tmp_path):
    cfg = configs.toy(n=48, r=8.0, nodes=80, species=1)
    cfg.boundary = [("BoundarySolverNoFluxD2Q5", A)]
    sim = lbib.Simulation(cfg.write(str(tmp_path)), lbib.FP64)
    with pytest.raises(lbib.LbibError) as e:
        sim.diff_begin(4)
    assert e.value.code == 91


def test_unknown_boundary_solver(lbib, tmp_path):
    cfg = configs.toy(n=48, r=8.0, nodes=80, species=1)
    cfg.boundary = [("NoSuchBoundarySolver", A)]
    with pytest.raises(lbib.LbibError) as e:
        lbib.Simulation(cfg.write(str(tmp_path)), lbib.FP64)
    assert e.value.code == 90
