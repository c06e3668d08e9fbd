"""DiracD2Q5 (libs/LbmLib/src/solver/CDESolver/DiracD2Q5.cpp) on the device.

* Known answer: the solver starts from the 2D heat kernel at t = 50 with
  D = 0.04 centred at (32, 32) (:39-66); with tau = 0.62 the D2Q5 lattice
  diffuses with D = (tau - 1/2) / 3 = 0.04, so after T steps the field is the
  heat kernel at t = 50 + T up to the lattice's discretisation error (about 2 %
  of the peak at T = 100, checked here at 3 %), and the total stays constant.
  The FP64 field also equals a numpy restatement of the same lattice
  dynamics to rounding.
* Against the reference build (FP64, exact): a moving membrane near the
  kernel, where DiracD2Q5's advect keeps the populations of links with a
  boundary node (:166-180) and nodes that change domain re-initialise from
  their neighbours (:182-228).
"""
import math
import os

import numpy as np
import pytest

from lbibcell_b200 import configs

pytestmark = pytest.mark.gpu

TAU = 0.62


@pytest.fixture(scope="module")
def lbib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from lbibcell_b200 import build, runner
    build.build()
    return runner


def _far_cell(n=128, T=100):
    # one small cell far from the kernel, no membrane forces, no outlet
    cfg = configs.Config(name="dirac", nx=n, ny=n, tau_fluid=1.0, iterations=T, report_step=T,
                         cells=[(1, configs.circle(100.0, 100.0, 5.0, 64, phase=0.1))],
                         species=[configs.Species("DiracD2Q5", TAU)], outlet=False, tension=None, area=None)
    return cfg


def _numpy_diffusion(n, T):
    """The same D2Q5 BGK dynamics at rest (no membrane in reach): the
    heat-kernel start, collide, then T times stream + collide."""
    y, x = np.mgrid[0:n, 0:n].astype(float)
    D, t0 = 0.04, 50.0
    dist = np.sqrt((32 - x) ** 2 + (32 - y) ** 2)
    k = np.exp(-dist * dist / (4.0 * D * t0)) / (4.0 * math.pi * D * t0)
    g = np.stack([k * 0.2] * 5)

    def collide(g):
        C = g.sum(0)
        eq = np.stack([C / 3.0, C / 6.0, C / 6.0, C / 6.0, C / 6.0])
        return g - g / TAU + eq / TAU

    g = collide(g)
    for _ in range(T):
        g[1] = np.roll(g[1], 1, axis=1)
        g[2] = np.roll(g[2], 1, axis=0)
        g[3] = np.roll(g[3], -1, axis=1)
        g[4] = np.roll(g[4], -1, axis=0)
        g = collide(g)
    return g.sum(0)


@pytest.mark.parametrize("precision", [0, 1])
def test_heat_kernel_known_answer(lbib, tmp_path, precision):
    n, T = 128, 100
    sim = lbib.Simulation(_far_cell(n, T).write(str(tmp_path)), precision)
    C0 = sim.lattice().g[0].sum(1)
    sim.step(T)
    C = sim.lattice().g[0].sum(1).reshape(n, n)
    y, x = np.mgrid[0:n, 0:n].astype(float)
    r2 = (32 - x) ** 2 + (32 - y) ** 2
    t = 50.0 + T
    exact = np.exp(-r2 / (4 * 0.04 * t)) / (4 * math.pi * 0.04 * t)
    near = r2 < 100
    err = np.abs(C - exact)[near].max() / exact.max()
    assert err < 0.03, err
    assert abs(C.sum() - C0.sum()) <= (1e-12 if precision == 0 else 1e-5) * C0.sum()
    want = _numpy_diffusion(n, T)
    scale = np.abs(want).max()
    tol = 1e-12 if precision == 0 else 1e-5
    assert np.abs(C - want).max() <= tol * scale


def test_dirac_with_membrane_matches_reference(lbib, oracle_mod, tmp_path):
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    cfg = configs.Config(name="dirac_membrane", nx=64, ny=64, tau_fluid=1.0, iterations=40, report_step=10,
                         cells=[(1, configs.circle(38.0, 35.0, 8.0, 100, phase=0.1))],
                         species=[configs.Species("DiracD2Q5", TAU)], tension=(0.1, 10), area=(1.3, 0.01, 0.004))
    paths = cfg.write(str(tmp_path / "cfg"))
    ref = oracle_mod.run_reference(paths, str(tmp_path / "ref"))
    sim = lbib.Simulation(paths, lbib.FP64)
    done = 0
    for t in (0, 10, 20, 30, 40):
        sim.step(t - done)
        done = t
        lat = sim.lattice()
        st = ref[t]
        for k in ("f", "g", "vel", "force", "dom"):
            a, b = getattr(lat, k), getattr(st, k)
            assert np.array_equal(a, b), (t, k, float(np.nanmax(np.abs(a.astype(float) - b.astype(float)))))
        ids, node = sim.membrane()
        assert np.array_equal(node, st.node), t


def test_dirac_refusals(lbib, tmp_path):
    cfg = _far_cell(128, 10)
    cfg.force_model = "GuoZhengShi2002ForceModel"
    with pytest.raises(lbib.LbibError) as e:
        lbib.Simulation(cfg.write(str(tmp_path / "a")), lbib.FP64)
    assert e.value.code == 90
    sim = lbib.Simulation(_far_cell(128, 10).write(str(tmp_path / "b")), lbib.FP64)
    with pytest.raises(lbib.LbibError) as e:
        sim.diff_begin(4, 2)
    assert e.value.code == 91
