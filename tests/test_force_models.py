"""FluidSolver's force models and its velocity initialisation on the device.

* GuoZhengShi2002ForceModel (GuoZhengShi2002ForceModel.cpp:29-78), the
  alternative base class FluidSolver.hpp:41 names in a comment, selected per
  handle by a "ForceModel" plugin line: FP64 identical to the reference built
  with that base class (tests/golden/guo48.npz, from oracle/_ref/ref_driver_guo),
  including the NE coefficient as the reference writes it (:51); the corrected
  coefficient identical to the oracle's restatement of it; FP32-shifted close
  to FP64.
* SimulationRunner::initSolvers(Field<double>) / FluidSolver::initWithVelocity
  (SimulationRunner.cpp:308-320, FluidSolver.cpp:62-101) through
  lbib_init_velocity: identical to the reference build.
"""
import os

import numpy as np
import pytest

from lbibcell_b200 import configs

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIELDS = ("f", "g", "vel", "force", "dom", "ctype")


@pytest.fixture(scope="module")
def lbib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from lbibcell_b200 import build, runner
    build.build()
    return runner


def _toy48(model=None):
    cfg = configs.toy(n=48, r=8.0, nodes=80, iterations=60, report_step=30, species=1)
    cfg.force_model = model
    return cfg


def _state(sim):
    lat = sim.lattice()
    ids, node = sim.membrane()
    out = {k: getattr(lat, k) for k in FIELDS}
    out.update(ids=ids, node=node, conn=sim.connections())
    return out


def _exact(got, want, what):
    for k, v in got.items():
        w = want(k)
        assert v.shape == w.shape, (what, k, v.shape, w.shape)
        if not np.array_equal(v, w):
            d = np.abs(v.astype(np.float64) - w.astype(np.float64))
            raise AssertionError(f"{what} {k}: max |diff| {d.max():.3e}")


def test_guo_fp64_matches_reference_build(lbib, tmp_path):
    gold = np.load(os.path.join(GOLD, "guo48.npz"))
    sim = lbib.Simulation(_toy48("GuoZhengShi2002ForceModel").write(str(tmp_path)), lbib.FP64)
    prev = 0
    for t in (0, 30, 60):
        sim.step(t - prev)
        prev = t
        _exact(_state(sim), lambda k: gold[f"{k}_{t}"], f"t={t}")


def test_guo_corrected_fp64_matches_oracle(lbib, oracle_mod, tmp_path):
    paths = _toy48("GuoZhengShi2002ForceModelCorrected").write(str(tmp_path))
    sim = lbib.Simulation(paths, lbib.FP64)
    o = oracle_mod.Oracle(paths)
    for n in (1, 29, 30):
        sim.step(n)
        o.step(n)
        st = o.state()
        _exact(_state(sim), lambda k: getattr(st, k), f"after {n}")


@pytest.mark.parametrize("model", ["GuoZhengShi2002ForceModel", "GuoZhengShi2002ForceModelCorrected"])
def test_guo_fp32_shifted_close_to_fp64(lbib, tmp_path, model):
    """FP32-shifted Guo vs FP64 Guo on config 1 (200x200 single cell) after 500
    steps: relative max-norm errors <= 1e-5 (rho-1 by max|rho-1|, u by max|u|,
    c by max c), membrane positions within 1e-6 lu."""
    cfg = configs.config1()
    cfg.force_model = model
    paths = cfg.write(str(tmp_path))
    a = lbib.Simulation(paths, lbib.FP64)
    b = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    a.step(500)
    b.step(500)
    la, lb = a.lattice(), b.lattice()
    ra, rb = la.f.sum(1) - 1.0, lb.f.sum(1) - 1.0
    e_rho = np.abs(ra - rb).max() / np.abs(ra).max()
    e_u = np.abs(la.vel - lb.vel).max() / np.abs(la.vel).max()
    ca, cb = la.g.sum(2), lb.g.sum(2)
    e_c = np.abs(ca - cb).max() / np.abs(ca).max()
    _, na = a.membrane()
    _, nb = b.membrane()
    e_x = np.abs(na[:, :2] - nb[:, :2]).max() if na.shape == nb.shape else np.inf
    print(f"{model} FP32-shifted vs FP64: rho {e_rho:.2e} u {e_u:.2e} c {e_c:.2e} x {e_x:.2e}")
    assert e_rho <= 1e-5 and e_u <= 1e-5 and e_c <= 1e-5
    assert e_x <= 1e-6


def test_force_model_refusals(lbib, tmp_path):
    with pytest.raises(lbib.LbibError) as e:
        lbib.Simulation(_toy48("NoSuchForceModel").write(str(tmp_path / "a")), lbib.FP64)
    assert e.value.code == 90
    sim = lbib.Simulation(_toy48("GuoZhengShi2002ForceModel").write(str(tmp_path / "b")), lbib.FP64)
    with pytest.raises(lbib.LbibError) as e:
        sim.diff_begin(10, 5)
    assert e.value.code == 91


@pytest.mark.parametrize("species", [1, 2])
def test_init_velocity_matches_reference(lbib, oracle_mod, tmp_path, species):
    """initSolvers(Field<double>(0.02, -0.01)) after the plain initSolvers, then
    30 full steps: every array identical to the reference build at t = 10,
    20, 30 (the reference's dump at t = 0 precedes the velocity set-up)."""
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    cfg = configs.toy(n=48, r=8.0, nodes=80, iterations=30, report_step=10, species=species)
    paths = cfg.write(str(tmp_path / "cfg"))
    dumps = oracle_mod.run_reference(paths, str(tmp_path / "ref"), extra=("velocity", "0.02", "-0.01"))
    sim = lbib.Simulation(paths, lbib.FP64)
    sim.init_velocity(0.02, -0.01)
    lat = sim.lattice()
    assert np.all(lat.vel[:, 0] == 0.02) and np.all(lat.vel[:, 1] == -0.01)
    prev = 0
    for t in (10, 20, 30):
        sim.step(t - prev)
        prev = t
        st = dumps[t]
        _exact(_state(sim), lambda k: getattr(st, k), f"t={t}")


def test_init_velocity_fp32_shifted(lbib, tmp_path):
    paths = configs.toy(n=48, r=8.0, nodes=80, iterations=30, report_step=10, species=1).write(str(tmp_path))
    a = lbib.Simulation(paths, lbib.FP64)
    b = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    for s in (a, b):
        s.init_velocity(0.02, -0.01)
    la, lb = a.lattice(), b.lattice()
    assert np.abs(la.f - lb.f).max() < 1e-7
    a.step(20)
    b.step(20)
    la, lb = a.lattice(), b.lattice()
    assert np.abs(la.vel - lb.vel).max() / np.abs(la.vel).max() < 1e-5
