"""The cell-junction bio solver (tutorial_01_BioSolverCellJunction.cpp:47-99;
the tutorial_02 and plain BioSolverCellJunction are the same solver) on the
device, against the reference build itself: every 10th iteration all type-7
forces go, and each node gets a spring to the closest node of another cell
within 1 lu, and that node one back.  FP64 results identical, and the force
list written by writeSimulation holds the same records in the same order."""
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


def _records(path):
    """ForceSolver::writeForceSolver lines as (type, id1, id2 or -1) and parameters."""
    keys, pars = [], []
    for line in open(path):
        if not line.strip() or line.startswith("#"):
            continue
        v = line.split()
        t = int(v[0])
        if t in (0, 5, 6, 7):
            keys.append((t, int(v[1]), int(v[2])))
            pars.append([float(x) for x in v[3:]])
        else:
            keys.append((t, int(v[1]), -1))
            pars.append([float(x) for x in v[2:]])
    return keys, pars


CASES = {
    # junctions after the tension plugin; tension renewed on the cleared list
    "after-tension": dict(tension=(0.1, 10), bio_first=False),
    # junctions first and tension every 5th iteration: the renewals between the
    # multiples of 10 edit a list that holds the junction springs
    "first-tension5": dict(tension=(0.1, 5), bio_first=True),
    "tutorial_02": dict(tension=(0.1, 10), bio_first=False, name="tutorial_02_BioSolverCellJunction"),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_junctions_match_reference(lbib, oracle_mod, tmp_path, case):
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    cfg = configs.junction_quad(iterations=60, report_step=30, **CASES[case])
    paths = cfg.write(str(tmp_path / "cfg"))
    dumps = oracle_mod.run_reference(paths, str(tmp_path / "ref"), extra=("write", str(tmp_path / "ref_out")))
    sim = lbib.Simulation(paths, lbib.FP64)
    done = 0
    for t in (30, 60):
        sim.step(t - done)
        done = t
        ref = dumps[t]
        lat = sim.lattice()
        for name in ("f", "g", "vel", "force", "dom"):
            a, b = getattr(lat, name), getattr(ref, name)
            assert np.array_equal(a, b), f"t={t} {name}: max |diff| {np.abs(a.astype(float) - b.astype(float)).max()}"
        ids, node = sim.membrane()
        assert np.array_equal(ids, ref.ids)
        assert np.array_equal(node, ref.node), f"t={t}: membrane state differs"
    ours = sim.write_simulation(str(tmp_path / "ours"))
    k_ref, p_ref = _records(str(tmp_path / "ref_out") + "_force.txt")
    k_our, p_our = _records(ours["force"])
    assert sum(1 for k in k_ref if k[0] == 7) > 100  # the geometry does form junctions
    assert k_our == k_ref
    # the reference writes parameters with 6 significant digits
    for a, b in zip(p_our, p_ref):
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=0)


def test_junctions_fp32_shifted(lbib, tmp_path):
    """The FP32-shifted run with junctions: same force records as the FP64 run
    after 30 steps, membrane positions within 1e-6 lu."""
    paths = configs.junction_quad(iterations=30).write(str(tmp_path / "cfg"))
    a = lbib.Simulation(paths, lbib.FP64)
    b = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    a.step(30)
    b.step(30)
    _, na = a.membrane()
    _, nb = b.membrane()
    assert na.shape == nb.shape
    assert np.abs(na[:, :2] - nb[:, :2]).max() <= 1e-6
    ka, _ = _records(a.write_simulation(str(tmp_path / "a"))["force"])
    kb, _ = _records(b.write_simulation(str(tmp_path / "b"))["force"])
    assert ka == kb and sum(1 for k in ka if k[0] == 7) > 100
