"""GeometryHandler::computeAreas through lbib_areas in its two ways.

* Right after lbib_step with an area regulator registered, the areas the
  step's bio stage formed come back with the step's status word: no device
  work at the call.
* After any other API call (here a lattice download) they are formed again on
  the device: in ring order (FP64) or from the exact fixed-point sums
  (FP32-shifted).

Both ways give the same values to the last bit, on both precisions, and the
FP64 values equal the ring-order sum the reference forms
(GeometryHandler.cpp:101-134) as restated by the oracle.
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


def _tissue(tmp_path, area=True):
    cells = configs.hex_tissue(320, 320, 44.0, 20.0, 2.0, 250, 0, cols=5, rows=5)
    cfg = configs.Config(name="hex25", nx=320, ny=320, tau_fluid=1.0, iterations=40, report_step=20, cells=cells,
                         species=[configs.Species(configs.SPECIES_NAMES[0], 0.8, source={1: 1e-3})])
    if not area:
        cfg.area = None
    return cfg.write(str(tmp_path))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("area", [True, False])
def test_areas_after_step_equal_recomputed(lbib, tmp_path, precision, area):
    sim = lbib.Simulation(_tissue(tmp_path, area), precision)
    for steps in (1, 9, 1):
        sim.step(steps)
        d1, a1 = (x.copy() for x in sim.areas_array())
        d1b, a1b = (x.copy() for x in sim.areas_array())  # a second call in a row
        sim.lattice()  # any other call: the next areas are formed again
        d2, a2 = (x.copy() for x in sim.areas_array())
        assert len(d1) == 25
        np.testing.assert_array_equal(d1, d2)
        np.testing.assert_array_equal(d1b, d1)
        np.testing.assert_array_equal(a1, a2)
        np.testing.assert_array_equal(a1b, a1)
        assert np.all(a1 > 100.0)


def test_areas_fp64_equal_oracle(lbib, oracle_mod, tmp_path):
    paths = _tissue(tmp_path)
    sim = lbib.Simulation(paths, lbib.FP64)
    o = oracle_mod.Oracle(paths)
    sim.step(7)
    o.step(7)
    got = sim.areas()
    want = o.areas()
    assert got.keys() == want.keys()
    for d in got:
        assert got[d] == want[d], d


def test_areas_fp32_close_to_fp64(lbib, tmp_path):
    paths = _tissue(tmp_path)
    a = lbib.Simulation(paths, lbib.FP64)
    b = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    aa, ab = a.areas(), b.areas()
    assert aa.keys() == ab.keys()
    for d in aa:
        # the same positions: each of a cell's n shoelace terms is rounded to
        # a multiple of 2^-24 (|error| <= 2^-25, halved in the area), so the
        # areas differ by at most n 2^-26 (3.7e-6 at 250 nodes) plus the
        # FP64 sum's own rounding (~1e-8 here)
        assert abs(ab[d] - aa[d]) <= 250 * 2.0 ** -26 + 1e-7, (d, ab[d], aa[d])


def test_per_step_calls_with_reused_arrays(lbib, tmp_path):
    """The per-step loop of a coupled driver (source rates in, areas out),
    with the same host arrays rewritten in place every step, gives the state
    and the areas of the same loop with fresh arrays each step."""
    paths = _tissue(tmp_path)
    a = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    b = lbib.Simulation(paths, lbib.FP32_SHIFTED)
    nd = a.domain_count()
    cap = a.sizes()["cells"] + 8
    src = np.zeros((1, nd))
    dom, area = np.zeros(cap, np.uint32), np.zeros(cap)
    rng = np.random.default_rng(3)
    for step in range(12):
        r = rng.uniform(0.0, 2e-3, (1, nd))
        src[...] = r
        a.set_species_sources(src)
        a.step(1)
        n = a.areas_into(dom, area)
        b.set_species_sources(r.copy())
        b.step(1)
        d2, a2 = np.zeros(cap, np.uint32), np.zeros(cap)
        n2 = b.areas_into(d2, a2)
        assert n == n2
        np.testing.assert_array_equal(dom[:n], d2[:n])
        np.testing.assert_array_equal(area[:n], a2[:n])
    la, lb = a.lattice(), b.lattice()
    np.testing.assert_array_equal(la.g, lb.g)
    np.testing.assert_array_equal(la.f, lb.f)
    # a smaller output array after the cached one: only its length is filled
    small_d, small_a = np.zeros(3, np.uint32), np.zeros(3)
    a.step(1)
    assert a.areas_into(small_d, small_a) == n
    with pytest.raises(ValueError):
        a.areas_into(np.zeros(cap, np.int64), area)
    a.close()
    b.close()
