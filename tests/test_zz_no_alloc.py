"""lbib_areas_static — the cell areas computed into a fixed device array, with
no allocation — against lbib_areas on the same handle, called through the C
ABI.  Collected last, so it runs both alone and after every other test."""
import ctypes

import numpy as np
import pytest

from lbibcell_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from lbibcell_b200 import _lib, build
    build.build()
    return _lib.load()


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _create(lib, paths, precision):
    h = ctypes.c_void_p()
    rc = lib.lbib_create_from_files(paths["parameters"].encode(), paths["geometry"].encode(),
                                    paths["force"].encode(), paths["plugins"].encode(), precision, 0,
                                    ctypes.byref(h))
    assert rc == 0, rc
    return h


def _areas(fn, h, cap):
    dom = np.full(cap, 0xFFFFFFFF, np.uint32)
    area = np.full(cap, np.nan)
    n = fn(h, _p(dom), _p(area), cap)
    assert n >= 0, n
    return n, dom[:n].copy(), area[:n].copy()


def _tissue(tmp_path):
    cells = configs.hex_tissue(320, 320, 44.0, 20.0, 2.0, 250, 0, cols=5, rows=5)
    cfg = configs.Config(name="hex25", nx=320, ny=320, tau_fluid=1.0, iterations=40, report_step=20, cells=cells,
                         species=[configs.Species(configs.SPECIES_NAMES[0], 0.8, source={1: 1e-3})])
    return cfg.write(str(tmp_path))


@pytest.mark.parametrize("precision", [0, 1])
def test_areas_static_matches_areas(lib, tmp_path, precision):
    paths = _tissue(tmp_path)
    h = _create(lib, paths, precision)
    try:
        for steps in (0, 7, 13):
            if steps:
                assert lib.lbib_step(h, steps) == 0
            n, dom, area = _areas(lib.lbib_areas, h, 64)
            assert n == 25
            # two calls in a row: the shared array is rewritten by each call
            for _ in range(2):
                n2, dom2, area2 = _areas(lib.lbib_areas_static, h, 64)
                assert n2 == n
                np.testing.assert_array_equal(dom2, dom)
                # same kernel, same summation order: equal to the last bit
                np.testing.assert_allclose(area2, area, rtol=0, atol=0)
            assert np.all(area > 100.0)
        # a short output buffer gets the first cells, the count stays the total
        n3, dom3, area3 = _areas(lib.lbib_areas_static, h, 3)
        assert n3 == 25
        dom_full = np.zeros(3, np.uint32)
        area_full = np.zeros(3)
        assert lib.lbib_areas_static(h, _p(dom_full), _p(area_full), 3) == 25
        np.testing.assert_array_equal(dom_full, dom[:3])
        np.testing.assert_array_equal(area_full, area[:3])
    finally:
        assert lib.lbib_destroy(h) == 0


def test_areas_static_two_handles_in_turn(lib, tmp_path):
    """Two simulations on one device share the array; called one after the
    other each gets its own cells."""
    a = _create(lib, _tissue(str(tmp_path / "a")), 0)
    b = _create(lib, configs.config1(iterations=20).write(str(tmp_path / "b")), 0)
    try:
        assert lib.lbib_step(a, 5) == 0 and lib.lbib_step(b, 5) == 0
        for _ in range(2):
            na, da, aa = _areas(lib.lbib_areas_static, a, 64)
            nb, db, ab = _areas(lib.lbib_areas_static, b, 64)
            ra = _areas(lib.lbib_areas, a, 64)
            rb = _areas(lib.lbib_areas, b, 64)
            assert (na, nb) == (ra[0], rb[0]) == (25, 1)
            np.testing.assert_array_equal(da, ra[1])
            np.testing.assert_array_equal(db, rb[1])
            np.testing.assert_allclose(aa, ra[2], rtol=0, atol=0)
            np.testing.assert_allclose(ab, rb[2], rtol=0, atol=0)
    finally:
        assert lib.lbib_destroy(a) == 0
        assert lib.lbib_destroy(b) == 0


def test_areas_static_rejections_keep_the_handle(lib, tmp_path):
    """Missing output buffers are refused with LBIB_ERR_INPUT, and the same
    handle still gives lbib_areas' values afterwards."""
    h = _create(lib, _tissue(tmp_path), 0)
    try:
        assert lib.lbib_step(h, 3) == 0
        assert lib.lbib_areas_static(h, None, None, 5) == -90  # LBIB_ERR_INPUT
        ref = _areas(lib.lbib_areas, h, 64)
        got = _areas(lib.lbib_areas_static, h, 64)
        assert got[0] == ref[0] == 25
        np.testing.assert_array_equal(got[1], ref[1])
        np.testing.assert_array_equal(got[2], ref[2])
        assert lib.lbib_step(h, 2) == 0
    finally:
        assert lib.lbib_destroy(h) == 0


def test_areas_static_ring_too_long(lib, tmp_path):
    """A cell whose ring holds more nodes than the area kernel sums in one
    block (4096) is reported as a capacity error, with the index of the cell,
    and the caller's buffer holds no value of an earlier call."""
    cfg = configs.Config(name="big_ring", nx=720, ny=720, tau_fluid=1.0, iterations=10, report_step=10,
                         cells=[(1, configs.circle(360.0, 360.0, 330.0, 4200, phase=0.1))],
                         species=[], area=None, tension=None)
    small = _create(lib, _tissue(str(tmp_path / "small")), 0)
    big = _create(lib, cfg.write(str(tmp_path / "big")), 0)
    try:
        _areas(lib.lbib_areas_static, small, 64)  # leaves 25 areas in the shared array
        dom = np.zeros(4, np.uint32)
        area = np.full(4, 7.0)
        assert lib.lbib_areas_static(big, _p(dom), _p(area), 4) == -70  # LBIB_ERR_CAPACITY
        assert not np.any(area[:1] > 100.0)  # no stale area of the other handle
        buf = ctypes.create_string_buffer(256)
        idx = ctypes.c_longlong(-1)
        lib.lbib_last_error(big, buf, 256, ctypes.byref(idx))
        assert b"ring" in buf.value and idx.value == 0
        assert lib.lbib_areas(big, _p(dom), _p(area), 4) == -70
        # the other handle is unaffected
        n, _, a = _areas(lib.lbib_areas_static, small, 64)
        assert n == 25 and np.all(a > 100.0)
    finally:
        assert lib.lbib_destroy(big) == 0
        assert lib.lbib_destroy(small) == 0
