"""The CPU oracle against the reference itself (golden fixtures from
oracle/_ref, generated by tests/golden/make_golden.py)."""
import hashlib
import json
import os

import numpy as np
import pytest

from lbibcell_b200 import configs

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIELDS = ("f", "g", "vel", "force", "dom", "ctype", "ids", "node", "conn")


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_toy48_bit_exact(oracle_mod, tmp_path):
    gold = np.load(os.path.join(GOLD, "toy48.npz"))
    cfg = configs.toy(n=48, r=8.0, nodes=80, iterations=60, report_step=30, species=1)
    o = oracle_mod.Oracle(cfg.write(str(tmp_path)))
    prev = 0
    for t in (0, 30, 60):
        o.step(t - prev)
        prev = t
        st = o.state()
        assert st.current_iteration == int(gold[f"iter_{t}"])
        for k in FIELDS:
            a, b = getattr(st, k), gold[f"{k}_{t}"]
            assert a.shape == b.shape, (t, k)
            assert np.array_equal(a, b), (t, k)


def test_config1_digests(oracle_mod, tmp_path):
    """200x200 single cell, 2000 steps: every state array identical to the
    reference build's at t = 0, 500, ..., 2000."""
    dig = json.load(open(os.path.join(GOLD, "config1_digest.json")))
    o = oracle_mod.Oracle(configs.config1().write(str(tmp_path)))
    prev = 0
    for t in (0, 500, 1000, 1500, 2000):
        o.step(t - prev)
        prev = t
        st = o.state()
        want = dig[str(t)]
        assert st.ids.shape[0] == want["M"]
        assert st.current_iteration == want["iteration"]
        for k in FIELDS:
            assert _digest(getattr(st, k)) == want[k], (t, k)


def test_fastcos_bounds(oracle_mod):
    """fastCos (GeometryNode.cpp:55-81) stays within 1e-3 of cos on [-pi, pi]."""
    L = oracle_mod.lib()
    xs = np.linspace(-np.pi, np.pi, 2001)
    err = max(abs(L.orc_fastcos(float(x)) - np.cos(x)) for x in xs)
    assert err < 1.1e-3


def test_delta_partition(oracle_mod):
    """The 4x4 Dirac stencil sums to ~1 (not exactly: fastCos is approximate)."""
    L = oracle_mod.lib()
    for X, Y in ((10.3, 20.7), (5.5, 5.5), (7.01, 3.99)):
        x0, y0 = int(np.ceil(X - 2)), int(np.ceil(Y - 2))
        s = sum(L.orc_delta(x - X, y - Y) for x in range(x0, x0 + 4) for y in range(y0, y0 + 4))
        assert abs(s - 1.0) < 5e-3


def _guo48(model="GuoZhengShi2002ForceModel"):
    cfg = configs.toy(n=48, r=8.0, nodes=80, iterations=60, report_step=30, species=1)
    cfg.force_model = model
    return cfg


def test_guo48_bit_exact(oracle_mod, tmp_path):
    """The oracle's Guo force model against the reference compiled with
    GuoZhengShi2002ForceModel as FluidSolver's base class (the alternative
    FluidSolver.hpp:41 names), every state array at t = 0, 30, 60."""
    gold = np.load(os.path.join(GOLD, "guo48.npz"))
    o = oracle_mod.Oracle(_guo48().write(str(tmp_path)))
    prev = 0
    for t in (0, 30, 60):
        o.step(t - prev)
        prev = t
        st = o.state()
        for k in FIELDS:
            a, b = getattr(st, k), gold[f"{k}_{t}"]
            assert a.shape == b.shape, (t, k)
            assert np.array_equal(a, b), (t, k)
    # the force model matters here: the Luo run differs
    luo = np.load(os.path.join(GOLD, "toy48.npz"))
    assert not np.array_equal(luo["f_60"], gold["f_60"])


def test_guo_corrected_differs_only_through_ne(oracle_mod, tmp_path):
    """The corrected Guo model (+6 v_y in the NE term's F_y factor, the
    expansion of (1 - 1/2tau) w_i [3 (e_i - v) + 9 (e_i . v) e_i] . F) is a
    different run from the reference's as written, close to it: the written
    NE term differs by 9 G2 v_y F_y, second order in the small velocity."""
    a = oracle_mod.Oracle(_guo48().write(str(tmp_path / "a")))
    b = oracle_mod.Oracle(_guo48("GuoZhengShi2002ForceModelCorrected").write(str(tmp_path / "b")))
    a.step(30)
    b.step(30)
    sa, sb = a.state(), b.state()
    assert not np.array_equal(sa.f, sb.f)
    assert np.abs(sa.f - sb.f).max() < 1e-4
