"""Differentiated runs with moving membrane nodes (lbib_diff_motion): the
adjoint of the spread, the interpolation and the move with the Dirac weights'
derivative, against central differences of the same forward.

The loss joins the final concentrations and the final node positions,
L = sum(w * C) + sum(v * X_T), so the gradients with respect to the node
forces, the relaxation times, the source rates and the starting positions all
run through the motion.  Tolerance: adjoint vs central difference within 1e-4
relative (plus a floor of 1e-7 of the gradient's scale for components that
are nearly zero), as for the frozen-geometry runs."""
import numpy as np
import pytest

from lbibcell_b200 import configs

pytestmark = pytest.mark.gpu

RTOL = 1e-4


@pytest.fixture(scope="module")
def lbib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from lbibcell_b200 import build, runner
    build.build()
    return runner


def _close(adj, fd, scale, what):
    err = abs(adj - fd)
    assert err <= RTOL * abs(fd) + 1e-7 * scale, f"{what}: adjoint {adj:.10e} vs central difference {fd:.10e}"


def _paths(tmp_path):
    cfg = configs.toy(n=64, r=10.0, nodes=100, iterations=100, species=2, tau_fluid=0.9)
    cfg.area = None
    return cfg.write(str(tmp_path))


class _Moving:
    """A moving-node differentiated run from the state after `steps_before`
    full steps, with parameters (F, tau, rates) and starting positions X0."""

    def __init__(self, runner, paths, T, K, precision=None, xy=None, steps_before=3, seed=0):
        self.runner = runner
        self.sim = runner.Simulation(paths, runner.FP64 if precision is None else precision)
        self.sim.step(steps_before)
        if xy is not None:
            ids, _ = self.sim.membrane()
            self.sim.upload_membrane(ids, xy, self.sim.connections())
            self.sim.cure_lattice()
        z = self.sim.sizes()
        self.S, self.M, self.L = z["S"], z["M"], z["nx"] * z["ny"]
        self.nD = self.sim.domain_count()
        rng = np.random.default_rng(seed)
        self.F = rng.normal(0.0, 5e-3, (self.M, 2))
        self.tau = np.array([0.9, 1.1, 0.8][: 1 + self.S])
        self.rates = rng.uniform(0.5e-3, 2e-3, (self.S, self.nD))
        self.w = rng.normal(size=(self.S, self.L))
        self.v = rng.normal(size=(self.M, 2))
        self.sim.diff_begin(T, K)
        self.sim.diff_motion(True, self.v)

    def loss(self, F=None, tau=None, rates=None):
        self.sim.diff_forward(self.F if F is None else F, self.tau if tau is None else tau,
                              self.rates if rates is None else rates)
        xT = self.sim.diff_positions()
        return float((self.sim.concentrations() * self.w).sum() + (xT * self.v).sum())

    def grads(self):
        self.loss()
        g = self.sim.diff_backward(self.w)
        g["x0"] = self.sim.diff_positions(grad=True)[1]
        return g


def test_motion_adjoint_vs_central_differences(lbib, tmp_path):
    """T = 24 with a checkpoint every 5 steps (last segment partial): dL/dF
    (single components and a random direction), dL/dtau, dL/d rate."""
    paths = _paths(tmp_path)
    P = _Moving(lbib, paths, T=24, K=5)
    g = P.grads()
    ids, st = P.sim.membrane()
    xT = P.sim.diff_positions()
    moved = np.abs(xT - st[:, :2]).max()
    assert moved > 1e-3, f"the nodes hardly moved ({moved:.2e} lu)"
    h = 1e-5
    for i in range(1 + P.S):
        tp, tm = P.tau.copy(), P.tau.copy()
        tp[i] += h
        tm[i] -= h
        fd = (P.loss(tau=tp) - P.loss(tau=tm)) / (2 * h)
        _close(g["tau"][i], fd, np.abs(g["tau"]).max(), f"dL/dtau[{i}]")
    for k in range(P.S):
        for d in (0, 1):
            rp, rm = P.rates.copy(), P.rates.copy()
            rp[k, d] += h
            rm[k, d] -= h
            fd = (P.loss(rates=rp) - P.loss(rates=rm)) / (2 * h)
            _close(g["rates"][k, d], fd, np.abs(g["rates"]).max(), f"dL/drate[{k},{d}]")
    scaleF = np.abs(g["force"]).max()
    assert scaleF > 0
    for i, c in ((0, 0), (P.M // 3, 1), (int(np.argmax(np.abs(g["force"][:, 0]))), 0)):
        Fp, Fm = P.F.copy(), P.F.copy()
        Fp[i, c] += h
        Fm[i, c] -= h
        fd = (P.loss(F=Fp) - P.loss(F=Fm)) / (2 * h)
        _close(g["force"][i, c], fd, scaleF, f"dL/dF[{i},{c}]")
    u = np.random.default_rng(7).normal(size=P.F.shape)
    fd = (P.loss(F=P.F + h * u) - P.loss(F=P.F - h * u)) / (2 * h)
    _close(float((g["force"] * u).sum()), fd, np.abs(g["force"] * u).sum(), "dL/dF . u")
    P.sim.diff_end()


def test_motion_adjoint_starting_positions(lbib, tmp_path):
    """dL/dX0 against central differences of runs whose starting positions
    are shifted (uploaded before lbib_diff_begin): one component and a
    random direction over every node."""
    paths = _paths(tmp_path)
    P = _Moving(lbib, paths, T=16, K=4)
    g = P.grads()
    L0 = P.loss()
    _, st = P.sim.membrane()
    X0 = st[:, :2].copy()
    P.sim.diff_end()
    h = 1e-5

    def loss_at(xy):
        Q = _Moving(lbib, paths, T=16, K=4, xy=xy)
        v = Q.loss(F=P.F, tau=P.tau, rates=P.rates)
        Q.sim.diff_end()
        return v

    # uploading the unchanged positions leaves the run as it was
    assert abs(loss_at(X0) - L0) <= 1e-9 * abs(L0)
    i = int(np.argmax(np.abs(g["x0"][:, 1])))
    Xp, Xm = X0.copy(), X0.copy()
    Xp[i, 1] += h
    Xm[i, 1] -= h
    fd = (loss_at(Xp) - loss_at(Xm)) / (2 * h)
    _close(g["x0"][i, 1], fd, np.abs(g["x0"]).max(), f"dL/dX0[{i},1]")
    u = np.random.default_rng(11).normal(size=X0.shape)
    fd = (loss_at(X0 + h * u) - loss_at(X0 - h * u)) / (2 * h)
    _close(float((g["x0"] * u).sum()), fd, np.abs(g["x0"] * u).sum(), "dL/dX0 . u")


def test_motion_fp32_shifted_close_to_fp64(lbib, tmp_path):
    """The same run on an FP32-shifted handle (FP32 forward and checkpoints,
    FP64 reverse arithmetic): gradients within 1e-3 of the FP64 run's."""
    paths = _paths(tmp_path)
    a = _Moving(lbib, paths, T=24, K=5)
    b = _Moving(lbib, paths, T=24, K=5, precision=lbib.FP32_SHIFTED)
    ga, gb = a.grads(), b.grads()
    for key in ("force", "tau", "rates", "x0"):
        scale = np.abs(ga[key]).max()
        assert np.abs(ga[key] - gb[key]).max() <= 1e-3 * scale, key
    a.sim.diff_end()
    b.sim.diff_end()


def test_motion_off_is_the_frozen_run(lbib, tmp_path):
    """Switched on and off again, a run is the frozen-geometry run bit for bit."""
    paths = _paths(tmp_path)
    P = _Moving(lbib, paths, T=12, K=4)
    P.loss()
    P.sim.diff_motion(False)
    P.sim.diff_forward(P.F, P.tau, P.rates)
    C = P.sim.concentrations()
    Q = lbib.Simulation(paths, lbib.FP64)
    Q.step(3)
    Q.diff_begin(12, 4)
    Q.diff_forward(P.F, P.tau, P.rates)
    np.testing.assert_array_equal(C, Q.concentrations())
    P.sim.diff_end()
    Q.diff_end()
