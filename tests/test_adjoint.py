"""Differentiated lattice runs (lbib_diff_*): the hand-written adjoint against
central finite differences of the FP64 forward and of the oracle (the CPU
restatement of the reference's lattice step), checkpoint-interval
invariance, and the torch.autograd.Function wrapper of the test harness.

Tolerance: adjoint vs central difference within 1e-4 relative (plus a floor of
1e-7 of the gradient's scale for components that are nearly zero)."""
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


def _cfg(n=64, species=2, tau_fluid=0.9, rates=None):
    cfg = configs.toy(n=n, r=10.0, nodes=100, iterations=100, species=species, tau_fluid=tau_fluid)
    cfg.area = None  # no mass source: the lattice step then matches the oracle's
    if rates is not None:
        for k, sp in enumerate(cfg.species):
            sp.source = {d: float(rates[k, d]) for d in range(rates.shape[1])}
    return cfg


def _close(adj, fd, scale, what):
    err = abs(adj - fd)
    assert err <= RTOL * abs(fd) + 1e-7 * scale, f"{what}: adjoint {adj:.10e} vs central difference {fd:.10e}"


class _Problem:
    """A differentiated run with parameters p = (forces, tau, rates) and the
    loss L = sum(w * C) of the final concentrations."""

    def __init__(self, runner, paths, T, K, seed=0, steps_before=0):
        self.sim = runner.Simulation(paths, runner.FP64)
        if steps_before:
            self.sim.step(steps_before)
        z = self.sim.sizes()
        self.S, self.M, self.L = z["S"], z["M"], z["nx"] * z["ny"]
        self.nD = self.sim.domain_count()
        rng = np.random.default_rng(seed)
        self.F = rng.normal(0.0, 2e-3, (self.M, 2))
        self.tau = np.array([0.9, 1.1, 0.8][: 1 + self.S])
        self.rates = rng.uniform(0.5e-3, 2e-3, (self.S, self.nD))
        self.w = rng.normal(size=(self.S, self.L))
        self.sim.diff_begin(T, K)

    def loss(self, F=None, tau=None, rates=None):
        self.sim.diff_forward(self.F if F is None else F, self.tau if tau is None else tau,
                              self.rates if rates is None else rates)
        return float((self.sim.concentrations() * self.w).sum())

    def grads(self):
        self.loss()
        return self.sim.diff_backward(self.w)


def test_adjoint_vs_central_differences_fp64(lbib, tmp_path):
    """Two species with linear sources and decay, box outlet, a membrane that
    has moved for 3 full steps; T=24 with a checkpoint every 5 steps (last
    segment partial)."""
    paths = _cfg().write(str(tmp_path))
    P = _Problem(lbib, paths, T=24, K=5, steps_before=3)
    g = P.grads()
    # relaxation times
    for i in range(1 + P.S):
        h = 1e-5
        tp, tm = P.tau.copy(), P.tau.copy()
        tp[i] += h
        tm[i] -= h
        fd = (P.loss(tau=tp) - P.loss(tau=tm)) / (2 * h)
        _close(g["tau"][i], fd, np.abs(g["tau"]).max(), f"dL/dtau[{i}]")
    # source rates of the exterior (0) and the cell (1), both species
    for k in range(P.S):
        for d in (0, 1):
            h = 1e-5
            rp, rm = P.rates.copy(), P.rates.copy()
            rp[k, d] += h
            rm[k, d] -= h
            fd = (P.loss(rates=rp) - P.loss(rates=rm)) / (2 * h)
            _close(g["rates"][k, d], fd, np.abs(g["rates"]).max(), f"dL/drate[{k},{d}]")
    # membrane node forces: single components and one random direction
    scaleF = np.abs(g["force"]).max()
    assert scaleF > 0
    for i, c in ((0, 0), (P.M // 3, 1), (int(np.argmax(np.abs(g["force"][:, 0]))), 0)):
        h = 1e-5
        Fp, Fm = P.F.copy(), P.F.copy()
        Fp[i, c] += h
        Fm[i, c] -= h
        fd = (P.loss(F=Fp) - P.loss(F=Fm)) / (2 * h)
        _close(g["force"][i, c], fd, scaleF, f"dL/dF[{i},{c}]")
    v = np.random.default_rng(7).normal(size=P.F.shape)
    h = 1e-5
    fd = (P.loss(F=P.F + h * v) - P.loss(F=P.F - h * v)) / (2 * h)
    _close(float((g["force"] * v).sum()), fd, np.abs(g["force"] * v).sum(), "dL/dF . v")
    P.sim.diff_end()


def test_adjoint_vs_central_differences_oracle(lbib, oracle_mod, tmp_path):
    """The differentiated forward is the oracle's lattice step bit for bit, and
    the adjoint matches central differences taken through the oracle."""
    T = 16
    base = _cfg()
    paths = base.write(str(tmp_path / "base"))
    P = _Problem(lbib, paths, T=T, K=4)
    lat0 = P.sim.lattice()
    g = P.grads()
    C_gpu = P.sim.concentrations()
    force = P.sim.lattice().force

    def oracle_loss(tau, rates, tag):
        cfg = _cfg(tau_fluid=float(tau[0]), rates=rates)
        for k, sp in enumerate(cfg.species):
            sp.tau = float(tau[1 + k])
        o = oracle_mod.Oracle(cfg.write(str(tmp_path / tag)))
        o.set_lattice(lat0.f, lat0.g, force)
        o.lattice_step(T, outlet=True)
        C = o.state().g.sum(axis=2)
        return C, float((C * P.w).sum())

    C_cpu, _ = oracle_loss(P.tau, P.rates, "same")
    np.testing.assert_array_equal(C_cpu, C_gpu)
    h = 1e-5
    for i in range(1 + P.S):
        tp, tm = P.tau.copy(), P.tau.copy()
        tp[i] += h
        tm[i] -= h
        fd = (oracle_loss(tp, P.rates, f"tp{i}")[1] - oracle_loss(tm, P.rates, f"tm{i}")[1]) / (2 * h)
        _close(g["tau"][i], fd, np.abs(g["tau"]).max(), f"oracle dL/dtau[{i}]")
    for k in range(P.S):
        rp, rm = P.rates.copy(), P.rates.copy()
        rp[k, 1] += h
        rm[k, 1] -= h
        fd = (oracle_loss(P.tau, rp, f"rp{k}")[1] - oracle_loss(P.tau, rm, f"rm{k}")[1]) / (2 * h)
        _close(g["rates"][k, 1], fd, np.abs(g["rates"]).max(), f"oracle dL/drate[{k},1]")
    P.sim.diff_end()


def test_checkpoint_interval_and_restore(lbib, tmp_path):
    """Gradients do not depend on the checkpoint interval; lbib_diff_end puts
    the snapshot back."""
    paths = _cfg(species=1).write(str(tmp_path))
    ref = None
    for K in (1, 4, 0, 13):
        P = _Problem(lbib, paths, T=13, K=K, steps_before=2)
        before = P.sim.lattice()
        g = P.grads()
        if ref is None:
            ref = g
        else:
            np.testing.assert_array_equal(g["force"], ref["force"])
            np.testing.assert_allclose(g["tau"], ref["tau"], rtol=1e-12)
            np.testing.assert_allclose(g["rates"], ref["rates"], rtol=1e-12, atol=1e-300)
        P.sim.diff_end()
        after = P.sim.lattice()
        for name in ("f", "g", "vel", "force", "dom"):
            np.testing.assert_array_equal(getattr(after, name), getattr(before, name), err_msg=name)
        P.sim.close()


def test_fp32_differentiated_run_matches_fp64(lbib, tmp_path):
    """An FP32-shifted handle's differentiated run (FP32 forward and states,
    FP64 reverse arithmetic and gradient sums) against the FP64 run of the same
    problem: the final concentrations within 1e-5 of their scale, every
    gradient group within 1e-3 relative of the FP64 adjoint (the two forward
    trajectories differ at the FP32 rounding level)."""
    paths = _cfg().write(str(tmp_path))
    g, C = {}, {}
    for prec in (lbib.FP64, lbib.FP32_SHIFTED):
        P = _Problem(lbib, paths, T=24, K=5, steps_before=3)
        P.sim.close()
        P.sim = lbib.Simulation(paths, prec)
        P.sim.step(3)
        P.sim.diff_begin(24, 5)
        g[prec] = P.grads()
        C[prec] = P.sim.concentrations()
        P.sim.diff_end()
    a64, a32 = lbib.FP64, lbib.FP32_SHIFTED
    assert np.abs(C[a64] - C[a32]).max() <= 1e-5 * np.abs(C[a64]).max()
    for k in ("tau", "rates", "force"):
        a, b = g[a64][k], g[a32][k]
        assert np.abs(a - b).max() <= 1e-3 * np.abs(a).max(), (k, np.abs(a - b).max(), np.abs(a).max())


def test_diff_rejects_call_order(lbib, tmp_path):
    paths = _cfg(species=1).write(str(tmp_path))
    s64 = lbib.Simulation(paths, lbib.FP64)
    s64.diff_begin(4)
    with pytest.raises(lbib.LbibError) as e:
        s64.diff_backward(np.zeros((1, 64 * 64)))
    assert e.value.code == 91


def test_autograd_function_wrapper(lbib, tmp_path):
    """The torch.autograd.Function of the harness: a nonlinear loss of the
    concentrations, gradients for all three parameter groups at once, checked
    along a random direction by a central difference."""
    import torch

    paths = _cfg().write(str(tmp_path))
    P = _Problem(lbib, paths, T=20, K=6, steps_before=2)
    sim = P.sim

    class LatticeRun(torch.autograd.Function):
        @staticmethod
        def forward(ctx, forces, tau, rates):
            sim.diff_forward(forces.detach().numpy(), tau.detach().numpy(), rates.detach().numpy())
            return torch.from_numpy(sim.concentrations())

        @staticmethod
        def backward(ctx, gC):
            g = sim.diff_backward(gC.detach().numpy())
            return torch.from_numpy(g["force"]), torch.from_numpy(g["tau"]), torch.from_numpy(g["rates"])

    w = torch.from_numpy(P.w)

    def loss_of(F, tau, rates):
        C = LatticeRun.apply(F, tau, rates)
        return (w * C).sum() + 50.0 * (C * C).sum()

    F = torch.tensor(P.F, requires_grad=True)
    tau = torch.tensor(P.tau, requires_grad=True)
    rates = torch.tensor(P.rates, requires_grad=True)
    loss = loss_of(F, tau, rates)
    loss.backward()
    rng = np.random.default_rng(3)
    vF = torch.from_numpy(rng.normal(size=P.F.shape) * 1e-3)
    vT = torch.from_numpy(rng.normal(size=P.tau.shape) * 1e-2)
    vR = torch.from_numpy(rng.normal(size=P.rates.shape) * 1e-4)
    directional = float((F.grad * vF).sum() + (tau.grad * vT).sum() + (rates.grad * vR).sum())
    h = 1e-3
    with torch.no_grad():
        lp = float(loss_of(F + h * vF, tau + h * vT, rates + h * vR))
        lm = float(loss_of(F - h * vF, tau - h * vT, rates - h * vR))
    fd = (lp - lm) / (2 * h)
    _close(directional, fd, abs(fd), "autograd directional derivative")
    sim.diff_end()


@pytest.mark.parametrize("nx", [520, 63])
def test_adjoint_row_blocks(lbib, tmp_path, nx):
    """Lattice widths that exercise every kind of row block of the adjoint
    step: 520 = two full blocks of 256 nodes (one of them away from the
    periodic x boundary) and a partial block of 8; 63 (odd) takes the
    direct-load kernel."""
    ny = 40
    sp = [configs.Species(configs.SPECIES_NAMES[k], t, decay=1e-4 * k, source={1: 1e-3})
          for k, t in enumerate((1.0, 0.8))]
    cfg = configs.Config(name=f"wide_{nx}", nx=nx, ny=ny, tau_fluid=0.9, iterations=100, report_step=50,
                         cells=[(1, configs.circle(nx / 2.0 + 0.3, ny / 2.0 + 0.2, 9.0, 90))], species=sp,
                         area=None)
    P = _Problem(lbib, cfg.write(str(tmp_path)), T=12, K=5, steps_before=2)
    g = P.grads()
    h = 1e-5
    for i in range(1 + P.S):
        tp, tm = P.tau.copy(), P.tau.copy()
        tp[i] += h
        tm[i] -= h
        fd = (P.loss(tau=tp) - P.loss(tau=tm)) / (2 * h)
        _close(g["tau"][i], fd, np.abs(g["tau"]).max(), f"dL/dtau[{i}]")
    rp, rm = P.rates.copy(), P.rates.copy()
    rp[1, 1] += h
    rm[1, 1] -= h
    fd = (P.loss(rates=rp) - P.loss(rates=rm)) / (2 * h)
    _close(g["rates"][1, 1], fd, np.abs(g["rates"]).max(), "dL/drate[1,1]")
    v = np.random.default_rng(11).normal(size=P.F.shape)
    fd = (P.loss(F=P.F + h * v) - P.loss(F=P.F - h * v)) / (2 * h)
    _close(float((g["force"] * v).sum()), fd, np.abs(g["force"] * v).sum(), "dL/dF . v")
    P.sim.diff_end()


def test_config4_adjoint_vs_central_differences(lbib, tmp_path):
    """The adjoint workload as specified: 512x512, 50 cells, one species
    (tau 0.8), T = 2000 with a checkpoint every 100 steps; loss
    L = sum_x (C(T) - c_target)^2 with c_target from a forward run whose 50
    per-cell source rates are perturbed by N(0, 0.1) relative; central
    differences of the FP64 forward with step h = 1e-6.  Every gradient entry
    of magnitude >= 1e-3 of the largest entry of its kind must match to 1e-4
    relative, with no floor; smaller entries to 1e-4 of that magnitude."""
    cfg = configs.config4()
    paths = cfg.write(str(tmp_path))
    sim = lbib.Simulation(paths, lbib.FP64)
    sim.step(3)
    nD = sim.domain_count()
    T, K, h = 2000, 100, 1e-6
    rates = np.zeros((1, nD))
    for d, r in cfg.species[0].source.items():
        rates[0, d] = r
    tau = np.array([cfg.tau_fluid, cfg.species[0].tau])
    # the membrane forces of the last force evaluation (the run's default)
    forces = np.ascontiguousarray(sim.membrane()[1][:, 4:6])
    sim.diff_begin(T, K)
    target_rates = rates * (1.0 + np.random.default_rng(4).normal(0.0, 0.1, rates.shape))
    sim.diff_forward(forces, tau, target_rates)
    c_target = sim.concentrations().copy()

    def loss(F=None, tau_=None, rates_=None):
        # every parameter passed: a call's parameters stay in effect for the next
        sim.diff_forward(forces if F is None else F, tau if tau_ is None else tau_,
                         rates if rates_ is None else rates_)
        C = sim.concentrations()
        return float(((C - c_target) ** 2).sum()), C

    L0, C0 = loss()
    g = sim.diff_backward(2.0 * (C0 - c_target))

    def check(adj, fd, mag, what):
        if abs(fd) >= mag:
            assert abs(adj - fd) <= RTOL * abs(fd), f"{what}: adjoint {adj:.10e} vs central difference {fd:.10e}"
        else:
            assert abs(adj - fd) <= RTOL * mag, f"{what}: adjoint {adj:.10e} vs central difference {fd:.10e}"

    # all 50 per-cell source rates (domains 1..50)
    magR = 1e-3 * np.abs(g["rates"][0, 1:]).max()
    assert magR > 0
    for d in range(1, nD):
        rp, rm = rates.copy(), rates.copy()
        rp[0, d] += h
        rm[0, d] -= h
        fd = (loss(rates_=rp)[0] - loss(rates_=rm)[0]) / (2 * h)
        check(g["rates"][0, d], fd, magR, f"dL/drate[{d}]")
    # the species' and the fluid's relaxation times
    for i in range(2):
        tp, tm = tau.copy(), tau.copy()
        tp[i] += h
        tm[i] -= h
        fd = (loss(tau_=tp)[0] - loss(tau_=tm)[0]) / (2 * h)
        check(g["tau"][i], fd, 1e-3 * np.abs(g["tau"]).max(), f"dL/dtau[{i}]")
    # membrane node forces (the tension of the last force evaluation): the
    # largest entries and a random direction in force space
    magF = 1e-3 * np.abs(g["force"]).max()
    assert magF > 0
    order = np.argsort(-np.abs(g["force"]).ravel())[:4]
    for flat in order:
        i, c = divmod(int(flat), 2)
        Fp, Fm = forces.copy(), forces.copy()
        Fp[i, c] += h
        Fm[i, c] -= h
        fd = (loss(F=Fp)[0] - loss(F=Fm)[0]) / (2 * h)
        check(g["force"][i, c], fd, magF, f"dL/dF[{i},{c}]")
    v = np.random.default_rng(9).normal(size=forces.shape)
    fd = (loss(F=forces + h * v)[0] - loss(F=forces - h * v)[0]) / (2 * h)
    check(float((g["force"] * v).sum()), fd, 0.0, "dL/dF . v")
    sim.diff_end()


# lattice() slot d holds the population of direction INV9[d] (after localSwap)
_INV9 = np.array([0, 3, 4, 1, 2, 7, 8, 5, 6])
_CX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])[_INV9]
_CY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])[_INV9]


def _kinetic(f, window):
    """Kinetic energy 1/2 |j|^2 / rho of the stored distributions over the
    nodes in `window`, and its gradient with respect to f (lattice() layout)."""
    rho = f.sum(1)
    jx, jy = f @ _CX, f @ _CY
    e = 0.5 * (jx * jx + jy * jy) / rho
    grad = (np.outer(jx, _CX) + np.outer(jy, _CY)) / rho[:, None] - (e / rho)[:, None]
    return float(e[window].sum()), grad * window[:, None]


def test_mass_source_and_flow_loss_gradients(lbib, tmp_path):
    """The per-domain mass source (rhoToAdd, lbib_diff_mass) and a loss of the
    flow (the kinetic energy in a central window, seeded through
    lbib_diff_fluid_seed) plus a concentration term: the adjoint against
    central differences of the FP64 forward, 1e-4 relative."""
    paths = _cfg(n=64).write(str(tmp_path))
    P = _Problem(lbib, paths, T=24, K=5, steps_before=3)
    n = 64
    yy, xx = np.divmod(np.arange(n * n), n)
    window = (abs(xx - 32) < 12) & (abs(yy - 32) < 12)
    mass = np.zeros(P.nD)
    mass[1] = 2e-3
    P.sim.diff_mass(mass)

    def loss(F=None, tau=None, rates=None, m=None):
        P.sim.diff_mass(mass if m is None else m)
        P.sim.diff_forward(P.F if F is None else F, P.tau if tau is None else tau,
                           P.rates if rates is None else rates)
        lat = P.sim.lattice()
        ke, dke = _kinetic(lat.f, window)
        return ke + float((P.sim.concentrations() * P.w).sum()), dke

    L0, dke = loss()
    P.sim.diff_fluid_seed(dke)
    g = P.sim.diff_backward(P.w)
    gm = P.sim.diff_mass()
    h = 1e-6
    for d in (0, 1):
        mp, mm = mass.copy(), mass.copy()
        mp[d] += h
        mm[d] -= h
        fd = (loss(m=mp)[0] - loss(m=mm)[0]) / (2 * h)
        _close(gm[d], fd, np.abs(gm).max(), f"dL/dmass[{d}]")
    for i in range(1 + P.S):
        tp, tm = P.tau.copy(), P.tau.copy()
        tp[i] += 1e-5
        tm[i] -= 1e-5
        fd = (loss(tau=tp)[0] - loss(tau=tm)[0]) / 2e-5
        _close(g["tau"][i], fd, np.abs(g["tau"]).max(), f"dL/dtau[{i}]")
    v = np.random.default_rng(3).normal(size=P.F.shape)
    fd = (loss(F=P.F + 1e-5 * v)[0] - loss(F=P.F - 1e-5 * v)[0]) / 2e-5
    _close(float((g["force"] * v).sum()), fd, np.abs(g["force"] * v).sum(), "dL/dF . v")
    P.sim.diff_fluid_seed(None)
    P.sim.diff_end()


def _node_forces(ids, xy, rec):
    """ForceSolver::calculateForce restated for the test (ForceStructs.hpp
    49-588): each record adds to its own node's force."""
    index = {int(i): k for k, i in enumerate(ids)}
    F = np.zeros((len(ids), 2))
    for t, a, b, p in zip(rec["type"], rec["id1"], rec["id2"], rec["par"]):
        i = index[int(a)]
        x1, y1 = xy[i]
        if t in (0, 7, 5, 6):
            dx, dy = xy[index[int(b)]] - xy[i]
            dist = np.sqrt(dx * dx + dy * dy)
            f = p[0] * (dist - p[1]) if t in (0, 7) else p[0]
            F[i] += (dx * f / dist, dy * f / dist)
        elif t == 1:
            dx, dy = p[0] - x1, p[1] - y1
            dist = np.sqrt(dx * dx + dy * dy)
            if dist != 0.0:
                f = p[2] * (dist - p[3])
                F[i] += (dx * f / dist, dy * f / dist)
        elif t == 2:
            F[i] += p[:2]
        elif t == 3:
            f = p[1] * (abs(p[0] - y1) - p[2])
            F[i, 1] += f if y1 < p[0] else -f
        elif t == 4:
            f = p[1] * (abs(p[0] - x1) - p[2])
            F[i, 0] += f if x1 < p[0] else -f
    return F


def test_force_record_parameter_gradients(lbib, tmp_path):
    """The a11 chain rule: dL/d of force-record parameters (lbib_diff_force_params)
    equals dL/dF . dF/dp of a numpy restatement of the force types (all eight),
    and central differences of the whole run in the parameter (the node forces
    re-formed from the perturbed records and passed as the run's forces)."""
    cfg = _cfg()
    cfg.tension = (0.05, 10)  # LbibMembraneTension: type-6 records on every node
    paths = cfg.write(str(tmp_path))
    P = _Problem(lbib, paths, T=20, K=5, steps_before=2)
    sim = P.sim
    ids, node = sim.membrane()
    xy = node[:, :2].copy()
    n = len(ids)
    # one record of each other type on a few nodes (partners two nodes on)
    extra = [(0, 0, 2, (0.02, 1.5, 0, 0)), (7, 5, 9, (0.01, 3.0, 0, 0)),
             (1, 11, 0, (xy[11, 0] + 3.0, xy[11, 1] - 2.0, 0.02, 1.0)), (2, 17, 0, (1e-3, -2e-3, 0, 0)),
             (3, 23, 0, (xy[23, 1] + 4.0, 0.02, 1.0, 0)), (4, 29, 0, (xy[29, 0] - 3.0, 0.015, 0.5, 0)),
             (5, 31, 33, (2e-3, 0, 0, 0))]
    sim.add_forces([e[0] for e in extra], [ids[e[1] % n] for e in extra], [ids[e[2] % n] for e in extra],
                   np.array([e[3] for e in extra], float))
    rec = sim.forces()
    assert set(rec["type"].tolist()) == set(range(8))
    F0 = _node_forces(ids, xy, rec)

    def loss(par):
        r = dict(rec, par=par)
        return P.loss(F=_node_forces(ids, xy, r))

    L0 = loss(rec["par"])
    g = sim.diff_backward(P.w)
    gp = sim.diff_force_params()
    assert gp.shape == (len(rec["type"]), 4)
    # the chain rule against a numpy differentiation of the restated forces
    index = {int(i): k for k, i in enumerate(ids)}
    for r in range(len(rec["type"])):
        i = index[int(rec["id1"][r])]
        for q in range(4):
            h = 1e-6 * max(1.0, abs(rec["par"][r, q]))
            pp, pm = rec["par"].copy(), rec["par"].copy()
            pp[r, q] += h
            pm[r, q] -= h
            dF = (_node_forces(ids, xy, dict(rec, par=pp))[i] - _node_forces(ids, xy, dict(rec, par=pm))[i]) / (2 * h)
            want = float(g["force"][i] @ dF)
            assert abs(gp[r, q] - want) <= 1e-6 * abs(want) + 1e-12 * np.abs(gp).max(), (r, q, gp[r, q], want)
    # central differences of the run in one parameter of each type
    assert np.abs(F0 - _node_forces(ids, xy, rec)).max() == 0.0
    checked = 0
    for t, q in ((6, 0), (0, 0), (0, 1), (7, 1), (1, 0), (1, 2), (2, 1), (3, 0), (3, 1), (4, 2), (5, 0)):
        r = int(np.nonzero(rec["type"] == t)[0][0])
        h = 1e-6 * max(1.0, abs(rec["par"][r, q]))
        pp, pm = rec["par"].copy(), rec["par"].copy()
        pp[r, q] += h
        pm[r, q] -= h
        fd = (loss(pp) - loss(pm)) / (2 * h)
        _close(gp[r, q], fd, np.abs(gp).max(), f"dL/dpar[type {t}, {q}]")
        checked += 1
    assert checked == 11 and np.isfinite(L0)
    sim.diff_end()


@pytest.mark.parametrize("T,K", [(13, 4), (12, 6), (15, 3), (9, 5)])
def test_overlapped_recompute_equals_serial(lbib, tmp_path, monkeypatch, T, K):
    """The reverse pass of an FP32-shifted run with two segment buffers (the
    next segment recomputed on a second stream while the current one is
    reversed) gives bit for bit
    the gradients of the one-buffer pass, on the first backward call after a
    forward (the last segment kept) and on a repeated one (every segment
    recomputed).  The per-domain rate gradients are sums by atomic adds over
    the lattice (their order varies from run to run): within 1e-12 relative."""
    paths = _cfg(species=2).write(str(tmp_path))
    out = {}
    for serial in ("1", "0"):
        monkeypatch.setenv("LBIB_DIFF_SERIAL", serial)
        P = _Problem(lbib, paths, T=T, K=K, steps_before=2)
        P.sim.close()
        P.sim = lbib.Simulation(paths, lbib.FP32_SHIFTED)  # FP32 states: the overlapped pass
        P.sim.step(2)
        P.sim.diff_begin(T, K)
        g1 = P.grads()
        g2 = P.sim.diff_backward(P.w)
        out[serial] = (g1, g2)
        P.sim.diff_end()
        P.sim.close()
    monkeypatch.delenv("LBIB_DIFF_SERIAL", raising=False)
    def same(x, y, k, what):
        if k == "rates":
            np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-300, err_msg=what)
        else:
            np.testing.assert_array_equal(x, y, err_msg=what)
    for i in range(2):
        for k in ("force", "tau", "rates"):
            same(out["0"][i][k], out["1"][i][k], k, f"call {i} {k}")
    for k in ("force", "tau", "rates"):
        same(out["0"][1][k], out["0"][0][k], k, f"repeat {k}")
