"""The force-list and range-query calls a host bio solver makes between steps
(ForceSolver::addForce / deleteForceType / deleteAllForces, ForceSolver.cpp:
107-139,170-215; Geometry::getGeometryNodesWithinRadius[WithAvoidance]
[Closest], Geometry.cpp:306-374), in bulk through the C ABI.

Added records are checked against the reference build restarted from a force
file that holds the same records as text; the queries against a restatement
of the reference's cell list (FastNeighborList.hpp) over the downloaded
membrane."""
import math
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


def _cfg(iterations):
    cfg = configs.toy(n=48, r=8.0, nodes=80, iterations=iterations, report_step=10, species=2)
    cfg.area = None  # the area regulator's targets are plugin state that no file holds
    return cfg


def _at_iteration(dumps, it):
    for k, st in dumps.items():
        if k != "stdout" and st.current_iteration == it:
            return st
    raise AssertionError(f"no reference dump at iteration {it}")


def _extra_records(ids):
    """A spring, an anchor, a constant force and a slider, as text lines and as
    arrays (parameters with <= 6 significant digits: the text is exact)."""
    a, b, c = int(ids[0]), int(ids[7]), int(ids[15])
    lines = [f"0\t{a}\t{b}\t0.002\t3.5", f"1\t{c}\t20.25\t30.5\t0.001\t1.5", f"2\t{b}\t0.0001\t-0.0002",
             f"3\t{a}\t22.5\t0.0005\t0.75"]
    types = [0, 1, 2, 3]
    id1 = [a, c, b, a]
    id2 = [b, 0, 0, 0]
    par = [[0.002, 3.5, 0, 0], [20.25, 30.5, 0.001, 1.5], [0.0001, -0.0002, 0, 0], [22.5, 0.0005, 0.75, 0]]
    return lines, (types, id1, id2, par)


def _by_node(path):
    """Force records grouped by their node in file order (ForceSolver's
    forcemap_ is keyed by node id, each list in insertion order)."""
    recs = []
    for line in open(path):
        v = line.split()
        if not v or v[0].startswith("#"):
            continue
        recs.append((int(v[1]), int(v[0]), tuple(round(float(t), 9) for t in v[2:])))
    return sorted(recs, key=lambda r: r[0])  # stable: file order within a node


def test_added_forces_match_reference(lbib, oracle_mod, tmp_path):
    """Written at iteration 23; the reference restarts from a force file with
    four more records appended, this library restarts from the plain files and
    adds the same records through lbib_add_forces; both run to iteration 43
    (the records act until the clearing at iteration 30)."""
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    paths = _cfg(43).write(str(tmp_path / "cfg"))
    sim = lbib.Simulation(paths, lbib.FP64)
    sim.step(23)
    w = sim.write_simulation(str(tmp_path / "gpu"))
    ids, _ = sim.membrane()
    lines, arrays = _extra_records(ids)
    extra_force = str(tmp_path / "force_extra.txt")
    with open(extra_force, "w") as f:
        f.write(open(w["force"]).read().rstrip("\n") + "\n" + "\n".join(lines) + "\n")
    rpaths = {"parameters": w["parameters"], "geometry": w["geometry"], "force": extra_force,
              "plugins": paths["plugins"]}
    dumps = oracle_mod.run_reference(rpaths, str(tmp_path / "ref"), extra=("restart", w["solver"]))
    plain = dict(rpaths, force=w["force"])
    again = lbib.Simulation(plain, lbib.FP64)
    again.load_solvers(w["solver"])
    again.add_forces(*arrays)
    # the list now holds, node by node, the tension records and then the new
    # ones: the force file the reference would write after loading extra_force
    mid = again.write_simulation(str(tmp_path / "mid"))
    assert _by_node(mid["force"]) == _by_node(extra_force)
    again.step(20)
    ref = _at_iteration(dumps, 43)
    lat = again.lattice()
    for name in ("f", "g", "vel", "dom"):
        a, b = getattr(lat, name), getattr(ref, name)
        assert np.array_equal(a, b), f"{name} differs (max {np.abs(a.astype(float) - b.astype(float)).max()})"
    i2, node = again.membrane()
    assert np.array_equal(i2, ref.ids) and np.array_equal(node[:, :2], ref.node[:, :2])


def test_delete_force_type(lbib, tmp_path):
    """Records added and then deleted by type leave the run as if never added;
    deleteAllForces followed by the next renewal equals the plain run too."""
    paths = _cfg(20).write(str(tmp_path / "cfg"))
    base = lbib.Simulation(paths, lbib.FP64)
    edited = lbib.Simulation(paths, lbib.FP64)
    base.step(3)
    edited.step(3)
    ids, _ = edited.membrane()
    _, (types, id1, id2, par) = _extra_records(ids)
    # type 2 and 3 only (0 and 1 would survive the deletes below)
    edited.add_forces(types[2:], id1[2:], id2[2:], par[2:])
    edited.delete_force_type(2)
    edited.delete_force_type(3)
    base.step(10)
    edited.step(10)
    a, b = base.lattice(), edited.lattice()
    assert np.array_equal(a.f, b.f) and np.array_equal(a.g, b.g)
    # with the records in place for one step the run differs
    other = lbib.Simulation(paths, lbib.FP64)
    other.step(3)
    other.add_forces(types[2:], id1[2:], id2[2:], par[2:])
    other.step(10)
    assert not np.array_equal(other.lattice().f, a.f)


def test_add_forces_unknown_node(lbib, tmp_path):
    sim = lbib.Simulation(_cfg(20).write(str(tmp_path)), lbib.FP64)
    with pytest.raises(lbib.LbibError) as e:
        sim.add_forces([2], [999999], [0], [[1e-4, 0, 0, 0]])
    assert e.value.code == 50


# -- range queries ---------------------------------------------------------------

def _ref_order(ids, xy, dom_of, x, y, r, nx, ny, avoid):
    """fastneighborlist: bins of 1 lu clamped to the lattice; the query visits
    bins by row, then column, ids ascending within a bin; keeps distance <= r
    and drops nodes of the avoided domain."""
    def b(p, n):
        p = max(p, 0.0)
        return min(int(math.floor(p / 1.0)), n - 1)
    bins = {}
    for k, i in enumerate(ids):
        bins.setdefault((b(xy[k, 1], ny), b(xy[k, 0], nx)), []).append(k)
    hits, dist = [], []
    for by in range(b(y - r, ny), b(y + r, ny) + 1):
        for bx in range(b(x - r, nx), b(x + r, nx) + 1):
            for k in sorted(bins.get((by, bx), []), key=lambda k: ids[k]):
                d = math.sqrt((xy[k, 0] - x) * (xy[k, 0] - x) + (xy[k, 1] - y) * (xy[k, 1] - y))
                if d > r or (avoid >= 0 and dom_of[ids[k]] == avoid):
                    continue
                hits.append(int(ids[k]))
                dist.append(d)
    closest = -1
    if hits:
        closest = hits[int(np.argmin(dist))]  # first of the smallest
    return hits, closest


def test_range_queries(lbib, tmp_path):
    cfg = configs.junction_quad(iterations=20)
    sim = lbib.Simulation(cfg.write(str(tmp_path)), lbib.FP64)
    sim.step(7)
    ids, st = sim.membrane()
    conn = sim.connections()
    dom_of = {int(c[1]): int(c[2]) for c in conn}  # a node's incoming connection
    rng = np.random.default_rng(3)
    pts = np.concatenate([st[rng.choice(len(ids), 20), :2] + rng.uniform(-1.5, 1.5, (20, 2)),
                          [[62.0, 62.0], [1.0, 1.0], [62.0, 42.3]]])
    for radius, avoid in ((1.0, -1), (2.5, 1), (4.0, 3), (0.3, -1)):
        for x, y in pts:
            want, _ = _ref_order(ids, st[:, :2], dom_of, x, y, radius, cfg.nx, cfg.ny, avoid)
            got = sim.nodes_within_radius(x, y, radius, avoid)
            assert got.tolist() == want, (x, y, radius, avoid)
        av = np.array([avoid] * len(pts))
        got = sim.closest_nodes(pts[:, 0], pts[:, 1], radius, av)
        want = [_ref_order(ids, st[:, :2], dom_of, x, y, radius, cfg.nx, cfg.ny, avoid)[1] for x, y in pts]
        assert got.tolist() == want
    assert sum(len(sim.nodes_within_radius(x, y, 2.5)) for x, y in pts) > 50


def test_force_types_4_and_5_match_reference(lbib, oracle_mod, tmp_path):
    """The force types no other test loads: 4, the vertical slider (a spring
    toward the line x = position), and 5, a pull of constant magnitude toward
    a partner node (ForceStructs.hpp), read from the force file beside a
    spring and an anchor; FP64 exact against the reference build up to
    iteration 9 (the records are cleared at iteration 10)."""
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    cfg = configs.toy(n=48, r=8.0, nodes=80, iterations=9, report_step=3, species=1)
    cfg.area = None
    cfg.tension = None
    cfg.forces = ["4\t5\t24.5\t0.001\t0.8", "5\t12\t40\t0.0003", "5\t40\t12\t0.0003",
                  "4\t33\t23\t0.002\t1.25", "0\t20\t60\t0.001\t2.5", "1\t70\t24\t24\t0.0005\t0.5"]
    paths = cfg.write(str(tmp_path / "cfg"))
    ref = oracle_mod.run_reference(paths, str(tmp_path / "ref"))
    sim = lbib.Simulation(paths, lbib.FP64)
    done = 0
    for t in (3, 6, 9):
        sim.step(t - done)
        done = t
        lat = sim.lattice()
        st = ref[t]
        for k in ("f", "g", "vel", "force", "dom"):
            assert np.array_equal(getattr(lat, k), getattr(st, k)), (t, k)
        ids, node = sim.membrane()
        assert np.array_equal(node, st.node), t
    # the records did act: the membrane moved otherwise without them
    cfg.forces = []
    plain = lbib.Simulation(cfg.write(str(tmp_path / "plain")), lbib.FP64)
    plain.step(9)
    assert np.abs(plain.membrane()[1][:, :2] - node[:, :2]).max() > 1e-3
