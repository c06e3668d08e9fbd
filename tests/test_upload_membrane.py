"""Topology edits by a host bio solver between steps (lbib_upload_membrane):
the Geometry edits a cell division makes (Geometry.cpp:381-452), given as the
new node and connection lists.

A run edited in place must continue exactly like a run restarted from files
that hold the edited geometry, and that restarted run exactly like the
reference build restarted from the same files (FP64)."""
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
    cfg = configs.toy(n=64, r=12.0, nodes=120, iterations=iterations, report_step=10, species=2)
    cfg.area = None  # the area regulator's targets are plugin state that no file holds
    return cfg


def _ring(ids, conns):
    """Node ids of the (single) ring in connection order, and the positions."""
    nxt = {int(a): int(b) for a, b, _ in conns}
    start = int(conns[0][0])
    ring, n = [start], nxt[start]
    while n != start:
        ring.append(n)
        n = nxt[n]
    return ring


def _divide(ids, st, conns):
    """A cell division as a host plugin makes it through GeometryHandler:
    split the one cell along the chord between two opposite ring nodes a and b.
    Daughter 1 keeps the ring from a to b and closes along a row of new nodes
    0.35 lu inside it; daughter 2 (a new domain) gets new copies of b and a,
    0.7 lu inside it, the rest of the ring, and a closing row of its own.  The
    connections of that rest are erased and created again with the new domain.
    Returns the edit (erased pairs, new node positions in creation order, new
    connections in creation order) and the resulting node and connection
    lists (kept connections in their order, then the created ones)."""
    pos = {int(i): st[k, :2] for k, i in enumerate(ids)}
    ring = _ring(ids, conns)
    dom = int(conns[0][2])
    n = len(ring)
    a, b = ring[0], ring[n // 2]
    pa, pb = pos[a], pos[b]
    d = pb - pa
    length = float(np.linalg.norm(d))
    normal = np.array([-d[1], d[0]]) / length  # toward daughter 2
    steps = int(length / 0.45)
    new_pos = []
    next_id = [int(ids.max()) + 1]

    def new(p):
        new_pos.append(p)
        next_id[0] += 1
        return next_id[0] - 1

    chord1 = [new(pb + (s / steps) * (pa - pb) - 0.35 * normal) for s in range(1, steps)]
    b2 = new(pb + 0.7 * normal)
    a2 = new(pa + 0.7 * normal)
    chord2 = [new(pa + (s / steps) * d + 0.7 * normal) for s in range(1, steps)]
    rest = ring[n // 2:] + [a]                      # b .. a along the ring
    erase = [(rest[i], rest[i + 1]) for i in range(len(rest) - 1)]
    d1 = [b] + chord1 + [a]
    d2 = [b2] + ring[n // 2 + 1:] + [a2] + chord2 + [b2]
    created = [(d1[i], d1[i + 1], dom) for i in range(len(d1) - 1)]
    created += [(d2[i], d2[i + 1], dom + 1) for i in range(len(d2) - 1)]
    gone = set(erase)
    kept = [(int(x), int(y), int(dm)) for x, y, dm in conns if (int(x), int(y)) not in gone]
    all_pos = dict(pos)
    for k, p in enumerate(new_pos):
        all_pos[int(ids.max()) + 1 + k] = p
    new_ids = np.array(sorted(all_pos), np.uint32)
    xy = np.array([all_pos[int(i)] for i in new_ids])
    return (erase, new_pos, created), (new_ids, xy, np.array(kept + created, np.uint32))


def _write_edit(path, edit):
    erase, new_pos, created = edit
    with open(path, "w") as f:
        for x, y in erase:
            f.write(f"erase\t{x}\t{y}\n")
        for p in new_pos:
            f.write(f"node\t{p[0]:.17g}\t{p[1]:.17g}\n")
        for x, y, dm in created:
            f.write(f"conn\t{x}\t{y}\t{dm}\n")


def _write_geometry(path, ids, xy, conns):
    with open(path, "w") as f:
        f.write("#Nodes (id\txPos\tyPos)\n")
        for i, (x, y) in zip(ids, xy):
            f.write(f"{int(i)}\t{x:.17g}\t{y:.17g}\n")
        f.write("#Connection (nodeId1\tnodeId2\tdomainId\tbsolver\tcdesolver\t...)\n")
        for a, b, d in conns:
            f.write(f"{int(a)}\t{int(b)}\t{int(d)}\n")


def _same(a, b, what):
    la, lb = a.lattice(), b.lattice()
    for name in ("f", "g", "vel", "dom"):
        x, y = getattr(la, name), getattr(lb, name)
        assert np.array_equal(x, y), f"{what}: {name} differs (max {np.abs(x.astype(float) - y.astype(float)).max()})"
    ia, na = a.membrane()
    ib, nb = b.membrane()
    assert np.array_equal(ia, ib) and np.array_equal(na[:, :2], nb[:, :2]), f"{what}: membrane differs"


def test_upload_unchanged_membrane(lbib, tmp_path):
    """Uploading the current membrane changes nothing."""
    paths = _cfg(40).write(str(tmp_path))
    a = lbib.Simulation(paths, lbib.FP64)
    b = lbib.Simulation(paths, lbib.FP64)
    a.step(13)
    b.step(13)
    ids, st = b.membrane()
    b.upload_membrane(ids, st[:, :2], b.connections())
    a.step(20)
    b.step(20)
    _same(a, b, "unchanged upload")


def test_division_matches_reference(lbib, oracle_mod, tmp_path):
    """A division at iteration 23, made here through lbib_upload_membrane and
    lbib_cure_lattice, and in the reference build through GeometryHandler's
    eraseConnection / createGeometryNode / createConnection and cureLattice, as
    the reference's division plugin does; FP64 results agree at iteration 43."""
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    paths = _cfg(43).write(str(tmp_path / "cfg"))
    sim = lbib.Simulation(paths, lbib.FP64)
    sim.step(23)
    ids, st = sim.membrane()
    edit, (new_ids, xy, conns) = _divide(ids, st, sim.connections())
    edit_file = str(tmp_path / "division.txt")
    _write_edit(edit_file, edit)
    # the reference build: the same run, the edit applied at iteration 23
    dumps = oracle_mod.run_reference(paths, str(tmp_path / "ref"), extra=("edit", 23, edit_file))
    sim.upload_membrane(new_ids, xy, conns)
    sim.cure_lattice()
    sim.step(20)
    ref = [s for k, s in dumps.items() if k != "stdout" and s.current_iteration == 43][0]
    lat = sim.lattice()
    for name in ("f", "g", "vel", "dom"):
        a, b = getattr(lat, name), getattr(ref, name)
        assert np.array_equal(a, b), f"{name} differs (max {np.abs(a.astype(float) - b.astype(float)).max()})"
    i2, node = sim.membrane()
    assert np.array_equal(i2, ref.ids) and np.array_equal(node[:, :2], ref.node[:, :2])
    assert len(sim.areas()) == 2
    assert set(np.unique(lat.dom).tolist()) == {0, 1, 2}


def test_upload_rejects_bad_lists(lbib, tmp_path):
    sim = lbib.Simulation(_cfg(20).write(str(tmp_path)), lbib.FP64)
    ids, st = sim.membrane()
    conns = sim.connections()
    with pytest.raises(lbib.LbibError):
        sim.upload_membrane(ids[::-1], st[::-1, :2], conns)  # ids must ascend
    sim2 = lbib.Simulation(_cfg(20).write(str(tmp_path / "b")), lbib.FP64)
    bad = conns.copy()
    bad[0, 1] = ids.max() + 100
    with pytest.raises(lbib.LbibError):
        sim2.upload_membrane(ids, st[:, :2], bad)


def test_connection_perturbation_listed_equals_full(lbib, tmp_path, monkeypatch, capfd):
    """GeometryHandler::perturbConnections inside a step (GeometryHandler.cpp:
    326-356): connections whose end points share an x or a y are perturbed
    by the host from the device's list of them (and the ring-closing test),
    without the membrane crossing the bus.  The same run with
    LBIB_FULL_HOST_EVENTS=1 (the reference's full ring walk on a host copy of
    the membrane) gives identical states.  The connections are made vertical
    and horizontal by an upload with the fluid at rest and no forces, so the
    first step's move keeps them: the walk's first connection (node 0 -> 1),
    the walk's last (node n-1 -> 0) and one at the top (30 -> 31)."""
    paths = _cfg(10).write(str(tmp_path))
    monkeypatch.setenv("LBIB_LOG_HOST_EVENTS", "1")

    def run(full):
        if full:
            monkeypatch.setenv("LBIB_FULL_HOST_EVENTS", "1")
        else:
            monkeypatch.delenv("LBIB_FULL_HOST_EVENTS", raising=False)
        sim = lbib.Simulation(paths, lbib.FP64)
        ids, st = sim.membrane()
        xy = st[:, :2].copy()
        n = len(ids)
        xy[1, 0] = xy[0, 0]
        xy[n - 1, 0] = xy[0, 0]
        xy[31, 1] = xy[30, 1]
        sim.upload_membrane(ids, xy, sim.connections())
        sim.step(1)
        _, moved = sim.membrane()
        sim.step(4)
        return sim, moved

    capfd.readouterr()
    a, moved_a = run(False)
    log_a = capfd.readouterr().err
    b, moved_b = run(True)
    log_b = capfd.readouterr().err
    assert "stage 5" in log_a and "listed" in log_a.split("stage 5")[1].splitlines()[0], log_a
    assert "stage 5" in log_b and "full membrane" in log_b.split("stage 5")[1].splitlines()[0], log_b
    assert np.array_equal(moved_a, moved_b)
    _same(a, b, "listed vs full connection perturbation")
