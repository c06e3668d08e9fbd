"""VTK XML files without VTK: the .vtm geometry reader
(Geometry::loadGeometryVTK, Geometry.cpp:162-306) and the blocks of the
vtk*Reporter functors (vtkCellReporter.cpp, vtkForceReporter.cpp,
vtkCDEReporter.cpp, vtkFluidReporter.cpp).

The reader runs on the host (CPU tests); the writers and a run started from a
.vtm geometry need the GPU.  Expected values come from an independent parse
with xml.etree."""
import os
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from lbibcell_b200 import configs


def _f32(v):
    return struct.unpack("f", struct.pack("f", v))[0]


def _vtp_polygons(points, polys, dom, ctype, desc):
    """A poly data block in the layout VTK's ASCII writer gives it (points as
    Float32, strings as character codes ended by 0)."""
    def arr(tag, typ, name, vals, comps=1):
        extra = f' NumberOfComponents="{comps}"' if comps != 1 else ""
        return (f'        <{tag} type="{typ}" Name="{name}"{extra} format="ascii">\n          '
                + " ".join(vals) + f"\n        </{tag}>\n")
    codes = []
    for s in desc:
        codes += [str(ord(c)) for c in s] + ["0"]
    conn = [str(i) for p in polys for i in p]
    offs, o = [], 0
    for p in polys:
        o += len(p)
        offs.append(str(o))
    pts = []
    for x, y in points:
        pts += [repr(_f32(x)), repr(_f32(y)), "0"]
    return ('<?xml version="1.0"?>\n<VTKFile type="PolyData" version="0.1" byte_order="LittleEndian">\n'
            f'  <PolyData>\n    <Piece NumberOfPoints="{len(points)}" NumberOfVerts="0" NumberOfLines="0" '
            f'NumberOfStrips="0" NumberOfPolys="{len(polys)}">\n      <PointData>\n'
            + arr("DataArray", "Float64", "domain_identifier", [str(d) for d in dom])
            + arr("DataArray", "Float64", "cell_type", [str(c) for c in ctype])
            + arr("Array", "String", "boundarydescriptors", codes)
            + "      </PointData>\n      <CellData>\n      </CellData>\n      <Points>\n"
            + arr("DataArray", "Float32", "Points", pts, 3)
            + "      </Points>\n      <Polys>\n"
            + arr("DataArray", "Int64", "connectivity", conn) + arr("DataArray", "Int64", "offsets", offs)
            + "      </Polys>\n    </Piece>\n  </PolyData>\n</VTKFile>\n")


def _vtm(blocks):
    return ('<?xml version="1.0"?>\n<VTKFile type="vtkMultiBlockDataSet" version="1.0">\n  <vtkMultiBlockDataSet>\n'
            + "".join(f'    <DataSet index="{k}" file="{f}">\n    </DataSet>\n' for k, f in enumerate(blocks))
            + "  </vtkMultiBlockDataSet>\n</VTKFile>\n")


def _two_cells(d, extra_block=None, binary=False):
    os.makedirs(os.path.join(d, "G_0"), exist_ok=True)
    a = configs.circle(30.0, 30.0, 8.0, 40, phase=0.1)
    b = configs.circle(55.0, 30.0, 6.0, 30, phase=0.2)
    points = np.concatenate([a, b])
    polys = [list(range(40)), list(range(40, 70))]
    dom = [3] * 40 + [7] * 30
    ctype = [2] * 40 + [1] * 30
    desc = ["\t"] * 70
    desc[41] = "\tBoundarySolverNoFluxD2Q5\tLbibCDESolverD2Q5_A\t"
    text = _vtp_polygons(points, polys, dom, ctype, desc)
    if binary:
        text = text.replace('format="ascii"', 'format="binary"', 1)
    open(os.path.join(d, "G_0", "G_0_0.vtp"), "w").write(text)
    blocks = ["G_0/G_0_0.vtp"]
    if extra_block:
        open(os.path.join(d, "G_0", "G_0_1.vtp"), "w").write(text)
        blocks.append("G_0/G_0_1.vtp")
    open(os.path.join(d, "G_0.vtm"), "w").write(_vtm(blocks))
    return os.path.join(d, "G_0.vtm"), points, polys, dom


def _expected(points, polys, dom):
    xy = np.array([[_f32(x), _f32(y)] for x, y in points])
    conns = []
    for p in polys:
        for k in range(len(p) - 1):
            conns.append((p[k], p[k + 1], dom[p[0]]))
        conns.append((p[-1], p[0], dom[p[0]]))
    return xy, np.array(conns, np.uint32)


def test_read_vtm_geometry(tmp_path):
    from lbibcell_b200 import runner
    path, points, polys, dom = _two_cells(str(tmp_path))
    ids, xy, conns = runner.read_vtm_geometry(path)
    want_xy, want_conns = _expected(points, polys, dom)
    assert ids.tolist() == list(range(70))
    assert np.array_equal(xy, want_xy)  # Float32 points, widened like vtkPoints::GetPoint
    assert np.array_equal(conns, want_conns)


def test_read_vtm_errors(tmp_path):
    from lbibcell_b200 import runner
    with pytest.raises(Exception):
        runner.read_vtm_geometry(str(tmp_path / "missing.vtm"))
    two, _, _, _ = _two_cells(str(tmp_path / "two"), extra_block=True)
    with pytest.raises(Exception):  # "more or less than one vtk polygon block"
        runner.read_vtm_geometry(two)
    binary, _, _, _ = _two_cells(str(tmp_path / "bin"), binary=True)
    with pytest.raises(Exception):
        runner.read_vtm_geometry(binary)


def _etree_polygon_block(vtm):
    """The poly data block with polygons, read with xml.etree."""
    d = os.path.dirname(vtm)
    found = []
    for ds in ET.parse(vtm).getroot().iter("DataSet"):
        root = ET.parse(os.path.join(d, ds.get("file"))).getroot()
        if root.get("type") != "PolyData":
            continue
        piece = root.find("PolyData/Piece")
        if int(piece.get("NumberOfPolys")) > 0:
            found.append(piece)
    assert len(found) == 1
    return found[0]


def test_reference_vtm_geometry():
    """The geometry file that the reference's tutorial_01 loads
    (apps/config/vtk/Cells_0.vtm), where the reference sources are present."""
    from oracle import oracle as O
    path = os.path.join(O.REFERENCE, "apps", "config", "vtk", "Cells_0.vtm")
    if not os.path.exists(path):
        pytest.skip("reference sources not present")
    from lbibcell_b200 import runner
    ids, xy, conns = runner.read_vtm_geometry(path)
    piece = _etree_polygon_block(path)
    pts = np.array(piece.find("Points/DataArray").text.split(), np.float32).reshape(-1, 3)
    assert np.array_equal(xy, pts[:, :2].astype(np.float64))
    con = [int(v) for v in piece.find("Polys/DataArray[@Name='connectivity']").text.split()]
    dom = [float(v) for v in piece.find("PointData/DataArray[@Name='domain_identifier']").text.split()]
    assert conns.shape == (len(con), 3)
    assert conns[:, 0].tolist() == con and conns[:, 1].tolist() == con[1:] + con[:1]
    assert set(conns[:, 2].tolist()) == {int(dom[con[0]])}


# -- GPU: writers and runs from a .vtm geometry --------------------------------------

@pytest.fixture(scope="module")
def lbib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from lbibcell_b200 import build, runner
    build.build()
    return runner


def _seq_sum(a):
    """Sum over the last axis in index order (std::accumulate), not numpy's
    pairwise order."""
    out = a[..., 0].copy()
    for q in range(1, a.shape[-1]):
        out = out + a[..., q]
    return out


def _arr(piece, path, name):
    for a in piece.iter():
        if a.get("Name") == name:
            return a
    raise KeyError(name)


@pytest.mark.gpu
def test_reporters_blocks(lbib, tmp_path):
    cfg = configs.junction_quad(iterations=20)
    sim = lbib.Simulation(cfg.write(str(tmp_path / "cfg")), lbib.FP64)
    sim.step(10)  # junction springs and tension records in the force list
    prefix = str(tmp_path / "out" / "Cells")
    os.makedirs(os.path.dirname(prefix))
    for kind, c in ((sim.VTK_CELLS, 1), (sim.VTK_CELL_PNG, 1), (sim.VTK_FORCES, 1), (sim.VTK_CDE, 1),
                    (sim.VTK_FLUID, 4)):
        vtm = sim.write_vtk(prefix, 10, kind, c)
    root = ET.parse(vtm).getroot()
    files = [ds.get("file") for ds in root.iter("DataSet")]
    assert files == ["Cells_10/Cells_10_0.vtp", "Cells_10/Cells_10_1.vtp", "Cells_10/Cells_10_2.vti",
                     "Cells_10/Cells_10_3.vti"]
    base = os.path.dirname(vtm)
    ids, st = sim.membrane()
    conn = sim.connections()
    # cells: one polygon per cell, points = the second node of each connection in ring order
    cells = ET.parse(os.path.join(base, files[0])).getroot().find("PolyData/Piece")
    assert int(cells.get("NumberOfPolys")) == 4 and int(cells.get("NumberOfPoints")) == len(ids)
    pts = np.array(_arr(cells, "", "Points").text.split(), np.float64).reshape(-1, 3)
    pos = {int(i): (np.float32(st[k, 0]), np.float32(st[k, 1])) for k, i in enumerate(ids)}
    first = {}
    for c in conn:
        first.setdefault(int(c[2]), c)
    start = first[min(first)]
    assert (np.float32(pts[0, 0]), np.float32(pts[0, 1])) == pos[int(start[1])]
    # forces: a line per record with a partner; the types are those of the list
    forces = ET.parse(os.path.join(base, files[1])).getroot().find("PolyData/Piece")
    ft = [int(v) for v in _arr(forces, "", "ForceType").text.split()]
    assert set(ft) == {6, 7} and int(forces.get("NumberOfLines")) == len(ft)
    w = sim.write_simulation(str(tmp_path / "w"))
    lines = [l.split() for l in open(w["force"]) if l.strip() and not l.startswith("#")]
    assert len(ft) == sum(1 for l in lines if l[0] in ("0", "5", "6", "7") and l[2] != "0")
    # CDE: one array per species, c = sum of g, every node
    lat = sim.lattice()
    cde = ET.parse(os.path.join(base, files[2])).getroot().find("ImageData")
    assert cde.get("WholeExtent") == f"0 {cfg.nx - 1} 0 {cfg.ny - 1} 0 0"
    c = np.array(_arr(cde, "", cfg.species[0].name).text.split(), np.float64)
    assert np.array_equal(c, _seq_sum(lat.g[0]))
    # fluid, coarsened by 4: density = sum f, velocity (ux, uy, 0)
    fl = ET.parse(os.path.join(base, files[3])).getroot().find("ImageData")
    assert fl.get("WholeExtent") == f"0 {cfg.nx // 4 - 1} 0 {cfg.ny // 4 - 1} 0 0" and fl.get("Spacing") == "4 4 4"
    rho = np.array(_arr(fl, "", "density").text.split(), np.float64)
    sel = (np.arange(0, cfg.ny, 4)[:, None] * cfg.nx + np.arange(0, cfg.nx, 4)[None, :]).ravel()
    assert np.array_equal(rho, _seq_sum(lat.f[sel]))
    vel = np.array(_arr(fl, "", "velocity").text.split(), np.float64).reshape(-1, 3)
    assert np.array_equal(vel[:, :2], lat.vel[sel]) and not vel[:, 2].any()


@pytest.mark.gpu
def test_run_from_vtm_matches_reference(lbib, oracle_mod, tmp_path):
    """A .vtm written by the cell reporter starts a run here; the reference
    build (whose VTK reader is not available without VTK) starts from the same
    geometry as text (ids 0..n-1, the Float32 positions); FP64 results agree
    after 30 steps."""
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    cfg = configs.junction_quad(iterations=30)
    cfg.bio = []
    paths = cfg.write(str(tmp_path / "cfg"))
    sim = lbib.Simulation(paths, lbib.FP64)
    vtm = sim.write_vtk(str(tmp_path / "Geo"), 0, sim.VTK_CELLS)
    ids, xy, conns = lbib.read_vtm_geometry(vtm)
    geo_txt = str(tmp_path / "geo_from_vtm.txt")
    with open(geo_txt, "w") as f:
        f.write("#Nodes (id\txPos\tyPos)\n")
        for i, (x, y) in zip(ids, xy):
            f.write(f"{i}\t{x:.17g}\t{y:.17g}\n")
        f.write("#Connection (nodeId1\tnodeId2\tdomainId\tbsolver\tcdesolver\t...)\n")
        for a, b, d in conns:
            f.write(f"{a}\t{b}\t{d}\n")
    ref = oracle_mod.run_reference(dict(paths, geometry=geo_txt), str(tmp_path / "ref"))
    mine = lbib.Simulation(dict(paths, geometry=vtm), lbib.FP64)
    mine.step(30)
    st = ref[30]
    lat = mine.lattice()
    for name in ("f", "g", "vel", "dom"):
        assert np.array_equal(getattr(lat, name), getattr(st, name)), name
    i2, node = mine.membrane()
    assert np.array_equal(i2, st.ids) and np.array_equal(node[:, :2], st.node[:, :2])
