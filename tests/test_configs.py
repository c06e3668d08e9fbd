"""Synthetic configurations: reference formats, counter-clockwise cells, margins."""
import numpy as np

from lbibcell_b200 import configs


def _signed_area(v):
    x, y = v[:, 0], v[:, 1]
    return 0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)


def test_config1_files(tmp_path):
    cfg = configs.config1()
    p = cfg.write(str(tmp_path))
    text = open(p["parameters"]).read()
    assert "SizeX:\t200" in text and "CDESolvers:\tLbibCDESolverD2Q5_A\t1.0" in text
    geo = open(p["geometry"]).read().splitlines()
    assert geo[0].startswith("#Nodes") and sum(1 for l in geo if not l.startswith("#")) == 500
    plug = open(p["plugins"]).read()
    assert "MassSolverBoxOutlet" in plug and "LbibAreaRegulator" in plug and "LbibMembraneTension" in plug


def test_cells_ccw_and_inside():
    for cfg in (configs.config1(), configs.toy()):
        for dom, v in cfg.cells:
            assert _signed_area(v) > 0
            assert v[:, 0].min() > 3 and v[:, 1].min() > 3
            assert v[:, 0].max() < cfg.nx - 3 and v[:, 1].max() < cfg.ny - 3


def test_config2_shape():
    cfg = configs.config2()
    assert cfg.nx == 1024 and len(cfg.species) == 2
    assert len(cfg.cells) == 400
    assert cfg.bio[0].split("\t")[0] == "LbibCellJunction"
    doms = [d for d, _ in cfg.cells]
    assert len(set(doms)) == len(doms)
    for _, v in cfg.cells:
        assert _signed_area(v) > 0
