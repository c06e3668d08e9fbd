"""Seeded synthetic configurations in LBIBCell's own text formats.

Each configuration is four files:

* ``parameters.txt`` -- the reference's global parameter file
  (``libs/LbmLib/src/GlobalSimulationParameters.cpp:34-72``): ``CurrentIterations:``,
  ``Iterations:``, ``ReportStep:``, ``SizeX:``, ``SizeY:``, ``tauFluid:``,
  ``CDESolvers: name tau ...``.
* ``geometry.txt`` -- the reference's txt geometry
  (``libs/LbmLib/src/geometry/Geometry.cpp:99-160``): ``#Nodes`` lines ``id x y`` then
  ``#Connection`` lines ``id1 id2 domainId [bsolver cdesolver]...``.  Cells are
  counter-clockwise polygons, so that the inside is the domain side of each
  connection (``libs/LbmLib/src/geometry/Connection.cpp:246-314``).
* ``force.txt`` -- the reference's force file (``apps/config/force.txt``); comment
  lines only unless a config adds static forces.
* ``plugins.txt`` -- the solver plugins to register and their parameters.  The
  reference hard-codes these constants inside each plugin; this file carries them
  instead.  One plugin per line, tab separated::

      MassSolver  MassSolverBoxOutlet
      BioSolver   LbibAreaRegulator    factor F strength K maxsource M
      BioSolver   LbibMembraneTension  force F frequency N
      BioSolver   LbibCellDivision     factor F frequency N
      ForceModel  GuoZhengShi2002ForceModel  (or ...Corrected; default Luo1993ForceModel)
      CDE         <species name>       init C0 decay D
      CDESource   <species name>       <domainId> <rate> [<domainId> <rate> ...]

  Bio solvers run in file order.  Species names are the ``CDESolvers:`` names of the
  parameter file (``LbibCDESolverD2Q5_A``, ``_B``, ``_C``); the reference orders
  species alphabetically (a ``std::map``).

Node coordinates are written with 17 significant digits, so that every reader
parses exactly the doubles that were generated.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

SPECIES_NAMES = ("LbibCDESolverD2Q5_A", "LbibCDESolverD2Q5_B", "LbibCDESolverD2Q5_C")


@dataclass
class Species:
    name: str
    tau: float
    init: float = 0.0
    decay: float = 0.0
    source: Dict[int, float] = field(default_factory=dict)


@dataclass
class Config:
    """A complete simulation set-up: lattice, cells, solvers."""

    name: str
    nx: int
    ny: int
    tau_fluid: float
    iterations: int
    report_step: int
    cells: List[Tuple[int, np.ndarray]]  # (domainId, (n, 2) CCW vertices)
    species: List[Species]
    outlet: bool = True
    current_iteration: int = 0
    tension: Optional[Tuple[float, int]] = (0.1, 10)  # (force, frequency)
    area: Optional[Tuple[float, float, float]] = (1.2, 0.01, 0.004)  # factor, strength, maxsource
    forces: List[str] = field(default_factory=list)
    # boundary solvers on every connection: (bsolver, cdesolver) pairs, as the
    # reference's geometry files list them (apps/config/tutorial_02_geometry.txt)
    boundary: List[Tuple[str, str]] = field(default_factory=list)
    # further bio solvers by name (e.g. "tutorial_01_BioSolverCellJunction"),
    # registered before (bio_first) or after the area regulator and tension
    bio: List[str] = field(default_factory=list)
    bio_first: bool = False
    # FluidSolver's force model: None (Luo1993ForceModel, the reference's),
    # "GuoZhengShi2002ForceModel" or "GuoZhengShi2002ForceModelCorrected"
    force_model: Optional[str] = None

    @property
    def lattice_nodes(self) -> int:
        return self.nx * self.ny

    @property
    def membrane_nodes(self) -> int:
        return sum(len(v) for _, v in self.cells)

    def write(self, directory: str) -> Dict[str, str]:
        """Write the four files into ``directory``; returns their paths."""
        os.makedirs(directory, exist_ok=True)
        paths = {k: os.path.join(directory, k + ".txt") for k in ("parameters", "geometry", "force", "plugins")}
        with open(paths["parameters"], "w") as f:
            f.write("#Global Parameter file\n")
            f.write(f"CurrentIterations:\t{self.current_iteration}\n")
            f.write(f"Iterations:\t{self.iterations}\n")
            f.write(f"ReportStep:\t{self.report_step}\n")
            f.write(f"SizeX:\t{self.nx}\n")
            f.write(f"SizeY:\t{self.ny}\n")
            f.write(f"tauFluid:\t{self.tau_fluid!r}\n")
            f.write("CDESolvers:")
            for s in self.species:
                f.write(f"\t{s.name}\t{s.tau!r}")
            f.write("\n")
        with open(paths["geometry"], "w") as f:
            f.write("#Nodes (id\txPos\tyPos)\n")
            nid = 1
            conns = []
            for dom, verts in self.cells:
                first = nid
                for x, y in verts:
                    f.write(f"{nid}\t{float(x):.17g}\t{float(y):.17g}\n")
                    nid += 1
                ids = list(range(first, nid))
                for i, a in enumerate(ids):
                    conns.append((a, ids[(i + 1) % len(ids)], dom))
            f.write("#Connection (nodeId1\tnodeId2\tdomainId\tbsolver\tcdesolver\t...)\n")
            desc = "".join(f"\t{bs}\t{cde}" for bs, cde in self.boundary)
            for a, b, d in conns:
                f.write(f"{a}\t{b}\t{d}{desc}\n")
        with open(paths["force"], "w") as f:
            f.write("#Force 6 {type=6 id1 id2 f}\tmembrane tension (renewed by LbibMembraneTension)\n")
            for line in self.forces:
                f.write(line.rstrip("\n") + "\n")
        with open(paths["plugins"], "w") as f:
            f.write("#lbibcell_b200 plugin file\n")
            if self.force_model:
                f.write(f"ForceModel\t{self.force_model}\n")
            if self.outlet:
                f.write("MassSolver\tMassSolverBoxOutlet\n")
            if self.bio_first:
                for name in self.bio:
                    f.write(f"BioSolver\t{name}\n")
            if self.area is not None:
                fa, st, mx = self.area
                f.write(f"BioSolver\tLbibAreaRegulator\tfactor\t{fa!r}\tstrength\t{st!r}\tmaxsource\t{mx!r}\n")
            if self.tension is not None:
                fo, fr = self.tension
                f.write(f"BioSolver\tLbibMembraneTension\tforce\t{fo!r}\tfrequency\t{fr}\n")
            if not self.bio_first:
                for name in self.bio:
                    f.write(f"BioSolver\t{name}\n")
            for s in self.species:
                f.write(f"CDE\t{s.name}\tinit\t{s.init!r}\tdecay\t{s.decay!r}\n")
                if s.source:
                    f.write(f"CDESource\t{s.name}")
                    for d in sorted(s.source):
                        f.write(f"\t{d}\t{s.source[d]!r}")
                    f.write("\n")
        return paths


def circle(cx: float, cy: float, r: float, n: int, phase: float = 0.0) -> np.ndarray:
    """n vertices at uniform angle, counter-clockwise."""
    t = phase + 2.0 * math.pi * np.arange(n) / n
    return np.stack([cx + r * np.cos(t), cy + r * np.sin(t)], axis=1)


def junction_quad(iterations: int = 60, report_step: int = 30, tension: Tuple[float, int] = (0.1, 10),
                  bio_first: bool = False, name: str = "tutorial_01_BioSolverCellJunction") -> Config:
    """Four cells of radius 19.6 on a 40 lu square grid in a 124x124 lattice:
    neighbouring membranes 0.8 lu apart, within the junction radius (1 lu) of
    the cell-junction solver, which is registered with them."""
    cells = []
    for k, (cx, cy) in enumerate([(42.0, 42.0), (82.0, 42.0), (42.0, 82.0), (82.0, 82.0)]):
        cells.append((k + 1, circle(cx, cy, 19.6, 240, phase=0.1 * (k + 1))))
    return Config(name="junction_quad", nx=124, ny=124, tau_fluid=1.0, iterations=iterations,
                  report_step=report_step, cells=cells,
                  species=[Species(SPECIES_NAMES[0], 1.0, source={1: 1e-3, 4: 1e-3})],
                  tension=tension, bio=[name], bio_first=bio_first)


def config1(iterations: int = 2000, report_step: int = 500) -> Config:
    """Single circular cell (tutorial_01 style): 200x200, r=20, 250 nodes, 1 species."""
    return Config(
        name="single_cell_200",
        nx=200, ny=200, tau_fluid=1.0,
        iterations=iterations, report_step=report_step,
        cells=[(1, circle(100.0, 100.0, 20.0, 250))],
        species=[Species(SPECIES_NAMES[0], 1.0, init=0.0, decay=0.0, source={1: 1e-3})],
    )


def toy(n: int = 64, r: float = 10.0, nodes: int = 100, iterations: int = 100, report_step: int = 25,
        species: int = 1, tau_fluid: float = 1.0) -> Config:
    """Small single-cell case for fast tests."""
    taus = (1.0, 0.8, 1.2)
    sp = [Species(SPECIES_NAMES[k], taus[k], init=0.0, decay=1e-4 * k, source={1: 1e-3 * (k + 1)})
          for k in range(species)]
    return Config(
        name=f"toy_{n}", nx=n, ny=n, tau_fluid=tau_fluid,
        iterations=iterations, report_step=report_step,
        cells=[(1, circle(n / 2.0, n / 2.0, r, nodes))],
        species=sp,
    )


def hex_tissue(nx: int, ny: int, spacing: float, r0: float, jitter: float, nodes_per_cell: int,
               seed: int, cols: int, rows: int) -> List[Tuple[int, np.ndarray]]:
    """cols x rows cells on a hexagonal grid (centred in the lattice), radius
    r0 + U(-jitter, jitter), each with a random phase for its first node."""
    rng = np.random.default_rng(seed)
    dy = spacing * math.sqrt(3.0) / 2.0
    w = (cols - 1) * spacing + spacing / 2.0
    h = (rows - 1) * dy
    x0, y0 = (nx - w) / 2.0, (ny - h) / 2.0
    cells = []
    dom = 1
    for row in range(rows):
        for col in range(cols):
            x = x0 + col * spacing + (spacing / 2.0 if row % 2 else 0.0)
            y = y0 + row * dy
            r = r0 + rng.uniform(-jitter, jitter)
            cells.append((dom, circle(x, y, r, nodes_per_cell, phase=rng.uniform(0, 2 * math.pi))))
            dom += 1
    return cells


def config2(iterations: int = 10000, report_step: int = 1000, seed: int = 0) -> Config:
    """1024x1024 tissue: 400 cells (20 x 20) on a hex grid (spacing 44), r=20+U(-2,2),
    250 nodes/cell, 2 species (tau 0.8, 1.2), secretion 1e-3/step from a seeded 10% of
    the cells; membrane tension, area regulator and cell junctions (the
    reference's tutorial_01 junction solver with a 2 lu rest length: springs
    between nodes of different cells closer than 1 lu push them apart)."""
    cells = hex_tissue(1024, 1024, 44.0, 20.0, 2.0, 250, seed, cols=20, rows=20)
    rng = np.random.default_rng(seed + 1)
    doms = [d for d, _ in cells]
    k = max(1, len(doms) // 10)
    sec = sorted(rng.choice(doms, size=k, replace=False).tolist())
    species = [Species(SPECIES_NAMES[0], 0.8, source={d: 1e-3 for d in sec}),
               Species(SPECIES_NAMES[1], 1.2, source={d: 1e-3 for d in sec})]
    # Cells of radius up to 22 on a 44 lu grid already touch; a growth target
    # would press neighbours into each other (and the reference's species
    # re-initialisation divides by zero for nodes trapped between two
    # membranes, CDESolverD2Q5.cpp:223).  The area regulator holds each cell's
    # initial area here.
    return Config(name="tissue_1024", nx=1024, ny=1024, tau_fluid=1.0, iterations=iterations,
                  report_step=report_step, cells=cells, species=species, area=(1.0, 0.01, 0.004),
                  bio=["LbibCellJunction\tradius\t1.0\tk\t0.02\tl0\t2.0"])


def poisson_tissue(nx: int, ny: int, rmin: float, rmax: float, spacing: float, seed: int,
                   margin: float = 6.0, gap: float = 3.0, max_cells: Optional[int] = None):
    """Cells placed by seeded dart throwing (Poisson-disk), radii U(rmin, rmax),
    membrane node spacing ``spacing``."""
    rng = np.random.default_rng(seed)
    cell_size = 2 * rmax + gap
    gw, gh = int(nx // cell_size) + 1, int(ny // cell_size) + 1
    grid: Dict[Tuple[int, int], List[int]] = {}
    placed: List[Tuple[float, float, float]] = []
    attempts = 0
    limit = 60 * (nx * ny) // int(cell_size * cell_size)
    while attempts < limit:
        attempts += 1
        r = rng.uniform(rmin, rmax)
        x = rng.uniform(margin + r, nx - margin - r)
        y = rng.uniform(margin + r, ny - margin - r)
        gx, gy = int(x // cell_size), int(y // cell_size)
        ok = True
        for ix in range(gx - 1, gx + 2):
            for iy in range(gy - 1, gy + 2):
                for j in grid.get((ix, iy), ()):
                    px, py, pr = placed[j]
                    if (px - x) ** 2 + (py - y) ** 2 < (pr + r + gap) ** 2:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        grid.setdefault((gx, gy), []).append(len(placed))
        placed.append((x, y, r))
        if max_cells is not None and len(placed) >= max_cells:
            break
    cells = []
    for i, (x, y, r) in enumerate(placed):
        n = max(8, int(round(2 * math.pi * r / spacing)))
        cells.append((i + 1, circle(x, y, r, n, phase=rng.uniform(0, 2 * math.pi))))
    return cells


def config3(iterations: int = 5000, report_step: int = 1000, seed: int = 0, cells: int = 6000) -> Config:
    """4096x4096 tissue: ``cells`` cells placed by seeded Poisson-disk sampling
    (dart throwing, gap 3 lu) with radii U(10,16) and membrane node spacing
    0.5 lu (~1.1M nodes for 6000 cells); membrane tension, cell junctions
    (radius 1 lu, k 0.02, rest length 2 lu), area growth toward 2.5x the
    initial area (LbibAreaRegulator: strength 0.01, at most 2e-4 per node and
    step) with division at 2x the initial area (LbibCellDivision, checked every
    100 iterations); 3 D2Q5 species (tau 0.55, 1.0, 1.5) with linear decay
    1e-4, secreted at 1e-3 per step by every tenth cell."""
    placed = poisson_tissue(4096, 4096, 10.0, 16.0, 0.5, seed, max_cells=cells)
    species = [Species(SPECIES_NAMES[k], t, decay=1e-4, source={d: 1e-3 for d, _ in placed[::10]})
               for k, t in enumerate((0.55, 1.0, 1.5))]
    return Config(name="tissue_4096", nx=4096, ny=4096, tau_fluid=1.0, iterations=iterations,
                  report_step=report_step, cells=placed, species=species, area=(2.5, 0.01, 2e-4),
                  bio=["LbibCellJunction\tradius\t1.0\tk\t0.02\tl0\t2.0",
                       "LbibCellDivision\tfactor\t2.0\tfrequency\t100"])


def config4(iterations: int = 2000, report_step: int = 1000, seed: int = 0) -> Config:
    """Adjoint workload, 512x512: 50 Poisson-disk cells r~U(12,18), node spacing
    0.5, one species (tau 0.8) produced in every cell at a seeded per-cell
    rate U(0.5, 1.5) * 1e-3.  Differentiated over T=2000 steps with a
    checkpoint every 100."""
    cells = poisson_tissue(512, 512, 12.0, 18.0, 0.5, seed, max_cells=50)
    rng = np.random.default_rng(seed + 4)
    rates = {d: float(1e-3 * rng.uniform(0.5, 1.5)) for d, _ in cells}
    species = [Species(SPECIES_NAMES[0], 0.8, source=rates)]
    return Config(name="adjoint_512", nx=512, ny=512, tau_fluid=1.0, iterations=iterations,
                  report_step=report_step, cells=cells, species=species, area=None)


def config5(iterations: int = 10000, report_step: int = 1000, seed: int = 0) -> Config:
    """Adjoint workload, 2048x2048: 1000 Poisson-disk cells r~U(10,16), two
    species (tau 0.8, 1.2) with seeded per-cell rates, and the area regulator
    (target 1.2x the first area, strength 0.01 per cell) whose per-cell
    strengths are the differentiated parameters.  Differentiated over
    T=10000 steps with sqrt(T) checkpoints."""
    cells = poisson_tissue(2048, 2048, 10.0, 16.0, 0.5, seed, max_cells=1000)
    rng = np.random.default_rng(seed + 5)
    species = [Species(SPECIES_NAMES[k], t, source={d: float(1e-3 * rng.uniform(0.5, 1.5)) for d, _ in cells})
               for k, t in enumerate((0.8, 1.2))]
    return Config(name="adjoint_2048", nx=2048, ny=2048, tau_fluid=1.0, iterations=iterations,
                  report_step=report_step, cells=cells, species=species, area=(1.2, 0.01, 0.004), tension=None)


CONFIGS = {"config1": config1, "config2": config2, "config3": config3, "config4": config4, "config5": config5,
           "toy": toy}
