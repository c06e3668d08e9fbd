"""The drop-in C++ host layer (lbibcell_b200/dropin, libLbmLib.so): LBIBCell's
application API (SimulationRunner, GeometryHandler, Geometry, ForceSolver,
the BioBaseSolver name registry, ReportHandler and the vtk reporters,
Parameters, UtilLib's Log and lbm_fail) over the device runtime.

* The reference's apps/tutorial_01.cpp and tutorial_02.cpp compile unmodified
  against the drop-in headers (here, where the reference sources are); the
  builds in oracle/_ref/apps run on the GPU, and tutorial_01's VTK output
  equals, byte for byte, that of the same configuration run through the C
  ABI, whose tutorial_01 plugin set matches the reference build exactly
  (tests/test_tutorial_plugins.py).
* An application (tests/dropin/dropin_app.cpp) with a user bio solver that
  the device does not know (tests/dropin/user_plugin.cpp, compiled unchanged
  into the reference build too) runs the plugin on the host between device
  steps: every state array equals the reference build's at every report.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from lbibcell_b200 import configs

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "lbibcell_b200")
DROPIN_INC = os.path.join(PKG, "dropin", "include")


@pytest.fixture(scope="module")
def dropin_lib():
    from lbibcell_b200 import build
    build.build()
    return build.build_dropin()


def test_dropin_library_exports_the_api(dropin_lib):
    out = subprocess.run(["nm", "-DC", "--defined-only", dropin_lib], capture_output=True, text=True,
                         check=True).stdout
    for sym in ("LbmLib::SimulationRunner::runSimulation()", "LbmLib::SimulationRunner::addBioSolver(",
                "LbmLib::geometry::GeometryHandler::computeAreas() const",
                "LbmLib::geometry::Geometry::Geometry(", "LbmLib::solver::ForceSolver::addForce(",
                "UtilLib::Log::setStream(", "LbmLib::reportHandler::writeVtkBlock("):
        assert sym in out, sym


@pytest.mark.parametrize("app", ["tutorial_01", "tutorial_02"])
def test_reference_apps_compile_unmodified(dropin_lib, app):
    from oracle import oracle as O
    src = os.path.join(O.REFERENCE, "apps", app + ".cpp")
    if not os.path.exists(src):
        pytest.skip("reference sources not present")
    subprocess.run(["g++", "-std=gnu++11", "-fsyntax-only", "-I" + DROPIN_INC, src], check=True)


def _build_app(tmp_path):
    exe = str(tmp_path / "dropin_app")
    subprocess.run(["g++", "-std=gnu++11", "-O2", "-I" + DROPIN_INC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "dropin", "dropin_app.cpp"), os.path.join(HERE, "dropin", "user_plugin.cpp"),
                    "-L" + PKG, "-lLbmLib", "-llbibcuda", "-Wl,-rpath," + PKG, "-o", exe], check=True)
    return exe


def _needs_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


@pytest.mark.gpu
@pytest.mark.parametrize("bio", [["tutorial_01_BioSolverMembraneTension", "UserPullSolver"],
                                 ["LbibMembraneTension", "LbibAreaRegulator", "UserPullSolver"]])
def test_user_plugin_app_matches_reference_build(dropin_lib, oracle_mod, tmp_path, bio):
    """Device bio solvers first (in the step), the user plugin after each
    step on the host: dumps at t = 0, 10, 20, 30, 40 identical to the
    reference build's, which links the same plugin source."""
    _needs_gpu()
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference build not available")
    cfg = configs.toy(n=64, r=12.0, nodes=120, iterations=40, report_step=10, species=1)
    cfg.cells = [(1, configs.circle(32.0, 32.0, 12.0, 120, phase=0.1))]
    cfg.tension = (0.05, 5) if "LbibMembraneTension" in bio else None
    cfg.area = (1.1, 0.01, 0.004) if "LbibAreaRegulator" in bio else None
    cfg.bio = [b for b in bio if not b.startswith("Lbib")]
    paths = cfg.write(str(tmp_path / "cfg"))
    ref = oracle_mod.run_reference(paths, str(tmp_path / "ref"))
    exe = _build_app(tmp_path)
    out = tmp_path / "dropin"
    out.mkdir()
    env = dict(os.environ, LBIB_PLUGIN_FILE=paths["plugins"])
    r = subprocess.run([exe, paths["parameters"], paths["geometry"], paths["force"], paths["plugins"], str(out)],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    for t in (0, 10, 20, 30, 40):
        got = oracle_mod.read_dump(str(out / f"dump_{t}.bin"))
        want = ref[t]
        assert got.current_iteration == want.current_iteration, t
        for k in ("f", "g", "vel", "force", "dom", "ctype", "ids", "node", "conn"):
            a, b = getattr(got, k), getattr(want, k)
            assert a.shape == b.shape, (t, k)
            assert np.array_equal(a, b), (t, k, float(np.abs(a.astype(float) - b.astype(float)).max()))
    # the plugin did act: type-2 forces on the membrane at t = 40
    assert np.abs(ref[40].node[:, 4]).max() > 0


def _tutorial01_dir(tmp_path, lbib):
    """config/ for tutorial_01: parameters (64x64, 20 iterations, reports
    every 10), the geometry as the .vtm the app loads (one cell, written by
    the cell reporter) and the force file.  The cell (area ~314) stays below
    the division threshold (380): a larger one, divided at iteration 0 from
    the Float32 positions of the .vtm, makes the reference's cell division
    join two coincident nodes and fail (Connection.cpp:315-323), in the
    reference build as here."""
    run = tmp_path / "run"
    (run / "config" / "vtk").mkdir(parents=True)
    cfg = configs.toy(n=64, r=10.0, nodes=100, iterations=20, report_step=10, species=0)
    cfg.cells = [(1, configs.circle(32.0, 32.0, 10.0, 100, phase=0.1))]
    cfg.species = [configs.Species("tutorial_01_CDESolverD2Q5_SIGNAL", 2.0)]
    cfg.tau_fluid = 2.0
    cfg.area = None
    cfg.tension = None
    seed = cfg.write(str(tmp_path / "seed"))
    sim = lbib.Simulation(seed, lbib.FP64)
    sim.write_vtk(str(run / "config" / "vtk" / "Cells"), 0, 1)
    sim.close()
    shutil.copy(seed["parameters"], run / "config" / "tutorial_01_parameters.txt")
    shutil.copy(seed["force"], run / "config" / "force.txt")
    plugins = tmp_path / "plugins.txt"
    plugins.write_text("MassSolver\tMassSolverBoxOutlet\n" + "".join(
        f"BioSolver\t{n}\n" for n in ("tutorial_01_BioSolverAreaRegulator", "tutorial_01_BioSolverMembraneTension",
                                      "tutorial_01_BioSolverCellJunction", "tutorial_01_BioSolverDifferentiation",
                                      "tutorial_01_BioSolverCellDivision")))
    return run, str(plugins)


@pytest.mark.gpu
def test_tutorial_01_unmodified_runs_on_the_device(dropin_lib, oracle_mod, tmp_path):
    _needs_gpu()
    exe = os.path.join(oracle_mod.REF_APPS, "tutorial_01")
    if not os.path.exists(exe):
        pytest.skip("the reference's tutorial_01 was not built against the drop-in (oracle/Makefile apps)")
    from lbibcell_b200 import runner
    run, plugins = _tutorial01_dir(tmp_path, runner)
    r = subprocess.run([exe], cwd=str(run), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "error" not in r.stdout.lower(), r.stdout
    out = run / "output"
    # the same configuration through the C ABI: the reporters' blocks in
    # tutorial_01's order (cells, PNG (nothing), forces, CDE, fluid/4), under
    # the same relative prefix
    abi = tmp_path / "abi"
    (abi / "output").mkdir(parents=True)
    ref = abi / "output"
    paths = {"parameters": str(run / "config" / "tutorial_01_parameters.txt"),
             "geometry": str(run / "config" / "vtk" / "Cells_0.vtm"),
             "force": str(run / "config" / "force.txt"), "plugins": plugins}
    sim = runner.Simulation(paths, runner.FP64)
    cwd = os.getcwd()
    os.chdir(abi)
    try:
        for t in (0, 10, 20):
            if t:
                sim.step(10)
            for kind, coarse in ((1, 1), (5, 1), (2, 1), (3, 1), (4, 4)):
                sim.write_vtk("output/Cells", t, kind, coarse)
    finally:
        os.chdir(cwd)
        sim.close()
    compared = 0
    for dirpath, _, files in os.walk(ref):
        for fn in files:
            a = os.path.join(dirpath, fn)
            b = os.path.join(out, os.path.relpath(a, ref))
            assert os.path.exists(b), os.path.relpath(a, ref)
            assert open(a, "rb").read() == open(b, "rb").read(), os.path.relpath(a, ref)
            compared += 1
    assert compared >= 3 * 5
    assert (out / "log.txt").exists()
