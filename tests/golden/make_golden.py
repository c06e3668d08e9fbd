"""Generate the golden fixtures from the reference itself.

Runs oracle/_ref/ref_driver (the reference LBIBCell sources compiled by
oracle/Makefile, parity flags, OMP_NUM_THREADS=1) and stores:

* ``toy48.npz`` -- full state arrays of a 48x48 single-cell run at t = 0, 30, 60
  (1 species; remeshing happens at step 1).
* ``guo48.npz`` -- the toy48 run with the reference compiled with
  GuoZhengShi2002ForceModel as FluidSolver's base class (ref_driver_guo).
* ``config1_digest.json`` -- SHA-256 digests of every state array of the 200x200
  single-cell configuration at t = 0, 500, 1000, 1500, 2000.
* ``tissue4096_digest.json`` -- the same for the 4096x4096 tissue of 6000
  cells (3 species, tension, junctions, growth, division at 2x area) at
  t = 0, 10, 20.
* ``tissue1024_digest.json`` -- the same for the 1024x1024 tissue of 400 cells
  (2 species, tension, area regulator, cell junctions) at t = 0, 70, 80.  The
  reference's species re-initialisation divides 0 by 0 for nodes trapped
  between touching membranes (CDESolverD2Q5.cpp:156-228); NaN values are
  hashed as one canonical NaN, since x86 and CUDA give 0/0 different sign bits.

Usage (needs the reference sources, i.e. only in the build container):
    make -C oracle ref && python tests/golden/make_golden.py [toy48 config1 tissue1024]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lbibcell_b200 import configs  # noqa: E402
from oracle import oracle as O  # noqa: E402

FIELDS = ("f", "g", "vel", "force", "dom", "ctype", "ids", "node", "conn")


def toy48() -> configs.Config:
    return configs.toy(n=48, r=8.0, nodes=80, iterations=60, report_step=30, species=1)


def digest(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a)
    if a.dtype.kind == "f" and np.isnan(a).any():
        a = np.where(np.isnan(a), np.nan, a)
    return hashlib.sha256(a.tobytes()).hexdigest()


def tissue1024() -> configs.Config:
    return configs.config2(iterations=80, report_step=10)


def guo48() -> configs.Config:
    cfg = toy48()
    cfg.force_model = "GuoZhengShi2002ForceModel"
    return cfg


def tissue4096() -> configs.Config:
    return configs.config3(iterations=20, report_step=10)


def _digests(ref, times):
    dig = {}
    for t in times:
        st = ref[t]
        dig[str(t)] = {k: digest(getattr(st, k)) for k in FIELDS}
        dig[str(t)]["M"] = int(st.ids.shape[0])
        dig[str(t)]["iteration"] = int(st.current_iteration)
        dig[str(t)]["nonfinite_g"] = int((~np.isfinite(st.g)).sum())
    return dig


def main(cases) -> None:
    if "tissue4096" in cases:
        with tempfile.TemporaryDirectory() as tmp:
            paths = tissue4096().write(os.path.join(tmp, "t4096"))
            ref = O.run_reference(paths, os.path.join(tmp, "t4096", "ref"), timeout=6 * 3600)
            with open(os.path.join(HERE, "tissue4096_digest.json"), "w") as f:
                json.dump(_digests(ref, (0, 10, 20)), f, indent=1, sort_keys=True)
    if "tissue1024" in cases:
        with tempfile.TemporaryDirectory() as tmp:
            paths = tissue1024().write(os.path.join(tmp, "t1024"))
            ref = O.run_reference(paths, os.path.join(tmp, "t1024", "ref"), timeout=3600)
            with open(os.path.join(HERE, "tissue1024_digest.json"), "w") as f:
                json.dump(_digests(ref, (0, 70, 80)), f, indent=1, sort_keys=True)
    if "toy48" in cases:
        with tempfile.TemporaryDirectory() as tmp:
            cfg = toy48()
            paths = cfg.write(os.path.join(tmp, "toy"))
            ref = O.run_reference(paths, os.path.join(tmp, "toy", "ref"))
            out = {}
            for t in (0, 30, 60):
                st = ref[t]
                for k in FIELDS:
                    out[f"{k}_{t}"] = getattr(st, k)
                out[f"iter_{t}"] = np.array(st.current_iteration)
            np.savez_compressed(os.path.join(HERE, "toy48.npz"), **out)

    if "guo48" in cases:
        # the reference built with the Guo force model (oracle/Makefile, ref_driver_guo)
        with tempfile.TemporaryDirectory() as tmp:
            paths = guo48().write(os.path.join(tmp, "guo"))
            ref = O.run_reference(paths, os.path.join(tmp, "guo", "ref"), driver=O.REF_DRIVER_GUO)
            out = {}
            for t in (0, 30, 60):
                st = ref[t]
                for k in FIELDS:
                    out[f"{k}_{t}"] = getattr(st, k)
                out[f"iter_{t}"] = np.array(st.current_iteration)
            np.savez_compressed(os.path.join(HERE, "guo48.npz"), **out)

    if "config1" in cases:
        with tempfile.TemporaryDirectory() as tmp:
            paths = configs.config1().write(os.path.join(tmp, "c1"))
            ref = O.run_reference(paths, os.path.join(tmp, "c1", "ref"))
            dig = _digests(ref, (0, 500, 1000, 1500, 2000))
            for v in dig.values():
                del v["nonfinite_g"]
            with open(os.path.join(HERE, "config1_digest.json"), "w") as f:
                json.dump(dig, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["toy48", "guo48", "config1", "tissue1024", "tissue4096"])
