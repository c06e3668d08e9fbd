"""Generate the golden fixtures from the reference itself.

Runs oracle/_ref/ref_driver (the reference LBIBCell sources compiled by
oracle/Makefile, parity flags, OMP_NUM_THREADS=1) and stores:

* ``toy48.npz`` -- full state arrays of a 48x48 single-cell run at t = 0, 30, 60
  (1 species; remeshing happens at step 1).
* ``config1_digest.json`` -- SHA-256 digests of every state array of the 200x200
  single-cell configuration at t = 0, 500, 1000, 1500, 2000.

Usage (needs the reference sources, i.e. only in the build container):
    make -C oracle ref && python tests/golden/make_golden.py
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
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
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

        cfg = configs.config1()
        paths = cfg.write(os.path.join(tmp, "c1"))
        ref = O.run_reference(paths, os.path.join(tmp, "c1", "ref"))
        dig = {}
        for t in (0, 500, 1000, 1500, 2000):
            st = ref[t]
            dig[str(t)] = {k: digest(getattr(st, k)) for k in FIELDS}
            dig[str(t)]["M"] = int(st.ids.shape[0])
            dig[str(t)]["iteration"] = int(st.current_iteration)
        with open(os.path.join(HERE, "config1_digest.json"), "w") as f:
            json.dump(dig, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
