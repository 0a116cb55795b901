"""Generates the golden fixtures of this directory from the reference.

Run here, where the reference sources are mounted and oracle/_ref holds the
reference compiled from them (make -C oracle):

    python tests/golden/make_golden.py [REFERENCE_DIR]

(default: $MBS_REFERENCE_DIR, else the directory `reference` beside this
repository)

Fixtures (small, committed):
  extinction_reference.json  the reference's extinction known answers
                             (tests/extinction_reference.tsv of the reference:
                             bullet and droxtal, C_ext with 0.3 % tolerance) and
                             the run options of tests/run_extinction_reference.sh
  jones_kat.npz              the 64 Jones samples of the reference's
                             tests/test_mueller_direct.cpp and the Mueller
                             matrices its AddMuellerFromJones returns
  hex10x20_batch.npz         a traced batch (hexagonal column L=20 D=10 um,
                             m=1.3116, 3 Sobol orientations, seed 42)
  hex10x20_mueller.npz       the reference's CPU HandleBeamsToLocal Mueller
                             grid (and no-shadow grid, extinction) of that batch
                             on the grid 0-180 deg, 12 azimuth x 60 zenith steps
  concave_batch.npz / concave_mueller.npz
                             the same for the reference's CUDA release-gate
                             particle (concave, absorbing, cutoffs off),
                             2 orientations, grid 8 x 45
"""
from __future__ import annotations

import csv
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

GRIDS = {"hex10x20": (0.0, 180.0, 12, 60), "concave": (0.0, 180.0, 8, 45)}
N_ORIENT = {"hex10x20": 3, "concave": 2}


def kat_samples():
    """Inputs of the reference's tests/test_mueller_direct.cpp:9-24."""
    J, W = [], []
    for s in range(64):
        x = 0.125 * (s + 1)
        J.append([np.sin(x), np.cos(0.7 * x), np.cos(1.3 * x), -np.sin(0.4 * x),
                  -np.sin(0.9 * x), np.cos(1.1 * x), np.cos(0.6 * x), np.sin(1.7 * x)])
        W.append(0.03125 * (s + 1))
    return np.array(J), np.array(W)


def main(ref_root: str) -> None:
    import oracle
    from mbs_fast_b200 import beams as B
    from tests import common

    # extinction known answers
    rows = []
    with open(os.path.join(ref_root, "tests", "extinction_reference.tsv")) as f:
        lines = [ln for ln in f if not ln.startswith("#")]
    for r in csv.DictReader(lines, delimiter="\t"):
        rows.append({"case": r["case"], "type": int(r["type"]),
                     "p": [float(v) for v in (r["p1"], r["p2"]) if v != "-"],
                     "cext": float(r["reference_Cext"]), "qext": float(r["reference_Qext"]),
                     "area": float(r["reference_Aproj"]),
                     "rel_tol": float(r["relative_tolerance"])})
    run = {"ri": [1.3116, 0.0], "wavelength": 0.532, "max_reflections": 12,
           "euler_grid": [64, 32]}
    with open(os.path.join(HERE, "extinction_reference.json"), "w") as f:
        json.dump({"source": "reference tests/extinction_reference.tsv, "
                             "tests/run_extinction_reference.sh", "run": run, "cases": rows},
                  f, indent=1)

    # Jones -> Mueller known answers
    J, W = kat_samples()
    direct, _ = oracle.ref_jones_kat(J, W)
    np.savez_compressed(os.path.join(HERE, "jones_kat.npz"), jones=J, weight=W, mueller=direct)

    # traced batches and the reference's Mueller grids
    for key in ("hex10x20", "concave"):
        cfg = common.CASES[key]
        batch = common.sobol_batch(key, N_ORIENT[key])
        batch.save(os.path.join(HERE, f"{key}_batch.npz"))
        spec = GRIDS[key]
        M, Mns, cext, _ = oracle.ref_batch(cfg, spec, batch)
        np.savez_compressed(os.path.join(HERE, f"{key}_mueller.npz"), M=M, Mns=Mns, cext=cext,
                            grid=np.array(spec[:2]), n_az=spec[2], n_zen=spec[3])


if __name__ == "__main__":
    default = os.environ.get("MBS_REFERENCE_DIR") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference")
    main(sys.argv[1] if len(sys.argv) > 1 else default)
