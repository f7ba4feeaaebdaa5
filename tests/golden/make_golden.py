"""Regenerates the oracle's committed regression fixtures (run from the repository root):

    python tests/golden/make_golden.py

oracle_cantilever_f64.npz: 8 cantilever rods x 16 vertices (5 mm segments, radius 40 um, E = 1e-3 GPa,
bend deviation 0.1 so they sag visibly), gravity -z, 10 colour2 iterations, 12 frames of 1/60 s, FP64 oracle.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from kamisimulator_b200 import synth  # noqa: E402
from oracle import oracle as orc  # noqa: E402


def main():
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_cantilever_f64.npz")
    cfg = dict(num_rods=8, verts=16, num_itr=10, gravity=np.array([0.0, 0.0, -9.81]), radius=40e-6, young=1e-3,
               deviation=0.1, schedule="colour2", frames=12)
    g = synth.cantilever(cfg["num_rods"], cfg["verts"], young=cfg["young"])
    g.strand_dev[:] = cfg["deviation"]
    s = orc.OracleSim(g, num_itr=cfg["num_itr"], max_h=1 / 60, gravity=tuple(cfg["gravity"]), radius=cfg["radius"],
                      schedule=cfg["schedule"], dtype=np.float64)
    for _ in range(cfg["frames"]):
        s.advance(1 / 60)
    np.savez(out, x=s.x, q=s.q, **cfg)
    print("wrote", out, "tip z", s.x[cfg["verts"] - 1, 2])


if __name__ == "__main__":
    main()
