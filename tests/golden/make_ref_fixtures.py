"""Generates tests/golden/ref_pins.npz from KamiSimulator's own code built from source
(oracle/_ref/libkami_ref.so, see oracle/ref/Makefile).  Needs a CUDA device:

    python tests/golden/make_ref_fixtures.py [out.npz]

Contents (all produced by the reference, inputs from kamisimulator_b200.synth with fixed seeds):
  cant_*   : Sim::configure + setYoung material of the 64 x 32 cantilever (E 3.9 GPa)
  groom_*  : the same for a 100-strand x 64 cut of the groom (E 2 GPa for every strand)
  jsoft_*  : positions / orientations after each of 6 frames (1/60 s, 10 iterations) of 8 soft
             cantilever rods x 16 (E 1e-3 GPa), the reference's Jacobi kernels
  jgroom_* : the same for 3 frames (1/120 s, 20 iterations) of the 100 x 64 groom
  sdf_*    : one SDFHeadCollision pass over 2000 particles, sphere grid 32^3 and a rotated
             capsule-union grid 24^3
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from kamisimulator_b200 import synth  # noqa: E402
from oracle.ref_sim import RefSim, sdf_project  # noqa: E402


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "ref_pins.npz")
    d = {}
    g = synth.cantilever()
    r = RefSim(g, young=3.9, num_itr=10, max_h=1 / 60)
    for k, v in r.material().items():
        d["cant_" + k] = v
    r.close()
    g = synth.groom(100, 64, seed=2)
    r = RefSim(g, young=2.0, num_itr=20, max_h=1 / 120)
    for k, v in r.material().items():
        d["groom_" + k] = v
    xs, qs = [], []
    for _ in range(3):
        r.advance(1 / 120)
        x, _, q = r.download()
        xs.append(x)
        qs.append(q)
    d["jgroom_x"], d["jgroom_q"] = np.stack(xs), np.stack(qs)
    r.close()
    g = synth.cantilever(8, 16, young=1e-3)
    r = RefSim(g, young=1e-3, num_itr=10, max_h=1 / 60)
    xs, qs = [], []
    for _ in range(6):
        r.advance(1 / 60)
        x, _, q = r.download()
        xs.append(x)
        qs.append(q)
    d["jsoft_x"], d["jsoft_q"] = np.stack(xs), np.stack(qs)
    r.close()
    rng = np.random.default_rng(3)
    for name, sdf, rot, tr in (("sphere", synth.sphere_sdf(32), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 0.0)),
                               ("capsules", synth.capsule_union_sdf(24, num_capsules=5), synth.head_rotation(0.2),
                                (0.01, -0.02, 0.0))):
        n = 2000
        p = rng.uniform(-0.25, 0.25, (n, 3)).astype(np.float32)
        v = rng.normal(0.0, 0.5, (n, 3)).astype(np.float32)
        li = (np.arange(n) % 8).astype(np.int32)
        rp, rv = sdf_project(p, v, li, sdf, rot, tr)
        d[f"sdf_{name}_p"], d[f"sdf_{name}_v"], d[f"sdf_{name}_li"] = p, v, li
        d[f"sdf_{name}_pout"], d[f"sdf_{name}_vout"] = rp, rv
        d[f"sdf_{name}_rot"], d[f"sdf_{name}_tr"] = np.asarray(rot, np.float32), np.asarray(tr, np.float32)
    np.savez_compressed(out, **d)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
