"""Long trajectories: the 64 x 32 cantilever over 100 frames (10 iterations, dt 1/60 s, one substep
per frame) stepped free-running through the C ABI, against the FP32 oracle on the same inputs and
schedule at every frame (1e-5 m / 1e-5 rad), with the distance to the FP64 replay of the same update
(YarnBall/sim/step.cpp:38-62 over iteration.cu:8-74 and cosserat.cu:112-337) printed beside it."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle.oracle import OracleSim, twist_angles
from tests import helpers
from tests.helpers import POS_TOL, TWIST_TOL

pytestmark = pytest.mark.gpu

CANTILEVER = dict(num_itr=10, max_h=1 / 60, gravity=(0.0, 0.0, -9.81), radius=40e-6, density=1300.0,
                  velocity_decay=0.05, damping=1e-6)


@pytest.mark.parametrize("form", ["fused", "sweep"])
def test_cantilever_100_frames_against_the_fp32_and_fp64_oracles(form):
    g = synth.cantilever()
    dt = 1 / 60
    o32 = OracleSim(g, dtype=np.float32, schedule="colour2", **CANTILEVER)
    o64 = OracleSim(g, dtype=np.float64, schedule="colour2", **CANTILEVER)
    s = helpers.gpu_solver(g, dict(CANTILEVER, schedule="colour2"), form=form)
    worst32 = [0.0, 0.0]
    worst64 = [0.0, 0.0]
    try:
        for _ in range(100):
            s.step(dt)
            o32.advance(dt)
            o64.advance(dt)
            x, _ = s.get_positions_velocities()
            q = s.get_orientations()
            worst32 = [max(worst32[0], float(np.abs(x - o32.x).max())),
                       max(worst32[1], float(np.abs(twist_angles(o32.q, q)).max()))]
            worst64 = [max(worst64[0], float(np.abs(x - o64.x).max())),
                       max(worst64[1], float(np.abs(twist_angles(o64.q, q)).max()))]
    finally:
        s.close()
    print(f"\n{form}: 100 frames, max over frames: GPU vs FP32 oracle {worst32[0]:.2e} m / {worst32[1]:.2e} rad; "
          f"GPU vs FP64 replay {worst64[0]:.2e} m / {worst64[1]:.2e} rad; tip height {o64.x[31, 2]:.3e} m")
    assert worst32[0] <= POS_TOL and worst32[1] <= TWIST_TOL, worst32
    # the rods bend under gravity (setYoung's millimetre units make them stiff: the tips sag 52 um),
    # more than the position bar and a thousand times the error found
    sag = float(-o64.x[31::32, 2].min())
    assert sag > POS_TOL and sag > 1e3 * worst32[0]
    assert np.isfinite(worst64).all()
