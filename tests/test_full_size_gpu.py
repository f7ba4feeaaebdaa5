"""Parity at the production sizes, on the kernels and tile shapes that run there.

* The batched workload: 64 independent grooms (strands log-uniform in [500, 20,000], 16-128
  vertices each, 26.4 M vertices) in one kami_vbd_batch_create handle, autotuned, stepped by one
  kami_vbd_batch_step of 2 steps (20 iterations, dt 1/120 s, head-sphere SDF 128^3).  Four whole
  grooms (the largest, the one with the longest strands, the smallest and one more) are compared with
  the FP32 oracle stepping that groom alone.
* One instance of the 80 M-vertex workload: 100,000 strands x 100 vertices, the 256^3 union of 12
  capsules, the head yawing +-30 deg at 1 Hz (a body transform per frame), 30 iterations, on the
  168-register C = 4 kernel that the autotuner picks there, over 2 frames.

Bars: positions within 1e-5 m and twist angles within 1e-5 rad against the FP32 oracle on the same
inputs and schedule (colour2); on the capsule body, for the strands the body does not touch, with a
statistical bar on the touched ones (see the test)."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle.oracle import OracleSim, twist_angles
from tests.helpers import POS_TOL, TWIST_TOL

pytestmark = pytest.mark.gpu

DT = 1 / 120


def _settings(num_itr, sdf):
    return dict(num_itr=num_itr, max_h=DT, gravity=(0.0, 0.0, -9.81), radius=40e-6, density=1300.0,
                velocity_decay=0.05, damping=1e-6, sdf=sdf)


def test_batched_64_grooms_full_size():
    from kamisimulator_b200.vbd import Solver

    grooms = synth.batched_grooms(64)
    st = _settings(20, synth.sphere_sdf(128, threshold=1e-3))
    b = Solver(grooms, form="fused", **st)
    tuned, _ = b.autotune(DT, trial_steps=4)  # restores the state and clock
    b.batch_step(DT, 2)
    x, _ = b.get_positions_velocities()
    q = b.get_orientations()
    sizes = [gg.num_vertices for gg in grooms]
    longest = [int(np.diff(gg.strand_begin).max()) for gg in grooms]
    sample = sorted({int(np.argmax(sizes)), int(np.argmax(longest)), int(np.argmin(sizes)), 17})
    worst = []
    for gi in sample:
        _, ns, v0, nv = b.groom_range(gi)
        assert ns == grooms[gi].num_strands and nv == grooms[gi].num_vertices
        o = OracleSim(grooms[gi], schedule="colour2", **st)
        o.advance(DT)
        o.advance(DT)
        ex = float(np.abs(x[v0:v0 + nv] - o.x).max())
        et = float(np.abs(twist_angles(o.q, q[v0:v0 + nv])).max())
        worst.append((gi, sizes[gi], ex, et))
        assert float(np.abs(o.x - grooms[gi].positions).max()) > 1e-4  # the strands moved
    b.close()
    print(f"\nbatched 64 grooms ({sum(sizes)} vertices, tuning {tuned}): " +
          ", ".join(f"groom {gi} ({n} v) {ex:.1e} m {et:.1e} rad" for gi, n, ex, et in worst))
    for gi, _, ex, et in worst:
        assert ex <= POS_TOL and et <= TWIST_TOL, (gi, ex, et)


def test_large_instance_with_a_yawing_capsule_body():
    """The body pass switches on where phi < 0, and its velocity fix (v -= ((v/|v|) . n) n,
    cudaSDFCollision.cu:258-265) then removes up to 1 m/s whatever |v| is.  A vertex the pass left on
    the capsules' surface decides the next frame's branch on a phi of rounding size, so on the strands
    the body touches, a different rounding can switch the fix on or off and move the next frame's
    positions by up to h x 1 m/s (8 mm).  On this instance about half of the 100,000 strands touch the
    capsules within the two frames, and the FP32 and FP64 oracles themselves differ by up to 3 mm on
    about a hundred of them.  The bars: every strand the body does not touch (found by the oracle
    without the body) within 1e-5 m / 1e-5 rad of the FP32 oracle; on the touched strands, 99 % within
    1e-5 m, and none beyond the velocity fix's reach."""
    from kamisimulator_b200.vbd import Solver

    rng = np.random.default_rng(11)
    g = synth.groom_strands(rng, np.full(100_000, 100))
    st = _settings(30, synth.capsule_union_sdf(256, num_capsules=12, radius_range=(0.02, 0.08)))
    s = Solver(g, form="fused", **st)
    s.set_tuning(4, 4, 1, 168)  # the kernel the autotuner picks for the 80 M-vertex batch
    assert s.get_tuning() == (4, 4, 1, 168)
    o32 = OracleSim(g, schedule="colour2", **st)
    o64 = OracleSim(g, schedule="colour2", dtype=np.float64, **st)
    free = OracleSim(g, schedule="colour2", **dict(st, sdf=None))
    for f in range(2):
        rot = synth.head_rotation(f * DT)
        s.set_body_transform(rot, (0.0, 0.0, 0.0))
        s.step(DT)
        for o in (o32, o64):
            o.set_body_transform(rot, (0.0, 0.0, 0.0))
            o.advance(DT)
        free.advance(DT)
    x, _ = s.get_positions_velocities()
    q = s.get_orientations()
    s.close()
    strand_of = np.repeat(np.arange(g.num_strands), np.diff(g.strand_begin))

    def per_strand(err):
        out = np.zeros(g.num_strands)
        np.maximum.at(out, strand_of, err)
        return out

    touched = per_strand(np.abs(o32.x - free.x).max(1)) > 0
    spread = per_strand(np.abs(o32.x - o64.x).max(1))
    ex = per_strand(np.abs(x - o32.x).max(1))
    et = per_strand(np.abs(twist_angles(o32.q, q)))
    ok = (ex <= POS_TOL) & (et <= TWIST_TOL)
    print(f"\n100,000 x 100, capsule SDF 256^3, yawing body, 2 frames: {int(touched.sum())} strands touched; "
          f"untouched: GPU {ex[~touched].max():.2e} m, {et[~touched].max():.2e} rad; touched: "
          f"{int((~ok[touched]).sum())} beyond 1e-5 (GPU up to {ex[touched].max():.2e} m; FP32 vs FP64 oracle "
          f"up to {spread.max():.2e} m, {int((spread > 1e-6).sum())} strands beyond 1e-6)")
    assert 0 < touched.sum() < g.num_strands
    assert ex[~touched].max() <= POS_TOL and et[~touched].max() <= TWIST_TOL
    assert ok[touched].mean() >= 0.99
    assert ex.max() <= DT * 1.0 + 1e-3
