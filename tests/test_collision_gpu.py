"""Hair-hair collision (EnableHairHairColl) on the GPU against the FP32 oracle: contact detection,
the IPC barrier + friction terms of the position sweep and the step limit (YarnBall/sim/
collision.cu, cosserat.cu:163-227).  Bars as for the plain step: per step, positions within
1e-5 m and twist angles within 1e-5 rad, from shared states."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle.oracle import twist_angles
from tests import helpers
from tests.helpers import POS_TOL, TWIST_TOL

pytestmark = pytest.mark.gpu

# StableCosseratRodsSolver at CurveRadius 4e-5: radius 0.05 CR, barrier 2 (1 - 0.05) CR (.cpp:176-180)
COLL = dict(radius=2e-6, barrier_thickness=7.6e-5)


def _settings(schedule="colour2", hair_hair=True, num_itr=10, **kw):
    st = dict(num_itr=num_itr, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), schedule=schedule, hair_hair=hair_hair,
              **COLL)
    st.update(kw)
    return st


def _gpu_state_from(o):
    counter = np.array([int(o.clock[3])], np.uint32).view(np.float32)[0]
    return np.concatenate([o.x.ravel(), o.v.ravel(), o.v_last.ravel(), o.q.ravel(),
                           np.array([o.clock[0], o.clock[1], o.clock[2], counter], np.float32)]).astype(np.float32)


def _lockstep(groom, st, frames, dt=1 / 120, velocities=None):
    """Oracle and GPU from the same state every frame; returns the worst position / twist error."""
    o = helpers.oracle_sim(groom, st, np.float32, velocities)
    g = helpers.gpu_solver(groom, st, form="sweep", velocities=velocities)
    worst_x = worst_t = 0.0
    try:
        for f in range(frames):
            if f > 0:
                g.set_state(_gpu_state_from(o))
            o.advance(dt)
            g.step(dt)
            x, _ = g.get_positions_velocities()
            ex = float(np.abs(x - o.x).max())
            et = float(np.abs(twist_angles(o.q, g.get_orientations())).max())
            worst_x, worst_t = max(worst_x, ex), max(worst_t, et)
        xs = g.get_positions_velocities()[0]
    finally:
        g.close()
    return worst_x, worst_t, xs, o.x.copy()


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_drape_rests_on_the_bar(schedule):
    g = synth.bar_and_drape(drape_young=3e-5)
    ex, et, x, _ = _lockstep(g, _settings(schedule), 40)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)
    nv = 25
    drape, bar = x[nv:], x[:nv]
    mid = int(np.argmin(np.abs(drape[:, 1])))
    # the soft strand lies on the bar, a barrier's width above it ...
    assert drape[mid, 2] - bar[12, 2] > 2 * COLL["radius"]
    # ... where without contacts it falls through
    free = helpers.gpu_solver(g, _settings(schedule, hair_hair=False), form="sweep")
    for _ in range(40):
        free.step(1 / 120)
    xf = free.get_positions_velocities()[0]
    free.close()
    assert xf[nv + mid, 2] - xf[12, 2] < -1e-3


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_tangle_matches_the_oracle(schedule):
    """12 strands falling onto each other: crossing contacts, friction, the step limit."""
    g = synth.tangle(12, 24, seed=3, young=5e-5, layer=1e-4)
    ex, et, x, _ = _lockstep(g, _settings(schedule), 12)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)
    free = helpers.gpu_solver(g, _settings(schedule, hair_hair=False), form="sweep")
    for _ in range(12):
        free.step(1 / 120)
    xf = free.get_positions_velocities()[0]
    free.close()
    assert np.abs(xf - x).max() > 1e-4  # the contacts changed the motion


def test_long_strands_with_contacts_match_the_oracle():
    """Strands of 600 vertices piling onto each other: sweep tiles of 640 slots, so one block of
    320 threads per tile runs each iteration."""
    g = synth.tangle(6, 600, seed=7, young=5e-5, layer=1e-4)
    st = _settings("colour2")
    s = helpers.gpu_solver(g, st, form="sweep")
    assert 16 < s.slots_per_lane <= 32
    s.close()
    ex, et, x, _ = _lockstep(g, st, 12)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)
    free = helpers.gpu_solver(g, _settings("colour2", hair_hair=False), form="sweep")
    for _ in range(12):
        free.step(1 / 120)
    xf = free.get_positions_velocities()[0]
    free.close()
    assert np.abs(xf - x).max() > 1e-4  # the contacts changed the motion (5e-4 m in the oracle)


def test_substeps_and_detection_period():
    """Two substeps per frame and detection on every second substep (the lists of the first
    substep carry over): per frame from shared states, then free running.  Free running, a contact
    found by one side and missed by the other at the detection threshold splits the FP32
    trajectories, so that check is at 1e-4 m."""
    g = synth.tangle(12, 20, seed=5, young=5e-5, layer=1e-4)
    st = _settings("colour2", max_h=1 / 240, detection_period=2)
    ex, et, _, _ = _lockstep(g, st, 8)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)
    o = helpers.oracle_sim(g, st, np.float32)
    s = helpers.gpu_solver(g, st, form="sweep")
    for _ in range(6):
        o.advance(1 / 120)
        s.step(1 / 120)
    x = s.get_positions_velocities()[0]
    s.close()
    assert np.abs(x - o.x).max() <= 1e-4


def test_more_than_16_contacts_is_reported():
    g = synth.contact_fence()
    st = _settings("colour2", num_itr=4)
    o = helpers.oracle_sim(g, st, np.float32)
    with pytest.raises(RuntimeError, match="16 contacts"):
        o.advance(1 / 120)
    from kamisimulator_b200.vbd import KamiError

    s = helpers.gpu_solver(g, st, form="sweep")
    s.step(1 / 120)
    with pytest.raises(KamiError, match="KAMI_ERR_CONTACTS"):
        s.get_positions_velocities()
    s.close()


def test_checkpoint_replay_with_contacts():
    g = synth.tangle(12, 20, seed=7, young=5e-5, layer=1e-4)
    s = helpers.gpu_solver(g, _settings("colour2"), form="sweep")
    for _ in range(3):
        s.step(1 / 120)
    snap = s.get_state()
    for _ in range(3):
        s.step(1 / 120)
    a = s.get_state()
    s.set_state(snap)
    for _ in range(3):
        s.step(1 / 120)
    np.testing.assert_array_equal(s.get_state(), a)
    s.close()


def test_grooms_of_a_batch_do_not_collide_with_each_other():
    """Two overlapping tangles in one batch handle step as two separate handles (each reference
    Sim detects only its own strands), while one handle over the concatenated strands sees the
    contacts between them."""
    from kamisimulator_b200.vbd import Solver

    g0 = synth.tangle(12, 20, seed=8, young=5e-5, layer=1e-4)
    g1 = synth.tangle(12, 20, seed=9, young=5e-5, layer=1e-4)
    g1.positions[:, 2] += 5e-5  # strands of equal height would cross at distance 0 (a 0/0 contact normal)
    st = _settings("colour2")
    b = Solver([g0, g1], form="sweep", **st)
    singles = [Solver(gg, form="sweep", **st) for gg in (g0, g1)]
    joined = Solver(synth.concat_grooms([g0, g1]), form="sweep", **st)
    for _ in range(4):
        b.step(1 / 120)
        joined.step(1 / 120)
        for s in singles:
            s.step(1 / 120)
    xb = b.get_positions_velocities()[0]
    xs = np.concatenate([s.get_positions_velocities()[0] for s in singles])
    xj = joined.get_positions_velocities()[0]
    for s in singles + [b, joined]:
        s.close()
    assert np.abs(xb - xs).max() <= 1e-6
    assert np.abs(xj - xs).max() > 1e-5


def test_ill_conditioned_tangle_within_the_fp32_spread():
    """24 soft strands piling up: the barrier amplifies rounding, and the FP32 oracle itself moves
    up to ~1.5e-5 m per step away from the FP64 one.  The GPU must stay within 3x that spread of
    the FP32 oracle, frame by frame from the FP64 state."""
    g = synth.tangle(24, 24, seed=3, young=3e-5, layer=1e-4)
    st = _settings("colour2")
    o64 = helpers.oracle_sim(g, st, np.float64)
    o32 = helpers.oracle_sim(g, st, np.float32)
    s = helpers.gpu_solver(g, st, form="sweep")
    worst_gpu = worst_fp32 = 0.0
    for f in range(12):
        for a in ("x", "v", "v_last", "q"):
            getattr(o32, a)[...] = getattr(o64, a)
        o32.clock[...] = o64.clock
        s.set_state(_gpu_state_from(o32))
        o64.advance(1 / 120)
        o32.advance(1 / 120)
        s.step(1 / 120)
        x = s.get_positions_velocities()[0]
        worst_gpu = max(worst_gpu, float(np.abs(x - o32.x).max()))
        worst_fp32 = max(worst_fp32, float(np.abs(o32.x - o64.x).max()))
    s.close()
    assert worst_fp32 > POS_TOL / 10  # the scene is as ill-conditioned as intended
    assert worst_gpu <= max(POS_TOL, 3 * worst_fp32), (worst_gpu, worst_fp32)
