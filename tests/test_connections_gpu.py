"""Connection springs (kami_vbd_desc::connection_index = Vertex::connectionIndex, YarnBall.h:56): the
stiffness-40 spring that cosseratItr adds to a tied vertex (YarnBall/sim/cosserat.cu:123-131), as
YarnBall sets it for glued endpoints (jsonBuilder.cpp:165-185) and the two ends of a closed curve
(reader.cpp:40-44).  Checked against the FP32 oracle (per step from shared states, both schedules)
and against the reference's own kernels built from source (Jacobi)."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle import oracle as orc
from oracle import ref_sim
from tests import helpers
from tests.helpers import POS_TOL, TWIST_TOL

pytestmark = pytest.mark.gpu


def _scene():
    """Four rods along +x from pinned roots 1 cm apart: the tips of rods 0 and 1 glued to each other,
    the tip of rod 2 tied both ways to the middle of rod 3, and rod 3's tip tied (one way) to its own
    root, a closed curve."""
    g = synth.cantilever(4, 16, young=2.0)
    conn = np.full(g.num_vertices, -1, np.int32)
    tip = [int(g.strand_begin[s + 1]) - 1 for s in range(4)]
    conn[tip[0]], conn[tip[1]] = tip[1], tip[0]
    mid3 = int(g.strand_begin[3]) + 8
    conn[tip[2]], conn[mid3] = mid3, tip[2]
    conn[tip[3]] = int(g.strand_begin[3])
    return g, conn


def _state_from(o):
    counter = np.array([int(o.clock[3])], np.uint32).view(np.float32)[0]
    return np.concatenate([o.x.ravel(), o.v.ravel(), o.v_last.ravel(), o.q.ravel(),
                           np.array([o.clock[0], o.clock[1], o.clock[2], counter], np.float32)]).astype(np.float32)


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_connection_springs_match_the_oracle(schedule):
    g, conn = _scene()
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, schedule=schedule)
    o = helpers.oracle_sim(g, dict(st, connection_index=conn), np.float32)
    free = helpers.oracle_sim(g, st, np.float32)
    s = helpers.gpu_solver(g, dict(st, connection_index=conn))
    worst_x = worst_t = effect = 0.0
    try:
        for f in range(12):
            if f > 0:
                s.set_state(_state_from(o))
                free.load_state(o.state())
            o.advance(1 / 120)
            free.advance(1 / 120)
            s.step(1 / 120)
            x, _ = s.get_positions_velocities()
            worst_x = max(worst_x, float(np.abs(x - o.x).max()))
            worst_t = max(worst_t, float(np.abs(orc.twist_angles(o.q, s.get_orientations())).max()))
            effect = max(effect, float(np.abs(free.x - o.x).max()))
    finally:
        s.close()
    assert effect > 1e-3  # the ties move the rods
    assert worst_x <= POS_TOL and worst_t <= TWIST_TOL, (worst_x, worst_t)


@pytest.mark.skipif(not ref_sim.available(), reason="oracle/_ref not built (needs the reference sources)")
def test_connection_springs_match_the_reference_kernels():
    """The reference's Jacobi kernels with the same connectionIndex against this solver's Jacobi sweep
    form and the oracle, per step from the reference's state.  The reference reads the partner's dx
    while other threads write it; two reference runs give its run-to-run spread."""
    g, conn = _scene()
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, schedule="jacobi")
    refs = [ref_sim.RefSim(g, young=2.0, num_itr=20, max_h=1 / 120) for _ in range(2)]
    for r in refs:
        r.set_connections(conn)
    o = helpers.oracle_sim(g, dict(st, connection_index=conn), np.float32)
    s = helpers.gpu_solver(g, dict(st, connection_index=conn))
    worst = dict(oracle=0.0, ours=0.0, spread=0.0, twist=0.0, moved=0.0)
    x_start = np.asarray(g.positions, np.float32)
    try:
        for _ in range(8):
            for r in refs:
                r.advance(1 / 120)
            o.advance(1 / 120)
            s.step(1 / 120)
            (x0, _, q0), (x1, _, _) = refs[0].download(), refs[1].download()
            xs, _ = s.get_positions_velocities()
            worst["spread"] = max(worst["spread"], float(np.abs(x0 - x1).max()))
            worst["oracle"] = max(worst["oracle"], float(np.abs(o.x - x0).max()))
            worst["ours"] = max(worst["ours"], float(np.abs(xs - x0).max()))
            worst["twist"] = max(worst["twist"], float(np.abs(orc.twist_angles(q0, s.get_orientations())).max()))
            worst["moved"] = max(worst["moved"], float(np.abs(x0 - x_start).max()))
    finally:
        for r in refs:
            r.close()
        s.close()
    print("connection reference pin", worst)
    assert worst["moved"] > 1e-3
    assert worst["oracle"] <= POS_TOL and worst["ours"] <= POS_TOL and worst["twist"] <= TWIST_TOL, worst


def test_connection_springs_take_the_sweep_form_and_are_refused_elsewhere():
    from kamisimulator_b200.vbd import KamiError

    g, conn = _scene()
    st = dict(num_itr=4, max_h=1 / 120, radius=40e-6, connection_index=conn)
    s = helpers.gpu_solver(g, st)  # AUTO
    try:
        with pytest.raises(KamiError, match="KAMI_ERR_UNSUPPORTED"):
            s.set_tuning(s.slots_per_lane + 2)  # the slot map of the ties is fixed
        with pytest.raises(KamiError, match="KAMI_ERR_UNSUPPORTED"):
            s.tape_reserve(1)  # the adjoint is the fused form's
    finally:
        s.close()
    with pytest.raises(KamiError, match="KAMI_ERR_UNSUPPORTED"):
        helpers.gpu_solver(g, st, form="fused")
    # a groom without ties keeps the fused form (whose colour2 steps can be recorded)
    plain = helpers.gpu_solver(g, dict(st, connection_index=np.full(g.num_vertices, -1, np.int32)))
    try:
        plain.tape_reserve(1)
    finally:
        plain.close()


def _tied_drape():
    """The soft strand falling onto the stiff one, the two middle vertices tied to each other: the
    spring pulls the crossing together, and the segments around the tie are exempt from contact
    (collision.cu:47-48) while the rest of the drape still lands on the bar."""
    g = synth.bar_and_drape(verts=16, gap=6e-5, bar_young=3e-5, drape_young=3e-5)
    conn = np.full(g.num_vertices, -1, np.int32)
    conn[8], conn[16 + 8] = 16 + 8, 8
    v0 = np.zeros((g.num_vertices, 3), np.float32)
    v0[16:, 2] = -0.02
    return g, conn, v0


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_connection_springs_with_hair_hair_contacts_match_the_oracle(schedule):
    g, conn, v0 = _tied_drape()
    st = dict(num_itr=10, max_h=1 / 120, gravity=(0.0, 0.0, -2.0), radius=2e-6, schedule=schedule, hair_hair=True,
              barrier_thickness=7.6e-5)
    o = helpers.oracle_sim(g, dict(st, connection_index=conn), np.float32, v0)
    untied = helpers.oracle_sim(g, st, np.float32, v0)
    s = helpers.gpu_solver(g, dict(st, connection_index=conn), form="sweep", velocities=v0)
    worst_x = worst_t = effect = 0.0
    try:
        for f in range(8):
            if f > 0:
                s.set_state(_state_from(o))
                untied.load_state(o.state())
            o.advance(1 / 120)
            untied.advance(1 / 120)
            s.step(1 / 120)
            x, _ = s.get_positions_velocities()
            worst_x = max(worst_x, float(np.abs(x - o.x).max()))
            worst_t = max(worst_t, float(np.abs(orc.twist_angles(o.q, s.get_orientations())).max()))
            effect = max(effect, float(np.abs(untied.x - o.x).max()))
    finally:
        s.close()
    assert effect > 1e-5  # the tie changes the motion
    assert worst_x <= POS_TOL and worst_t <= TWIST_TOL, (worst_x, worst_t)


@pytest.mark.skipif(not ref_sim.available(), reason="oracle/_ref not built (needs the reference sources)")
def test_connection_springs_with_hair_hair_contacts_match_the_reference_kernels():
    """The reference's own hair-hair kernels (its detection with the glued-pair exemption, the
    contact terms and the connection spring of cosseratItr) with the same connectionIndex, against
    this solver's Jacobi sweep form, per step from the oracle's state."""
    g, conn, v0 = _tied_drape()
    st = dict(num_itr=10, max_h=1 / 120, gravity=(0.0, 0.0, -2.0), radius=2e-6, schedule="jacobi", hair_hair=True,
              barrier_thickness=7.6e-5)
    o = helpers.oracle_sim(g, dict(st, connection_index=conn), np.float32, v0)
    s = helpers.gpu_solver(g, dict(st, connection_index=conn), form="sweep")
    refs = [ref_sim.RefSim(g, young=3e-5, radius=2e-6, num_itr=10, max_h=1 / 120, gravity=(0.0, 0.0, -2.0))
            for _ in range(2)]
    worst = dict(oracle=0.0, ours=0.0, spread=0.0, twist=0.0)
    try:
        for r in refs:
            r.set_connections(conn)
        for _ in range(6):
            state = (o.x.copy(), o.v.copy(), o.v_last.copy(), o.q.copy(), o.clock.copy())
            outs = []
            for r in refs:
                r.set_state(*state[:4], state[4][:3])
                assert r.step_hair_hair(1 / 120, 7.6e-5) == 0
                outs.append(r.download())
            s.set_state(_state_from(o))
            o.advance(1 / 120)
            s.step(1 / 120)
            (x0, _, q0), (x1, _, _) = outs
            xs, _ = s.get_positions_velocities()
            worst["spread"] = max(worst["spread"], float(np.abs(x0 - x1).max()))
            worst["oracle"] = max(worst["oracle"], float(np.abs(o.x - x0).max()))
            worst["ours"] = max(worst["ours"], float(np.abs(xs - x0).max()))
            worst["twist"] = max(worst["twist"], float(np.abs(orc.twist_angles(q0, s.get_orientations())).max()))
    finally:
        for r in refs:
            r.close()
        s.close()
    print("tied hair-hair reference pin", worst)
    assert worst["oracle"] <= POS_TOL and worst["ours"] <= POS_TOL and worst["twist"] <= TWIST_TOL, worst


def test_ties_in_a_batch_handle_are_per_groom():
    """connection_index holds each groom's own vertex indices: two tied grooms in one batch handle step
    as they do in two handles of their own, bit for bit."""
    from kamisimulator_b200.vbd import Solver

    g0, c0 = _scene()
    g1 = synth.cantilever(3, 12, young=3.0)
    c1 = np.full(g1.num_vertices, -1, np.int32)
    c1[11], c1[23] = 23, 11  # the tips of the first two rods
    st = dict(num_itr=12, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6)
    b = Solver([g0, g1], connection_index=[c0, c1], **st)
    s0 = Solver(g0, connection_index=c0, **st)
    s1 = Solver(g1, connection_index=c1, **st)
    try:
        for _ in range(5):
            b.step(1 / 120)
            s0.step(1 / 120)
            s1.step(1 / 120)
        xb = b.get_positions_velocities()[0]
        x0 = s0.get_positions_velocities()[0]
        x1 = s1.get_positions_velocities()[0]
    finally:
        for s in (b, s0, s1):
            s.close()
    np.testing.assert_array_equal(xb, np.concatenate([x0, x1]))
