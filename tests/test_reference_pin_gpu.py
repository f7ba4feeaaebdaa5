"""Pins against KamiSimulator's own code built from source (oracle/_ref/libkami_ref.so): the
reference's material set-up, its Jacobi step kernels and its SDF kernel, run live on the GPU and
compared with the CPU oracle and with this solver's CUDA kernels.

The reference's Jacobi kernels race at block boundaries, so their results vary from run to run;
each comparison is reported next to that run-to-run spread."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle import oracle as orc
from oracle import ref_sim
from tests import helpers
from tests.helpers import POS_TOL, TWIST_TOL

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_sim.available(), reason="oracle/_ref not built (needs the reference sources)")]


@pytest.mark.parametrize("case", ["cantilever", "groom"])
def test_material_matches_reference(case):
    if case == "cantilever":
        g, E = synth.cantilever(), 3.9
    else:
        g, E = synth.groom(300, 64, seed=2), 2.0
        g.strand_young[:] = E
    r = ref_sim.RefSim(g, young=E, num_itr=10, max_h=1 / 60)
    m = r.material()
    r.close()
    o = orc.configure(g, dtype=np.float32)
    np.testing.assert_array_equal(o["flags"], m["flags"])
    for k in ("inv_mass", "l_rest", "k_stretch", "q", "q_rest"):
        np.testing.assert_allclose(o[k], m[k], rtol=5e-7, atol=1e-7, err_msg=k)  # <= 4 ulp
    # this solver's own set-up (vbd_host.cpp), read back through the C ABI
    s = helpers.gpu_solver(g, dict(num_itr=10, max_h=1 / 60, radius=40e-6))
    np.testing.assert_allclose(s.get_orientations(), m["q"], rtol=5e-7, atol=1e-7)
    np.testing.assert_allclose(s.get_rest_darboux(), m["q_rest"], rtol=5e-7, atol=1e-7)
    s.close()


@pytest.mark.parametrize("form", ["fused", "sweep"])
def test_jacobi_step_matches_reference_kernels(form):
    """Reference Sim (racy Jacobi) vs the oracle's and this solver's Jacobi schedule, 6 steps of a
    300 x 64 groom cut with 20 iterations."""
    g = synth.groom(300, 64, seed=2)
    g.strand_young[:] = 2.0
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, schedule="jacobi")
    refs = [ref_sim.RefSim(g, young=2.0, num_itr=20, max_h=1 / 120) for _ in range(2)]
    o = helpers.oracle_sim(g, st, np.float32)
    s = helpers.gpu_solver(g, st, form=form)
    worst = dict(oracle=0.0, ours=0.0, spread=0.0, twist=0.0)
    for _ in range(6):
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
    for r in refs:
        r.close()
    s.close()
    print("reference pin", worst)
    assert worst["oracle"] <= POS_TOL and worst["ours"] <= POS_TOL and worst["twist"] <= TWIST_TOL, worst


def test_hair_hair_step_matches_reference_kernels():
    """The reference's own hair-hair kernels (buildCollisionList's distance test and list
    assembly, recomputeStepLimitKernel, cosseratItr's contact terms, in Sim::advance's order)
    against the oracle's and this solver's Jacobi schedule with contacts, one step at a time from
    shared states.  Two soft 16-vertex strands cross 60 um apart, the upper one pressing down.  The
    reference's detection runs over every segment pair: its LBVH cannot run as shipped (LBVH::compute
    reads d_flags[0] before sizing it, KittenGpuLBVH/lbvh.cu:366-370), and any broadphase that keeps
    the overlapping boxes hands the same pairs to the distance test."""
    g = synth.bar_and_drape(verts=16, gap=6e-5, bar_young=3e-5, drape_young=3e-5)
    v0 = np.zeros((g.num_vertices, 3), np.float32)
    v0[16:, 2] = -0.02
    st = dict(num_itr=10, max_h=1 / 120, gravity=(0.0, 0.0, -2.0), radius=2e-6, schedule="jacobi", hair_hair=True,
              barrier_thickness=7.6e-5)
    o = helpers.oracle_sim(g, st, np.float32, v0)
    free = helpers.oracle_sim(g, dict(st, hair_hair=False), np.float32, v0)
    s = helpers.gpu_solver(g, st, form="sweep")
    refs = [ref_sim.RefSim(g, young=3e-5, radius=2e-6, num_itr=10, max_h=1 / 120, gravity=(0.0, 0.0, -2.0))
            for _ in range(2)]
    worst = dict(oracle=0.0, ours=0.0, spread=0.0, twist=0.0, contact_effect=0.0)
    for _ in range(6):
        state = (o.x.copy(), o.v.copy(), o.v_last.copy(), o.q.copy(), o.clock.copy())
        outs = []
        for r in refs:
            r.set_state(*state[:4], state[4][:3])
            assert r.step_hair_hair(1 / 120, 7.6e-5) == 0  # no MAX_COLLISIONS_PER_SEGMENT overflow
            outs.append(r.download())
        counter = np.array([int(o.clock[3])], np.uint32).view(np.float32)[0]
        s.set_state(np.concatenate([a.ravel() for a in state[:4]] +
                                   [np.array([o.clock[0], o.clock[1], o.clock[2], counter], np.float32)]).astype(np.float32))
        free.load_state(o.state())
        o.advance(1 / 120)
        free.advance(1 / 120)
        s.step(1 / 120)
        (x0, _, q0), (x1, _, _) = outs
        xs, _ = s.get_positions_velocities()
        worst["spread"] = max(worst["spread"], float(np.abs(x0 - x1).max()))
        worst["oracle"] = max(worst["oracle"], float(np.abs(o.x - x0).max()))
        worst["ours"] = max(worst["ours"], float(np.abs(xs - x0).max()))
        worst["twist"] = max(worst["twist"], float(np.abs(orc.twist_angles(q0, s.get_orientations())).max()))
        worst["contact_effect"] = max(worst["contact_effect"], float(np.abs(free.x - o.x).max()))
    for r in refs:
        r.close()
    s.close()
    print("hair-hair reference pin", worst)
    assert worst["contact_effect"] > 3e-5  # the contacts move the strands in these steps
    assert worst["oracle"] <= POS_TOL and worst["ours"] <= POS_TOL and worst["twist"] <= TWIST_TOL, worst


def test_sdf_pass_matches_reference_kernel():
    rng = np.random.default_rng(4)
    for sdf, rot, tr in ((synth.sphere_sdf(64), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 0.0)),
                         (synth.capsule_union_sdf(40, num_capsules=6), synth.head_rotation(0.1), (0.02, 0.0, -0.01))):
        n_strands, per = 4000, 4
        p = rng.uniform(-0.25, 0.25, (n_strands * per, 3)).astype(np.float32)
        li = np.tile(np.arange(per), n_strands).astype(np.int32)
        rp, rv = ref_sim.sdf_project(p, np.zeros_like(p), li, sdf, rot, tr)
        # the same pass through the oracle and through this solver: a zero-iteration, zero-gravity step
        # leaves positions unchanged, then projects
        g = synth.Groom(np.arange(0, n_strands * per + 1, per, dtype=np.int32), p, np.ones(n_strands, np.float32),
                        np.ones(n_strands, np.float32))
        st = dict(num_itr=0, max_h=1.0, gravity=(0.0, 0.0, 0.0), radius=40e-6, sdf=sdf, pin_roots=False,
                  velocity_decay=0.0)
        o = helpers.oracle_sim(g, st, np.float32)
        o.set_body_transform(rot, tr)
        o.advance(1e-3)
        s = helpers.gpu_solver(g, st, form="fused")
        s.set_body_transform(rot, tr)
        s.step(1e-3)
        xs, _ = s.get_positions_velocities()
        s.close()
        assert np.mean(np.any(rp != p, axis=1)) > 0.01  # the pass really projected some particles
        assert float(np.abs(o.x - rp).max()) <= 1e-6
        assert float(np.abs(xs - rp).max()) <= 1e-6


def test_reference_gpu_speed_on_the_groom():
    """The reference's own CUDA Sim (Jacobi kernels, one CUDA graph per advance, error check per
    advance) against this solver on the 10,000 x 64 groom, 20 iterations, dt = max_h = 1/120, no SDF.
    Reported (pytest -s); the assertion only checks that the fused form is faster."""
    import time

    import torch

    g = synth.groom(10000, 64, seed=2)
    g.strand_young[:] = 2.0
    r = ref_sim.RefSim(g, young=2.0, num_itr=20, max_h=1 / 120)
    for _ in range(3):
        r.advance(1 / 120)
    n = 50
    t0 = time.perf_counter()
    for _ in range(n):
        r.advance(1 / 120)  # returns after the reference's own stream synchronisation
    ref_ms = (time.perf_counter() - t0) * 1e3 / n
    r.close()
    out = {"reference_ms_per_step": ref_ms,
           "reference_vertex_iters_per_s": g.num_vertices * 20 / (ref_ms * 1e-3)}
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6)
    for form, sched in (("fused", "jacobi"), ("fused", "colour2"), ("sweep", "jacobi")):
        s = helpers.gpu_solver(g, dict(st, schedule=sched), form=form)
        for _ in range(3):
            s.step(1 / 120)
        s.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            s.step(1 / 120)
        s.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / n
        out[f"ours_{form}_{sched}_ms_per_step"] = ms
        s.close()
    print("reference GPU speed", out)
    assert out["ours_fused_jacobi_ms_per_step"] < ref_ms


def test_batched_form_against_the_reference_per_groom_sims():
    """The batched form against the reference's own plain per-groom GPU form: the 64 uneven grooms of
    the batched workload (26.4 M vertices), each as one YarnBall::Sim built from the reference's
    source and stepped in turn (CantileverTestSolver's pattern, CantileverTestSolver.cpp:106-111),
    against one kami_vbd_batch_step handle over all of them.  Same settings on both sides: Jacobi, 20
    iterations, one substep of 1/120 s, no SDF (the reference's Sim has no SDF pass).  Prints the
    rates; the batched form must be at least 5x the reference's per-groom Sims."""
    import time

    from kamisimulator_b200.vbd import Solver

    grooms = synth.batched_grooms(seed=3)
    for g in grooms:
        g.strand_young[:] = 2.0
    nv = sum(g.num_vertices for g in grooms)
    refs = [ref_sim.RefSim(g, young=2.0, num_itr=20, max_h=1 / 120) for g in grooms]
    try:
        for r in refs:
            r.advance(1 / 120)
        frames = 3
        t0 = time.perf_counter()
        for _ in range(frames):
            for r in refs:
                r.advance(1 / 120)  # returns after the reference's own stream synchronisation
        ref_ms = (time.perf_counter() - t0) * 1e3 / frames
    finally:
        for r in refs:
            r.close()
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, schedule="jacobi")
    b = Solver(grooms, **st)
    try:
        b.autotune(1 / 120, trial_steps=4)
        b.batch_step(1 / 120, 4)
        b.synchronize()
        n = 24
        t0 = time.perf_counter()
        b.batch_step(1 / 120, n)
        b.synchronize()
        ours_ms = (time.perf_counter() - t0) * 1e3 / n
    finally:
        b.close()
    out = {"vertices": nv, "reference_per_groom_ms_per_frame": ref_ms, "batched_ms_per_frame": ours_ms,
           "reference_vertex_iters_per_s": nv * 20 / (ref_ms * 1e-3),
           "batched_vertex_iters_per_s": nv * 20 / (ours_ms * 1e-3), "ratio": ref_ms / ours_ms}
    print("batched vs the reference's per-groom Sims", out)
    assert out["ratio"] >= 5.0, out
