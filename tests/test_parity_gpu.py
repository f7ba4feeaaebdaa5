"""GPU parity: the CUDA solver (through the C ABI) against the FP32 oracle on the same inputs and
schedule.  Bars (per step): positions within 1e-5 m, twist angles within 1e-5 rad."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle.oracle import twist_angles
from tests import helpers
from tests.helpers import POS_TOL, TWIST_TOL

pytestmark = pytest.mark.gpu


def _lockstep(groom, settings, form, frames, dt, velocities=None, reseed_each_frame=False, body=None):
    """Steps oracle and GPU side by side; returns the max position / twist error over all frames."""
    o = helpers.oracle_sim(groom, settings, np.float32, velocities)
    g = helpers.gpu_solver(groom, settings, form=form, velocities=velocities)
    worst_x, worst_t = 0.0, 0.0
    try:
        for f in range(frames):
            if body is not None:
                rot, tr = body(f)
                o.set_body_transform(rot, tr)
                g.set_body_transform(rot, tr)
            if reseed_each_frame and f > 0:
                st = np.concatenate([o.x.ravel(), o.v.ravel(), o.v_last.ravel(), o.q.ravel(),
                                     np.array([o.clock[0], o.clock[1], o.clock[2], 0.0], np.float32)])
                g.set_state(st.astype(np.float32))
            o.advance(dt)
            g.step(dt)
            x, v = g.get_positions_velocities()
            q = g.get_orientations()
            ex = float(np.abs(x - o.x).max())
            et = float(np.abs(twist_angles(o.q, q)).max())
            worst_x, worst_t = max(worst_x, ex), max(worst_t, et)
            assert np.isfinite(x).all()
    finally:
        g.close()
    return worst_x, worst_t


@pytest.mark.parametrize("form", ["fused", "sweep"])
@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_cantilever(form, schedule):
    g = synth.cantilever()
    st = dict(num_itr=10, max_h=1 / 60, gravity=(0.0, 0.0, -9.81), radius=40e-6, schedule=schedule)
    ex, et = _lockstep(g, st, form, 10, 1 / 60)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)


@pytest.mark.parametrize("form", ["fused", "sweep"])
def test_soft_uneven_strands_with_sdf_wind_substeps(form):
    """Uneven strands (several per tile), large motion, wind, the SDF pass and 3 substeps."""
    g = helpers.soft_groom(120, (4, 60), seed=21)
    v = helpers.random_velocities(g, 0.3, seed=3)
    sdf = synth.sphere_sdf(64, radius=0.09, half_extent=0.2, threshold=2e-3)
    st = helpers.soft_settings(schedule="colour2", max_h=1 / 180, num_itr=5, sdf=sdf,
                               wind=(2.0, 1.0, 0.7, 0.4, 3.0))
    ex, et = _lockstep(g, st, form, 8, 1 / 60, velocities=v, reseed_each_frame=True)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)


@pytest.mark.parametrize("form", ["fused", "sweep"])
def test_soft_uneven_strands_jacobi(form):
    """The Jacobi schedule on soft uneven strands, per step from shared states.  Jacobi is the
    reference's intended order but its twist is ill-conditioned: with substeps these strands blow
    up in FP64 too, and after ~5 frames even one step amplifies rounding past 1e-5 rad, so the
    check covers the first 4 single-substep frames."""
    g = helpers.soft_groom(120, (4, 60), seed=21, young_scale=1e-2)
    v = helpers.random_velocities(g, 0.1, seed=3)
    sdf = synth.sphere_sdf(64, radius=0.09, half_extent=0.2, threshold=2e-3)
    st = helpers.soft_settings(schedule="jacobi", max_h=1 / 60, num_itr=5, sdf=sdf, wind=(2.0, 1.0, 0.7, 0.4, 3.0))
    ex, et = _lockstep(g, st, form, 4, 1 / 60, velocities=v, reseed_each_frame=True)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)


@pytest.mark.parametrize("form", ["fused", "sweep"])
@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_groom_cut_with_head_sdf_per_step(form, schedule):
    """A 400-strand cut of the 10,000 x 64 groom with the 128^3 head sphere, 20 iterations, under the
    production schedule (colour2) and the reference kernels' own order (jacobi)."""
    g = synth.groom(400, 64, seed=2)
    sdf = synth.sphere_sdf(128)
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, sdf=sdf, schedule=schedule)
    ex, et = _lockstep(g, st, form, 6, 1 / 120, reseed_each_frame=True)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)


def test_rotating_body():
    g = helpers.soft_groom(60, (10, 50), seed=8)
    sdf = synth.capsule_union_sdf(48, num_capsules=4, half_extent=0.3, threshold=1e-3)
    st = helpers.soft_settings(sdf=sdf, num_itr=8)
    ex, et = _lockstep(g, st, "fused", 6, 1 / 60, reseed_each_frame=True,
                       body=lambda f: (synth.head_rotation(f / 60.0), (0.01 * f, 0.0, 0.0)))
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)


@pytest.mark.parametrize("form", ["auto", "sweep"])
def test_long_strands(form):
    """Strands longer than a tile of 128 slots: the fused form takes groups of tiles (auto), the sweep
    form wider tiles."""
    g = helpers.soft_groom(20, (150, 250), seed=5)
    st = helpers.soft_settings(num_itr=4)
    s = helpers.gpu_solver(g, st, form=form)
    assert s.slots_per_lane == 4 if form == "auto" else s.slots_per_lane >= 6
    s.close()
    ex, et = _lockstep(g, st, form, 4, 1 / 60, reseed_each_frame=True)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)


def test_fused_and_sweep_agree_at_full_groom_size():
    """Size-independent check at the full 10,000 x 64 groom: the two kernel forms agree."""
    g = synth.groom()
    sdf = synth.sphere_sdf(128)
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, sdf=sdf)
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="sweep")
    for _ in range(3):
        a.step(1 / 120)
        b.step(1 / 120)
    xa, _ = a.get_positions_velocities()
    xb, _ = b.get_positions_velocities()
    qa, qb = a.get_orientations(), b.get_orientations()
    assert np.abs(xa - xb).max() <= POS_TOL
    assert np.abs(twist_angles(qa, qb)).max() <= TWIST_TOL
    np.testing.assert_allclose(np.linalg.norm(qa, axis=1), 1.0, atol=1e-5)
    # roots are pinned and skipped by the SDF pass: they do not move
    roots = g.strand_begin[:-1]
    np.testing.assert_array_equal(xa[roots], g.positions[roots])
    a.close()
    b.close()


def test_full_groom_one_step_against_oracle():
    g = synth.groom()
    sdf = synth.sphere_sdf(128)
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, sdf=sdf)
    ex, et = _lockstep(g, st, "fused", 1, 1 / 120)
    assert ex <= POS_TOL and et <= TWIST_TOL, (ex, et)


def test_deterministic_replay():
    g = synth.groom(500, 64)
    st = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, sdf=synth.sphere_sdf(64))
    outs = []
    for _ in range(2):
        s = helpers.gpu_solver(g, st, form="fused")
        for _ in range(3):
            s.step(1 / 120)
        outs.append(s.get_positions_velocities()[0])
        s.close()
    np.testing.assert_array_equal(outs[0], outs[1])


def test_state_checkpoint_resume():
    g = helpers.soft_groom(50, (6, 40))
    st = helpers.soft_settings()
    s = helpers.gpu_solver(g, st)
    s.step(1 / 60)
    snap = s.get_state()
    s.step(1 / 60)
    s.step(1 / 60)
    x1 = s.get_positions_velocities()[0].copy()
    s.set_state(snap)
    s.step(1 / 60)
    s.step(1 / 60)
    x2 = s.get_positions_velocities()[0]
    np.testing.assert_array_equal(x1, x2)
    s.close()


def test_host_and_device_boundary_copies():
    import torch

    g = helpers.soft_groom(30, (6, 30))
    s = helpers.gpu_solver(g, helpers.soft_settings())
    x0 = g.positions + 0.01
    v0 = np.full_like(g.positions, 0.25)
    s.set_positions_velocities(x0, v0)
    x, v = s.get_positions_velocities()
    np.testing.assert_array_equal(x, x0)
    np.testing.assert_array_equal(v, v0)
    xd = torch.zeros((g.num_vertices, 3), dtype=torch.float32, device="cuda")
    vd = torch.zeros_like(xd)
    s.get_positions_velocities(xd, vd)
    np.testing.assert_array_equal(xd.cpu().numpy(), x0)
    xd2 = xd * 2
    torch.cuda.synchronize()
    s.set_positions_velocities(xd2, vd)
    np.testing.assert_array_equal(s.get_positions_velocities()[0], 2 * x0.astype(np.float32))
    s.close()


def test_nonfinite_input_raises_status():
    from kamisimulator_b200.vbd import KamiError

    g = helpers.soft_groom(30, (6, 30))
    s = helpers.gpu_solver(g, helpers.soft_settings())
    snap = s.get_state()
    x = g.positions.copy()
    x[5] = np.nan
    s.set_positions_velocities(x, None)
    s.step(1 / 60)
    with pytest.raises(KamiError) as ei:
        s.get_positions_velocities()
    assert ei.value.status == 4
    # the status word is cleared once reported; a restored state steps cleanly again
    s.set_state(snap)
    s.step(1 / 60)
    s.get_positions_velocities()
    s.close()


@pytest.mark.parametrize("form,tuning,schedule", [
    ("sweep", None, "colour2"), ("fused", None, "colour2"), ("fused", (2, 4, 8, 120), "colour2"),
    ("fused", (4, 4, 8, 1), "colour2"), ("fused", (4, 4, 8, 2), "colour2"), ("fused", (4, 4, 8, 1), "jacobi"),
    ("fused", (4, 4, 8, 168), "colour2"), ("fused", (4, 2, 8, 168), "jacobi"),
    ("fused", (2, 4, 8, 120), "jacobi")])
@pytest.mark.parametrize("pin_roots", [True, False])
def test_nonfinite_strand_does_not_leak(form, tuning, schedule, pin_roots):
    """A strand that turns non-finite leaves every other strand untouched (bit for bit), as the
    reference's per-vertex flag tests guarantee; strands are packed several per tile here, and with
    4 slots per lane several per lane, for every kernel variant."""
    from kamisimulator_b200.vbd import KamiError

    g = helpers.soft_groom(64, (5, 30), seed=17)
    st = helpers.soft_settings(pin_roots=pin_roots, schedule=schedule)
    clean = helpers.gpu_solver(g, st, form=form)
    bad = helpers.gpu_solver(g, st, form=form)
    if tuning is not None:
        clean.set_tuning(*tuning)
        bad.set_tuning(*tuning)
    victim = 10
    a, b = g.strand_begin[victim], g.strand_begin[victim + 1]
    x = g.positions.copy()
    x[(a + b) // 2] = np.nan
    bad.set_positions_velocities(x, None)
    for _ in range(3):
        clean.step(1 / 60)
        bad.step(1 / 60)
    xc, _ = clean.get_positions_velocities()
    with pytest.raises(KamiError):
        bad.get_positions_velocities()
    xb = bad.split_state(bad.get_state())["x"]
    keep = np.ones(g.num_vertices, bool)
    keep[a:b] = False
    np.testing.assert_array_equal(xb[keep], xc[keep])
    assert not np.isfinite(xb[a:b]).all()
    clean.close()
    bad.close()


def test_fp32_peak_probe():
    """kami_fp32_peak (the bench-only probe library): the FFMA / FFMA2 chain throughput that bench.py
    divides the fused step's FP32 rate by is a plausible B200 figure (nominal FP32: 74 TFLOP/s at
    1965 MHz)."""
    import bench

    fma, fma2 = bench.fp32_probe(0)
    assert 30.0 < fma < 150.0, fma
    assert 30.0 < fma2 < 300.0, fma2


def test_stepping_calls_check_dt():
    """Every stepping entry point rejects a dt that is not finite or that needs more than
    KAMI_MAX_SUBSTEPS (10^6) substeps of max_h, before it converts the substep count to an integer;
    dt <= 0 is a no-op for kami_vbd_step (Sim::advance returns for h <= 0)."""
    from kamisimulator_b200.vbd import KamiError

    g = synth.cantilever(4, 8)
    st = dict(num_itr=4, max_h=1e-9, gravity=(0.0, 0.0, -9.81), radius=40e-6)
    s = helpers.gpu_solver(g, st, form="fused")
    x0, _ = s.get_positions_velocities()
    s.set_hair_layout(g.num_strands, 8)
    hx = np.zeros((g.num_strands, 8, 3), np.float32)
    for dt in (float("nan"), float("inf"), 1.0):  # 1 s / 1 ns is 10^9 substeps
        for call in (lambda: s.step(dt), lambda: s.step_n(dt, 2), lambda: s.step_host(dt, x0.copy(), x0.copy()),
                     lambda: s.step_hair(dt, hx, hx, hx, hx)):
            with pytest.raises(KamiError, match="INVALID_ARGUMENT"):
                call()
    s.step(-1.0)
    s.step(0.0)
    np.testing.assert_array_equal(s.get_positions_velocities()[0], x0)
    with pytest.raises(KamiError, match="INVALID_ARGUMENT"):
        s.set_launch_mode(7)
    s.close()
