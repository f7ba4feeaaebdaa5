"""Strands longer than one warp tile on the fused form: groups of 2-8 tiles, one CTA of as many warps
per group, a strand running on from lane 31 of one tile into lane 0 of the next (KamiSimulator's
default resampling to 1 mm segments gives strands of hundreds of vertices)."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle.oracle import twist_angles
from tests import helpers
from tests.test_parity_gpu import _lockstep

pytestmark = pytest.mark.gpu


def _settings(schedule="colour2", **kw):
    st = dict(num_itr=10, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, schedule=schedule,
              sdf=synth.sphere_sdf(64, threshold=2e-3))
    st.update(kw)
    return st


def _mixed(seed=5):
    # lengths 20-450: single tiles, and groups of 2 and 4 tiles of 128 slots
    rng = np.random.default_rng(seed)
    return synth.groom_strands(rng, rng.integers(20, 451, 160))


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_long_strands_fused_match_the_oracle(schedule):
    g = _mixed()
    st = _settings(schedule)
    s = helpers.gpu_solver(g, st, form="auto")
    assert s.slots_per_lane == 4  # the fused form in groups of tiles (the sweep form would take C = 16)
    s.close()
    ex, et = _lockstep(g, st, "auto", 6, 1 / 120, reseed_each_frame=True)
    assert ex <= helpers.POS_TOL and et <= helpers.TWIST_TOL, (ex, et)


@pytest.mark.parametrize("tuning", [(4, 1, 8, 168), (2, 1, 8, 1), (2, 1, 8, 120)])
def test_long_strand_variants_and_sweep_form_agree(tuning):
    g = _mixed(seed=6)
    st = _settings()
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="fused")
    b.set_tuning(*tuning)
    assert b.get_tuning()[0] == tuning[0]
    c = helpers.gpu_solver(g, st, form="sweep")
    assert c.slots_per_lane > 4  # the sweep form holds a strand in one tile
    for _ in range(4):
        for s in (a, b, c):
            s.step(1 / 120)
    xa, xb, xc = (s.get_positions_velocities()[0] for s in (a, b, c))
    assert np.abs(xa - xb).max() <= 1e-6
    assert np.abs(xa - xc).max() <= 1e-6
    assert np.abs(twist_angles(a.get_orientations(), b.get_orientations())).max() <= helpers.TWIST_TOL
    for s in (a, b, c):
        s.close()


def test_long_strands_step_n_and_host_frames():
    g = _mixed(seed=7)
    st = _settings()
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="fused")
    frames = 6
    bt = np.array([list(synth.head_rotation(f / 120.0)) + [0.001 * f, 0.0, 0.0] for f in range(frames)], np.float32)
    for f in range(frames):
        a.set_body_transform(bt[f, :4], bt[f, 4:])
        a.step(1 / 120)
    b.set_tuning(steps_per_launch=4)
    b.step_n(1 / 120, frames, bt)
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    # kami_vbd_step_host: pageable arrays take the three calls; pinned ones the frame kernel over groups,
    # which equals them to rounding (it is compiled on its own)
    import torch

    x, v = a.get_positions_velocities()
    v = v + np.float32(0.01)
    xo, vo = b.step_host(1 / 120, x.copy(), v.copy())
    a.set_positions_velocities(x, v)
    a.step(1 / 120)
    xa, va = a.get_positions_velocities()
    np.testing.assert_array_equal(xo, xa)
    np.testing.assert_array_equal(vo, va)
    xp = torch.from_numpy(xa.copy()).pin_memory()
    vp = torch.from_numpy(va.copy()).pin_memory()
    b.step_host(1 / 120, xp, vp)
    a.step(1 / 120)
    xa, va = a.get_positions_velocities()
    np.testing.assert_allclose(xp.numpy(), xa, rtol=0, atol=1e-6)
    np.testing.assert_allclose(vp.numpy(), va, rtol=0, atol=2e-4)
    a.close()
    b.close()


def test_long_strands_autotune_and_adjoint_scope():
    g = _mixed(seed=8)
    st = _settings()
    s = helpers.gpu_solver(g, st, form="fused")
    s.step(1 / 120)
    before = s.get_state()
    best, rate = s.autotune(1 / 120, trial_steps=4)
    assert best[0] in (2, 4) and best[3] in (1, 120, 168) and rate > 0
    np.testing.assert_array_equal(s.get_state(), before)
    s.tape_reserve(2)  # the adjoint covers every group size the tuning may pick
    s.step_record(1 / 120)
    s.close()


@pytest.mark.parametrize("slots", [4, 2])
def test_nonfinite_long_strand_does_not_leak(slots):
    """A strand that turns non-finite leaves every other strand of its group untouched, across the
    warps of the group too."""
    from kamisimulator_b200.vbd import KamiError

    g = helpers.soft_groom(48, (60, 300), seed=19)
    st = helpers.soft_settings()
    clean = helpers.gpu_solver(g, st, form="fused")
    bad = helpers.gpu_solver(g, st, form="fused")
    clean.set_tuning(slots_per_lane=slots)
    bad.set_tuning(slots_per_lane=slots)
    victim = int(np.argmax(np.diff(g.strand_begin)))  # the longest strand spans several tiles
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
