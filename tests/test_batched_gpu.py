"""Batched stepping (kami_vbd_step_n), tile shapes and the autotuner."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from tests import helpers

pytestmark = pytest.mark.gpu


def _uneven(seed=3, scale=0.02):
    grooms = synth.batched_grooms(6, strands_range=(500, 20_000), verts_range=(16, 128), seed=seed,
                                  strand_scale=scale)
    return synth.concat_grooms(grooms)


def _settings():
    return dict(num_itr=8, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, sdf=synth.sphere_sdf(64))


def test_step_n_equals_single_steps_with_moving_body():
    g = _uneven()
    st = _settings()
    frames = 11
    bt = np.array([list(synth.head_rotation(f / 120.0)) + [0.002 * f, 0.0, 0.0] for f in range(frames)], np.float32)
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="fused")
    b.set_tuning(steps_per_launch=4)
    for f in range(frames):
        a.set_body_transform(bt[f, :4], bt[f, 4:])
        a.step(1 / 120)
    b.step_n(1 / 120, frames, bt)
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    # a second call replays the captured graph
    for f in range(frames):
        a.set_body_transform(bt[f, :4], bt[f, 4:])
        a.step(1 / 120)
    b.step_n(1 / 120, frames, bt)
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    a.close()
    b.close()


def test_relayout_keeps_the_trajectory():
    g = synth.groom(300, 60, seed=6)
    st = _settings()
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="fused")
    assert a.slots_per_lane == 2
    for _ in range(3):
        a.step(1 / 120)
        b.step(1 / 120)
    b.set_tuning(slots_per_lane=4, warps_per_block=2)
    assert b.get_tuning()[:2] == (4, 2)
    # the 120-register variant of the C = 2 kernel gives the same trajectory
    a.set_tuning(register_cap=120)
    assert a.get_tuning()[3] == 120
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    for _ in range(3):
        a.step(1 / 120)
        b.step(1 / 120)
    xa, _ = a.get_positions_velocities()
    xb, _ = b.get_positions_velocities()
    assert np.abs(xa - xb).max() <= 1e-6
    a.close()
    b.close()


def test_autotune_picks_a_shape_and_restores_the_state():
    g = _uneven(seed=4)
    st = _settings()
    s = helpers.gpu_solver(g, st, form="fused")
    s.step(1 / 120)
    before = s.get_state()
    best, rate = s.autotune(1 / 120, trial_steps=8)
    assert best[0] in (4,) and best[1] in (1, 2, 4, 8) and best[2] in (1, 4, 8) and best[3] in (1, 120)
    assert rate > 0
    np.testing.assert_array_equal(s.get_state(), before)
    ref = helpers.gpu_solver(g, st, form="fused")
    ref.step(1 / 120)
    s.step_n(1 / 120, 5)
    for _ in range(5):
        ref.step(1 / 120)
    assert np.abs(s.get_positions_velocities()[0] - ref.get_positions_velocities()[0]).max() <= 1e-6
    s.close()
    ref.close()
