"""The sweep form's iteration in one launch (sweep_iteration_kernel, tiles of up to 1024 slots)
against the per-sweep launches (sweep_position_kernel and sweep_orientation_kernel: four per
colour2 iteration, two per Jacobi iteration, which tiles over 1024 slots keep): the same operands
and arithmetic, so the same state bit for bit, with and without connection springs."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
@pytest.mark.parametrize("tied", [False, True])
def test_one_launch_iteration_equals_the_sweep_launches(tied, schedule):
    g = helpers.soft_groom(200, (8, 60), seed=17)
    st = helpers.soft_settings(sdf=synth.sphere_sdf(64, threshold=2e-3), num_itr=8, max_h=1 / 120, schedule=schedule)
    if tied:  # every strand's tip tied to the next strand's tip, both ways
        conn = np.full(g.num_vertices, -1, np.int32)
        tips = np.asarray(g.strand_begin[1:]) - 1
        for a, b in zip(tips[0::2], tips[1::2]):
            conn[a], conn[b] = b, a
        st["connection_index"] = conn
    one = helpers.gpu_solver(g, dict(st, slots_per_lane=2), form="sweep")    # 64-slot tiles: one launch
    four = helpers.gpu_solver(g, dict(st, slots_per_lane=34), form="sweep")  # 1088-slot tiles: per-sweep launches
    try:
        assert (one.slots_per_lane, four.slots_per_lane) == (2, 34)
        for _ in range(6):
            one.step(1 / 60)
            four.step(1 / 60)
        a, b = one.get_state(), four.get_state()
        moved = np.abs(one.get_positions_velocities()[0] - g.positions).max()
    finally:
        one.close()
        four.close()
    assert moved > 1e-3
    np.testing.assert_array_equal(a, b)
