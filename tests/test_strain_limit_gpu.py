"""Strain limiting (kami_vbd_strain_limit): the SDF solver's StrainLimiting kernel
(SDFCollisionSolver/cudaSDFCollision.cu:176-199), which SDFBodyCollisionSolver::SolveNextStep runs
after its SDF pass when UseStrainLimiting is set (SDFBodyCollisionSolver.cpp:186).  The GPU result
is checked against the FP32 oracle restatement and against the reference's own kernel, built from
its sources, on strands stretched and compressed past the tolerance, for every tile layout."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle import oracle as orc
from oracle import ref_sim
from tests import helpers

pytestmark = pytest.mark.gpu

# helper_math's normalize is v * rsqrtf(v . v) on the device and v / sqrtf(v . v) on the host: the
# oracle's corrections may differ from the device's by a few ulp of the positions
ORACLE_TOL = 2e-6  # m


def _strained(groom, seed, lo=0.7, hi=1.3):
    """The groom's positions with every segment scaled by a random factor in [lo, hi] (strands rebuilt
    from the root), so that most segments are off their rest length by more than the tolerance."""
    rng = np.random.default_rng(seed)
    x = np.asarray(groom.positions, np.float32).copy()
    for s in range(groom.num_strands):
        a, b = groom.strand_begin[s], groom.strand_begin[s + 1]
        seg = np.diff(groom.positions[a:b], axis=0) * rng.uniform(lo, hi, (b - a - 1, 1))
        x[a + 1:b] = x[a] + np.cumsum(seg, axis=0)
    return x.astype(np.float32)


def _rest_lengths(groom):
    return orc.configure(groom)["l_rest"].astype(np.float32)


def _gpu_strain_limit(groom, x, err, form="auto", tuning=None):
    s = helpers.gpu_solver(groom, dict(num_itr=2, max_h=1 / 120), form=form)
    try:
        if tuning is not None:
            s.set_tuning(*tuning)
        v = np.zeros_like(x)
        s.set_positions_velocities(x, v)
        s.strain_limit(err)
        out, vel = s.get_positions_velocities()
    finally:
        s.close()
    assert np.array_equal(vel, v)  # positions only
    return out


@pytest.mark.parametrize("form,tuning", [("fused", (2, 4, 1, 120)), ("fused", (4, 4, 1, 168)), ("sweep", None)])
def test_strain_limit_matches_the_reference_kernel(form, tuning):
    """Segments stretched and compressed by up to 30 %: the same result as the reference's kernel on
    every layout, and every segment within the tolerance afterwards."""
    g = helpers.soft_groom(300, (6, 64), seed=21)
    x = _strained(g, 5)
    l0 = _rest_lengths(g)
    ours = _gpu_strain_limit(g, x, 0.1, form, tuning)
    ref = ref_sim.strain_limit(x, g.strand_begin, l0, 0.1)
    moved = np.abs(ref - x).max(axis=1) > 0
    assert moved.mean() > 0.5  # most vertices were corrected
    np.testing.assert_allclose(ours, ref, rtol=0, atol=1e-7)
    # every segment ends within the tolerance, measured from the corrected vertex before it
    for s in range(g.num_strands):
        a, b = g.strand_begin[s], g.strand_begin[s + 1]
        lens = np.linalg.norm(np.diff(ours[a:b].astype(np.float64), axis=0), axis=1)
        assert np.all(np.abs(lens - l0[a:b - 1]) <= 0.1 * l0[a:b - 1] + 1e-6)


def test_strain_limit_matches_the_oracle_on_stretched_strands():
    """The FP32 oracle restatement against the GPU (and the reference's kernel) where the march is well
    conditioned: stretched strands.  Under compression the march is not: a vertex pushed out to its
    rest length can leave the next segment short, and then an ulp of difference in that vertex grows
    by l0 / l at every later correction (a one-ulp change of the input moves the oracle's own result
    by 4e-4 m on the mixed input above), so there the reference's kernel is the bar."""
    g = helpers.soft_groom(300, (6, 64), seed=21)
    x = _strained(g, 7, 1.0, 1.3)
    l0 = _rest_lengths(g)
    ours = _gpu_strain_limit(g, x, 0.1)
    oracle = orc.strain_limit(x, g.strand_begin, l0, 0.1)
    assert (np.abs(oracle - x).max(axis=1) > 0).mean() > 0.5
    assert np.abs(ours - oracle).max() <= ORACLE_TOL
    np.testing.assert_allclose(ref_sim.strain_limit(x, g.strand_begin, l0, 0.1), oracle, rtol=0, atol=ORACLE_TOL)


def test_strain_limit_on_strands_across_groups_of_tiles():
    """Strands of 200 vertices run across groups of 4 tiles (C = 2): the march follows them from tile
    to tile."""
    g = synth.groom(64, 200, seed=3)
    x = _strained(g, 6)
    l0 = _rest_lengths(g)
    s = helpers.gpu_solver(g, dict(num_itr=2, max_h=1 / 120), form="fused")
    try:
        s.set_tuning(2, 1, 1, 1)
        assert s.tiles_per_group() > 1
        s.set_positions_velocities(x, np.zeros_like(x))
        s.strain_limit(0.05)
        ours = s.get_positions_velocities()[0]
    finally:
        s.close()
    np.testing.assert_allclose(ours, ref_sim.strain_limit(x, g.strand_begin, l0, 0.05), rtol=0, atol=1e-7)


def test_step_then_strain_limit_in_stream_order():
    """A step followed by strain limiting, as SDFBodyCollisionSolver::SolveNextStep orders the SDF pass
    and the limit: the limit sees the step's positions."""
    g = helpers.soft_groom(120, (8, 40), seed=9)
    st = helpers.soft_settings(sdf=synth.sphere_sdf(64, threshold=2e-3))
    l0 = _rest_lengths(g)
    a = helpers.gpu_solver(g, st)
    b = helpers.gpu_solver(g, st)
    try:
        for _ in range(4):
            a.step(1 / 60)
            b.step(1 / 60)
            x = b.get_positions_velocities()[0]
            a.strain_limit(0.01)
            want = ref_sim.strain_limit(x, g.strand_begin, l0, 0.01)
            got = a.get_positions_velocities()[0]
            np.testing.assert_allclose(got, want, rtol=0, atol=1e-7)
            b.set_positions_velocities(got, b.get_positions_velocities()[1])
    finally:
        a.close()
        b.close()


def test_strain_limit_arguments_and_the_tape():
    from kamisimulator_b200.vbd import KamiError

    g = synth.cantilever(4, 16)
    s = helpers.gpu_solver(g, dict(num_itr=2, max_h=1 / 120), form="fused")
    try:
        for bad in (-0.1, float("nan"), float("inf")):
            with pytest.raises(KamiError, match="KAMI_ERR_INVALID_ARGUMENT"):
                s.strain_limit(bad)
        s.strain_limit(0.0)  # exact rest lengths: allowed
        s.tape_reserve(1)
        s.step_record(1 / 120)
        with pytest.raises(KamiError, match="KAMI_ERR_STATE"):
            s.strain_limit(0.1)
    finally:
        s.close()


def test_strain_limit_on_a_batch_handle_matches_each_groom_on_its_own():
    """A batch handle limits every groom's strands: the same positions, bit for bit, as each groom's
    own handle (the walk's arithmetic does not depend on where a strand sits in the tiles)."""
    from kamisimulator_b200.vbd import Solver

    g0 = helpers.soft_groom(120, (6, 64), seed=31)
    g1 = synth.groom(80, 40, seed=5)
    x0, x1 = _strained(g0, 1), _strained(g1, 2)
    st = dict(num_itr=2, max_h=1 / 120)
    b = Solver([g0, g1], **st)
    s0, s1 = Solver(g0, **st), Solver(g1, **st)
    try:
        b.set_positions_velocities(np.concatenate([x0, x1]), np.zeros((g0.num_vertices + g1.num_vertices, 3), np.float32))
        s0.set_positions_velocities(x0, np.zeros_like(x0))
        s1.set_positions_velocities(x1, np.zeros_like(x1))
        for s in (b, s0, s1):
            s.strain_limit(0.1)
        xb = b.get_positions_velocities()[0]
        want = np.concatenate([s0.get_positions_velocities()[0], s1.get_positions_velocities()[0]])
    finally:
        for s in (b, s0, s1):
            s.close()
    assert np.abs(want - np.concatenate([x0, x1])).max() > 1e-4
    np.testing.assert_array_equal(xb, want)
