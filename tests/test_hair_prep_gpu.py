"""kami_hair_resample and kami_hair_subdivide on the GPU: resampling equals the reference's own
resampleCMR (built from source) and the oracle bit for bit, with BuildYarnBallHair's subsampling to
the Hair's row; subdivision equals DivideHair's interpolation formula in float32."""
import numpy as np
import pytest

from kamisimulator_b200 import synth, vbd
from oracle import oracle as orc
from oracle import ref_sim

pytestmark = pytest.mark.gpu


def _padded(g, mv):
    counts = np.diff(g.strand_begin).astype(np.int32)
    x = np.zeros((g.num_strands, mv, 3), np.float32)
    for s in range(g.num_strands):
        x[s, :counts[s]] = g.positions[g.strand_begin[s]:g.strand_begin[s + 1]]
    return counts, x


@pytest.mark.parametrize("target", [1e-3, 2.5e-3])
def test_gpu_resample_is_bit_exact(target):
    g = synth.groom(300, 64, seed=3)
    counts, x = _padded(g, 200)
    c, r = vbd.hair_resample(counts, x, target)
    for s in range(g.num_strands):
        pts = g.positions[g.strand_begin[s]:g.strand_begin[s + 1]]
        want = orc.resample_cmr(pts, target)
        assert c[s] == want.shape[0]
        np.testing.assert_array_equal(r[s, :c[s]], want)
        if ref_sim.cpu_available() and want.shape[0] >= 16:  # see tests/test_hair_prep.py on short passes
            np.testing.assert_array_equal(r[s, :c[s]], ref_sim.resample_cmr(pts, target))


def test_resample_subsamples_to_the_hair_row_and_skips_short_strands():
    g = synth.groom_strands(np.random.default_rng(6), np.array([3, 40, 2, 64]))
    counts, x = _padded(g, 64)
    c, r = vbd.hair_resample(counts, x, 5e-4)  # ~4 samples per 2 mm segment: longer than 64
    assert c[0] == 3 and c[2] == 2
    np.testing.assert_array_equal(r[0], x[0])
    np.testing.assert_array_equal(r[2], x[2])
    for s in (1, 3):
        full = orc.resample_cmr(g.positions[g.strand_begin[s]:g.strand_begin[s + 1]], 5e-4)
        if full.shape[0] <= 64:
            np.testing.assert_array_equal(r[s, :c[s]], full)
            continue
        assert c[s] == 64
        stride = np.float32(full.shape[0] - 2) / np.float32(64 - 2)
        idx = [0] + [int(np.float32(stride * np.float32(v))) for v in range(1, 63)] + [full.shape[0] - 1]
        np.testing.assert_array_equal(r[s], full[idx])  # StableCosseratRodsSolver.cpp:147-158


def test_gpu_subdivide_equals_divide_hair():
    g = synth.groom_strands(np.random.default_rng(7), np.array([5, 1, 12, 9]))
    counts, x = _padded(g, 12)
    v = np.random.default_rng(8).normal(size=x.shape).astype(np.float32)
    oc, ox, ov = vbd.hair_subdivide(counts, x, 3, v)
    assert ox.shape == (4, 34, 3)
    np.testing.assert_array_equal(oc, np.where(counts > 0, (counts - 1) * 3 + 1, 0))
    den = np.float32(3)
    for s, n in enumerate(counts):
        for w in range(oc[s]):
            seg, i = divmod(w, 3)
            if seg == n - 1:
                np.testing.assert_array_equal(ox[s, w], x[s, seg])
                continue
            num = np.float32(i)
            want = ((den - num) * x[s, seg] + num * x[s, seg + 1]) / den  # HairModification.cpp:5-10
            np.testing.assert_array_equal(ox[s, w], want.astype(np.float32))
            wv = ((den - num) * v[s, seg] + num * v[s, seg + 1]) / den
            np.testing.assert_array_equal(ov[s, w], wv.astype(np.float32))
