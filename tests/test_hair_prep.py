"""Hair preprocessing restated in the oracle, against the reference's own code built from source on
the CPU (oracle/_ref/libkami_ref_cpu.so): Resample::resampleCMR (YarnBall/io/resample.h)."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle import oracle as orc
from oracle import ref_sim

needs_ref = pytest.mark.skipif(not ref_sim.cpu_available(), reason="oracle/_ref not built (needs the reference sources)")


# The reference's resampleCMRCoords writes one entry before its list when a pass has 8 samples or
# fewer (resample.h:78-79: ts[ts.size() - 2 - i] for i up to min(size, 8) - 1), which corrupts the
# heap; it is only called for strands whose result (by the oracle, which equals it) is well above.
SAFE_FOR_REFERENCE = 16


@needs_ref
@pytest.mark.parametrize("target", [7e-4, 1e-3, 2.5e-3])
def test_oracle_resample_equals_the_reference(target):
    """Curled 64-point strands (48 to 180 samples: the two-way merge runs) and 12- to 20-point
    strands (single direction), bit for bit."""
    g = synth.groom(40, 64, seed=2)
    short = synth.groom_strands(np.random.default_rng(5), np.array([12, 14, 16, 20]))
    compared = 0
    for gg in (g, short):
        for s in range(gg.num_strands):
            pts = gg.positions[gg.strand_begin[s]:gg.strand_begin[s + 1]]
            a = orc.resample_cmr(pts, target)
            if a.shape[0] < SAFE_FOR_REFERENCE:
                continue
            np.testing.assert_array_equal(a, ref_sim.resample_cmr(pts, target))
            compared += 1
    assert compared >= 40


def test_resample_gives_even_segments():
    g = synth.groom(10, 64, seed=4)
    for s in range(g.num_strands):
        pts = g.positions[g.strand_begin[s]:g.strand_begin[s + 1]]
        r = orc.resample_cmr(pts, 1e-3)
        seg = np.linalg.norm(np.diff(r.astype(np.float64), axis=0), axis=1)
        assert np.abs(seg - seg.mean()).max() < 0.05 * seg.mean()
        assert abs(seg.mean() - 1e-3) < 0.1e-3
