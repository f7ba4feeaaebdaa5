"""Sag-free initialisation (kami_vbd_sag_free; Sim::SagFree, YarnBall/YBSimulator.cu:480-674):
the GPU kernel against the CPU restatement in the oracle, the oracle against the reference's own
SagFree built from source, and the effect it exists for: strands that hang under gravity keep
their initial shape."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle import oracle as orc
from oracle import ref_sim
from oracle.oracle import twist_angles
from tests import helpers

pytestmark = pytest.mark.gpu

ST = dict(num_itr=20, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6)


YOUNG = 0.05  # soft enough that the rest lengths change well above rounding


def _groom():
    g = synth.groom(300, 32, seed=7)
    g.strand_young[:] = YOUNG  # one modulus: the reference's driver takes one
    g.strand_dev[:] = 1.0
    return g


@pytest.mark.skipif(not ref_sim.available(), reason="oracle/_ref not built (needs the reference sources)")
def test_oracle_sag_free_matches_the_reference():
    g = _groom()
    r = ref_sim.RefSim(g, young=YOUNG, num_itr=20, max_h=1 / 120, gravity=ST["gravity"])
    r.sag_free(g.strand_begin, 2)
    m = r.material()
    r.close()
    base = orc.configure(g, radius=40e-6, dtype=np.float32)
    lr, q, qr = orc.sag_free(g, base, ST["gravity"], 2)
    assert np.abs(lr / base["l_rest"] - 1).max() > 1e-5  # it did work
    assert np.abs(q - base["q"]).max() > 1e-6
    np.testing.assert_allclose(lr, m["l_rest"], rtol=1e-6, atol=0)
    np.testing.assert_allclose(q, m["q"], rtol=0, atol=2e-6)
    np.testing.assert_allclose(qr, m["q_rest"], rtol=1e-5, atol=1e-6)


def test_gpu_sag_free_matches_the_oracle():
    g = _groom()
    s = helpers.gpu_solver(g, dict(ST, sag_free_itr=2), form="fused")
    base = orc.configure(g, radius=40e-6, dtype=np.float32)
    lr, q, qr = orc.sag_free(g, base, ST["gravity"], 2)
    np.testing.assert_allclose(s.get_orientations(), q, rtol=0, atol=2e-6)
    np.testing.assert_allclose(s.get_rest_darboux(), qr, rtol=1e-5, atol=1e-6)
    # the rest lengths show in the dynamics: step both from the sag-free set-up
    o = helpers.oracle_sim(g, ST, np.float32)
    o.l_rest[:], o.q[:], o.q_rest[:] = lr, q, qr
    worst = 0.0
    for _ in range(5):
        s.step(1 / 120)
        o.advance(1 / 120)
        x = s.get_positions_velocities()[0]
        worst = max(worst, float(np.abs(x - o.x).max()))
    assert worst <= helpers.POS_TOL
    assert np.abs(twist_angles(o.q, s.get_orientations())).max() <= helpers.TWIST_TOL
    s.close()


def test_sag_free_strands_move_less_from_their_initial_shape():
    """Strands grown out of the head (E = 0.01 GPa) move less from their initial shape over half a
    second after sag-free initialisation.  The reference's method is a partial compensation: on
    this groom it removes about a tenth of the motion (the oracle gives 8.5e-5 -> 7.6e-5 m mean)."""
    g = synth.groom(200, 32, seed=9)
    g.strand_young[:] = 1e-2
    moved = {}
    for k in (0, 3):
        s = helpers.gpu_solver(g, dict(ST, num_itr=30, sag_free_itr=k), form="fused")
        for _ in range(60):
            s.step(1 / 120)
        x = s.get_positions_velocities()[0]
        s.close()
        moved[k] = float(np.linalg.norm(x - g.positions, axis=1).mean())
    assert moved[3] < 0.95 * moved[0], moved
