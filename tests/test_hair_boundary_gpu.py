"""Device-resident Hair boundary (kami_vbd_set_hair_layout / upload_hair / download_hair): the
solver reads and writes KamiSimulator's padded [strand][vertex] Hair arrays directly, with the
strandRefs mapping of StableCosseratRodsSolver (strands of fewer than 4 vertices are not in the
solver, .cpp:134-136)."""
import numpy as np
import pytest

from kamisimulator_b200 import synth
from tests import helpers

pytestmark = pytest.mark.gpu

MAXV = 40


def _hair():
    """A Hair of 9 strands, 3 of them too short for the solver; returns (Hair padded xyz, counts,
    solver groom, strand_refs)."""
    counts = np.array([12, 3, 30, 2, 25, 8, 1, 40, 16], np.int32)
    g_all = synth.groom_strands(np.random.default_rng(4), counts)
    padded = np.full((len(counts), MAXV, 3), -7.0, np.float32)  # sentinel in entries the solver does not own
    for s, n in enumerate(counts):
        padded[s, :n] = g_all.positions[g_all.strand_begin[s]:g_all.strand_begin[s + 1]]
    refs = np.array([s for s, n in enumerate(counts) if n >= 4], np.int32)
    keep = [padded[u, :counts[u]] for u in refs]
    g = synth.Groom(strand_begin=np.concatenate([[0], np.cumsum([len(k) for k in keep])]).astype(np.int32),
                    positions=np.concatenate(keep).astype(np.float32),
                    strand_young=np.full(len(refs), 1e-3, np.float32), strand_dev=np.ones(len(refs), np.float32))
    return padded, counts, g, refs


def _padded_from_packed(base, x, g, refs):
    out = base.copy()
    for s, u in enumerate(refs):
        a, b = g.strand_begin[s], g.strand_begin[s + 1]
        out[u, :b - a] = x[a:b]
    return out


def test_download_and_upload_match_the_packed_boundary():
    import torch

    padded, counts, g, refs = _hair()
    st = dict(num_itr=6, max_h=1 / 60, gravity=(0.0, 0.0, -9.81), radius=40e-6)
    s = helpers.gpu_solver(g, st, form="fused")
    from kamisimulator_b200.vbd import KamiError

    with pytest.raises(KamiError, match="KAMI_ERR_STATE"):
        s.download_hair(padded.copy())
    with pytest.raises(KamiError, match="referenced twice"):
        s.set_hair_layout(len(counts), MAXV, np.full(len(refs), refs[0]))
    with pytest.raises(KamiError, match="max_verts"):
        s.set_hair_layout(len(counts), 20, refs)
    s.set_hair_layout(len(counts), MAXV, refs)
    for _ in range(3):
        s.step(1 / 60)
    x, v = s.get_positions_velocities()
    # host arrays: solver entries replaced, the others kept
    hx, hv = padded.copy(), np.full_like(padded, -7.0)
    s.download_hair(hx, hv)
    np.testing.assert_array_equal(hx, _padded_from_packed(padded, x, g, refs))
    np.testing.assert_array_equal(hv, _padded_from_packed(np.full_like(padded, -7.0), v, g, refs))
    # device arrays: the same values, no host copy
    dx = torch.tensor(padded, device="cuda")
    dv = torch.zeros_like(dx)
    s.download_hair(dx, dv)
    np.testing.assert_array_equal(dx.cpu().numpy(), hx)
    # upload from padded device arrays = set_positions_velocities of the packed values
    rng = np.random.default_rng(1)
    nx = hx + rng.normal(scale=1e-4, size=hx.shape).astype(np.float32)
    nvel = rng.normal(scale=1e-2, size=hx.shape).astype(np.float32)
    s.upload_hair(torch.tensor(nx, device="cuda"), torch.tensor(nvel, device="cuda"))
    x2, v2 = s.get_positions_velocities()
    packed_x = np.concatenate([nx[u, :counts[u]] for u in refs])
    packed_v = np.concatenate([nvel[u, :counts[u]] for u in refs])
    np.testing.assert_array_equal(x2, packed_x)
    np.testing.assert_array_equal(v2, packed_v)
    # and from host arrays
    s.upload_hair(hx, None)
    np.testing.assert_array_equal(s.get_positions_velocities()[0], x)
    s.close()


def test_usc_file_to_device_hair_round_trip(tmp_path):
    """A .data file read padded (as ImportUSCHairSalonToHair fills the Hair), stepped, and written
    back through the device-resident Hair."""
    import torch

    from kamisimulator_b200 import vbd

    padded, counts, g, refs = _hair()
    vbd.write_usc(tmp_path / "in.data", counts, padded, max_verts=MAXV)
    c, hair = vbd.read_usc(tmp_path / "in.data", max_verts=MAXV)
    np.testing.assert_array_equal(c, counts)
    s = helpers.gpu_solver(g, dict(num_itr=6, max_h=1 / 60, gravity=(0.0, 0.0, -9.81), radius=40e-6), form="fused")
    s.set_hair_layout(len(c), MAXV, refs)
    d = torch.tensor(hair, device="cuda")
    for _ in range(2):
        s.step(1 / 60)
    s.download_hair(d)
    out = d.cpu().numpy()
    vbd.write_usc(tmp_path / "out.data", c, out, max_verts=MAXV)
    c2, back = vbd.read_usc(tmp_path / "out.data", max_verts=MAXV)
    np.testing.assert_array_equal(back, np.where(np.arange(MAXV)[None, :, None] < c[:, None, None], out, 0.0))
    x = s.get_positions_velocities()[0]
    np.testing.assert_array_equal(np.concatenate([back[u, :c[u]] for u in refs]), x)
    s.close()


def _pinned(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory()


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_step_hair_frames_equal_upload_step_download(schedule):
    """kami_vbd_step_hair on page-locked padded Hair arrays (one launch: the frame kernel reads each
    tile's strands from the Hair, steps them and writes them back) against UploadHair, SolveNextStep,
    DownloadHair as three calls on pageable arrays; the entries the solver does not own keep their
    values.  Frames with input and output, with output only (the device state is current) and with
    input only (the results stay on the device) all agree."""
    import torch

    padded, counts, g, refs = _hair()
    st = dict(num_itr=6, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, sdf=synth.sphere_sdf(64),
              schedule=schedule)
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="fused")
    for s in (a, b):
        s.set_hair_layout(len(counts), MAXV, refs)
    ha, va = padded.copy(), np.full_like(padded, -7.0)
    hb, vb = _pinned(padded), _pinned(np.full_like(padded, -7.0))
    a.download_hair(None, va)  # the solver's initial velocities into the owned entries
    b.download_hair(None, vb)  # (page-locked: the gather kernel writes the host array itself)
    np.testing.assert_array_equal(vb.numpy(), va)
    rng = np.random.default_rng(2)
    for f in range(6):
        kick = (1e-3 * rng.standard_normal(va.shape)).astype(np.float32)
        va += kick
        vb += torch.from_numpy(kick)
        a.upload_hair(ha, va)
        a.step(1 / 60)
        a.download_hair(ha, va)
        if f % 3 == 0:
            b.step_hair(1 / 60, hb, vb, hb, vb)
        elif f % 3 == 1:
            b.upload_hair(hb, vb)
            b.step_hair(1 / 60, None, None, hb, vb)
        else:
            b.step_hair(1 / 60, hb, vb, None, None)
            b.download_hair(hb, vb)
        np.testing.assert_allclose(hb.numpy(), ha, rtol=0, atol=1e-6)
        np.testing.assert_allclose(vb.numpy(), va, rtol=0, atol=2e-4)
        hb.copy_(torch.from_numpy(ha))  # continue from the same state
        vb.copy_(torch.from_numpy(va))
    owned = np.zeros(padded.shape[:2], bool)
    for u in refs:
        owned[u, :counts[u]] = True
    np.testing.assert_array_equal(hb.numpy()[~owned], padded[~owned])  # not the solver's: untouched
    assert np.abs(ha[owned] - padded[owned]).max() > 1e-4
    a.close()
    b.close()
