"""Host frames (kami_vbd_step_host): one call uploads positions and velocities, steps and downloads.
With page-locked buffers the fused frame kernel reads and writes the host arrays itself; its
results must equal the three calls kami_vbd_set_positions_velocities -> kami_vbd_step ->
kami_vbd_get_positions_velocities to rounding: every tile runs the same arithmetic on the same data,
but the frame kernel is compiled on its own, so the compiler may contract a few multiply-adds
differently (last-bit differences, far below the 1e-5 m parity bound)."""
import numpy as np
import pytest
import torch

from kamisimulator_b200 import synth
from tests import helpers

pytestmark = pytest.mark.gpu

DT = 1 / 120


def _uneven():
    # ~116k vertices in strands of 16-128 vertices (several strands per tile), tiles of 128 slots
    grooms = synth.batched_grooms(6, strands_range=(500, 20_000), verts_range=(16, 128), seed=3, strand_scale=0.05)
    return synth.concat_grooms(grooms)


def _settings(**kw):
    st = dict(num_itr=8, max_h=1 / 120, gravity=(0.0, 0.0, -9.81), radius=40e-6, sdf=synth.sphere_sdf(64))
    st.update(kw)
    return st


def _pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory()


def _same(xb, vb, xa, va):
    np.testing.assert_allclose(np.asarray(xb), xa, rtol=0, atol=1e-6)  # m
    np.testing.assert_allclose(np.asarray(vb), va, rtol=0, atol=2e-4)  # m/s (1e-6 m over a 1/120 s step)


def _sequential(s, x, v, dt=DT):
    s.set_positions_velocities(x, v)
    s.step(dt)
    return s.get_positions_velocities()


@pytest.mark.parametrize("tuning,schedule", [(None, "colour2"), ((4, 2, 8, 1), "colour2"), ((4, 4, 8, 2), "colour2"),
                                             ((4, 8, 8, 1), "jacobi"), (None, "jacobi")])
def test_step_host_equals_upload_step_download(tuning, schedule):
    g = _uneven()
    st = _settings(schedule=schedule)
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="fused")
    if tuning is not None:
        a.set_tuning(*tuning)
        b.set_tuning(*tuning)
    xa, va = a.get_positions_velocities()
    xb, vb = _pinned(xa), _pinned(va)
    rng = np.random.default_rng(0)
    for f in range(6):
        rot, tr = synth.head_rotation(f / 120.0), [0.001 * f, 0.0, 0.0]
        a.set_body_transform(rot, tr)
        b.set_body_transform(rot, tr)
        # the host edits the hair between frames, as a caller of UploadHair would
        kick = (1e-3 * rng.standard_normal(va.shape)).astype(np.float32)
        va = va + kick
        vb += torch.from_numpy(kick)
        xa, va = _sequential(a, xa, va)
        b.step_host(DT, xb, vb)  # in place
        _same(xb.numpy(), vb.numpy(), xa, va)
        # continue both from the same state, so that last-bit differences do not accumulate
        xb.copy_(torch.from_numpy(xa))
        vb.copy_(torch.from_numpy(va))
    assert np.abs(xa - g.positions.reshape(-1, 3)).max() > 1e-4  # the hair moved
    a.close()
    b.close()


def test_step_host_follows_new_buffers_and_retuning():
    # the frame kernel must follow the buffers of each call, and a new tile shape needs new strand runs
    g = _uneven()
    st = _settings()
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="fused")
    xa, va = a.get_positions_velocities()
    pairs = [(_pinned(xa), _pinned(va)), (_pinned(np.zeros_like(xa)), _pinned(np.zeros_like(va)))]
    outs = (_pinned(np.zeros_like(xa)), _pinned(np.zeros_like(va)))
    for f in range(6):
        if f == 3:
            a.set_tuning(4, 2, 8, 1)
            b.set_tuning(4, 2, 8, 1)
        xi, vi = pairs[f % 2]
        xi.copy_(torch.from_numpy(xa))
        vi.copy_(torch.from_numpy(va + np.float32(1e-3 * f)))
        xa, va = _sequential(a, xa, va + np.float32(1e-3 * f))
        if f % 3 == 2:
            b.step_host(DT, xi, vi, *outs)
            xo, vo = outs
        else:
            b.step_host(DT, xi, vi)
            xo, vo = xi, vi
        _same(xo.numpy(), vo.numpy(), xa, va)
    a.close()
    b.close()


def test_step_host_separate_outputs_from_pageable_arrays():
    g = _uneven()
    st = _settings()
    a = helpers.gpu_solver(g, st, form="fused")
    b = helpers.gpu_solver(g, st, form="fused")
    x0, v0 = a.get_positions_velocities()
    x_in, v_in = x0.copy(), v0.copy()
    xo, vo = np.zeros_like(x0), np.zeros_like(v0)
    b.step_host(DT, x_in, v_in, xo, vo)
    np.testing.assert_array_equal(x_in, x0)  # inputs untouched
    np.testing.assert_array_equal(v_in, v0)
    xa, va = _sequential(a, x0, v0)
    _same(xo, vo, xa, va)
    a.close()
    b.close()


@pytest.mark.parametrize("case", ["sweep", "c2_r120", "zero_dt"])
def test_step_host_small_and_three_call_cases(case):
    g = synth.groom(200, 32, seed=4) if case == "c2_r120" else _uneven()
    st = _settings()
    form = "sweep" if case == "sweep" else "fused"
    dt = 0.0 if case == "zero_dt" else DT
    a = helpers.gpu_solver(g, st, form=form)
    b = helpers.gpu_solver(g, st, form=form)
    if case == "c2_r120":
        a.set_tuning(2, 1, 8, 120)
        b.set_tuning(2, 1, 8, 120)
    x0, v0 = a.get_positions_velocities()
    v0 = v0 + np.float32(0.01)
    for _ in range(2):
        xa, va = _sequential(a, x0, v0, dt)
        xb, vb = b.step_host(dt, _pinned(x0), _pinned(v0))
        xb, vb = xb.numpy(), vb.numpy()
        _same(xb, vb, xa, va)
        x0, v0 = xa, va
    if case == "zero_dt":
        np.testing.assert_array_equal(xb, a.get_positions_velocities()[0])
    a.close()
    b.close()


def test_step_host_rejects_bad_arrays():
    g = synth.groom(50, 16, seed=5)
    s = helpers.gpu_solver(g, _settings(), form="fused")
    x, v = s.get_positions_velocities()
    with pytest.raises(ValueError):
        s.step_host(DT, x[:-1], v)
    with pytest.raises(ValueError):
        s.step_host(DT, x.astype(np.float64), v)
    with pytest.raises(ValueError):
        s.step_host(DT, torch.from_numpy(x).cuda(), v)
    s.close()
