"""kami_vbd_step_noalloc: the step for callers that cannot let the library allocate device memory
(an engine that owns a fixed device pool or budget, or a real-time frame loop in which an
allocation's device-wide synchronisation would miss the deadline).  The caller owns every state
buffer; the entry point's scratch is a fixed __device__ array.

The test plays such a caller: it allocates the state itself (torch), advances it with two
no-alloc calls in a row, and checks each result against the handle API (kami_vbd_create /
kami_vbd_step) on the same groom, within the parity tolerances of the other tests.  This file is
collected last so that a stop-at-first-failure run has already run every other test."""
import ctypes

import numpy as np
import pytest

from tests import helpers
from tests.helpers import POS_TOL, TWIST_TOL, NoAllocArgs, bind_noalloc

pytestmark = pytest.mark.gpu


def test_noalloc_step_matches_handle_step_on_two_calls():
    import torch

    from kamisimulator_b200 import vbd
    from oracle import oracle as orc
    from oracle.oracle import twist_angles

    lib, step_noalloc = bind_noalloc()
    groom = helpers.soft_groom(200, (5, 61), seed=31)  # uneven strands: many start at an odd index
    v0 = helpers.random_velocities(groom, 0.2, seed=9)
    st = helpers.soft_settings(num_itr=6, max_h=1 / 120)  # two substeps per call
    dt = 1 / 60

    handle = helpers.gpu_solver(groom, st, form="sweep", velocities=v0)
    mat = orc.configure(groom, radius=st["radius"], density=st["density"], dtype=np.float32)
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)  # noqa: E731
    sb = t(groom.strand_begin.astype(np.int32))
    x = t(groom.positions.astype(np.float32))
    v = t(v0)
    vl = torch.zeros_like(x)
    q = t(handle.get_orientations())
    qr = t(handle.get_rest_darboux())
    im, lr, ks = t(mat["inv_mass"]), t(mat["l_rest"]), t(mat["k_stretch"])

    desc = vbd.Desc()
    assert lib.kami_vbd_desc_init(ctypes.byref(desc)) == 0
    desc.gravity[:] = st["gravity"]
    desc.damping, desc.velocity_decay, desc.acceleration_ratio = st["damping"], st["velocity_decay"], 1.0
    desc.external_force_multiplier = 1.0
    desc.wind_peak = 0.0
    desc.num_itr = st["num_itr"]
    desc.max_h = st["max_h"]
    desc.schedule = 0

    args = NoAllocArgs()
    args.num_vertices, args.num_strands = groom.num_vertices, groom.num_strands
    for name, ten in (("strand_begin", sb), ("positions", x), ("velocities", v), ("last_velocities", vl),
                      ("orientations", q), ("rest_darboux", qr), ("inv_mass", im), ("rest_length", lr),
                      ("stretch_stiffness", ks)):
        setattr(args, name, ten.data_ptr())
    args.clock[:] = (np.float32(st["max_h"]), 0.0, 0.0)
    torch.cuda.synchronize()

    for call in range(2):
        free_before = torch.cuda.mem_get_info()[0]
        rc = step_noalloc(ctypes.byref(desc), ctypes.byref(args), dt, None)
        assert rc == 0, lib.kami_vbd_last_error_string().decode()
        torch.cuda.synchronize()
        if call == 1:  # the first call may load the module; after it the device's free memory stays put
            assert torch.cuda.mem_get_info()[0] == free_before
        handle.step(dt)
        xh, vh = handle.get_positions_velocities()
        qh = handle.get_orientations()
        ex = float(np.abs(x.cpu().numpy() - xh).max())
        ev = float(np.abs(v.cpu().numpy() - vh).max())
        et = float(np.abs(twist_angles(qh, q.cpu().numpy())).max())
        assert ex <= POS_TOL and et <= TWIST_TOL, (call, ex, et)
        assert ev <= POS_TOL / (dt / 2), (call, ev)  # velocity = displacement / substep length
        assert float(np.abs(xh - groom.positions).max()) > 1e-3  # the strands really moved
    assert args.clock[0] == pytest.approx(st["max_h"])
    assert args.clock[2] == pytest.approx(2 * dt)
    handle.close()


def test_noalloc_rejects_more_vertices_than_its_scratch():
    from kamisimulator_b200 import vbd

    lib, step_noalloc = bind_noalloc()
    desc = vbd.Desc()
    lib.kami_vbd_desc_init(ctypes.byref(desc))
    args = NoAllocArgs()
    args.num_vertices = 262144 + 1
    args.num_strands = 1
    rc = step_noalloc(ctypes.byref(desc), ctypes.byref(args), 1 / 60, None)
    assert rc == 6  # KAMI_ERR_UNSUPPORTED
    assert "262144" in lib.kami_vbd_last_error_string().decode()


def test_noalloc_clamps_an_overlong_last_strand():
    """strand_begin[num_strands] past num_vertices is clamped to the vertex range on the device: the
    step equals the one with well-formed offsets, bit for bit, and reads nothing past the arrays."""
    import torch

    from kamisimulator_b200 import vbd
    from oracle import oracle as orc

    lib, step_noalloc = bind_noalloc()
    groom = helpers.soft_groom(40, (5, 30), seed=5)
    st = helpers.soft_settings(num_itr=4, max_h=1 / 60)
    handle = helpers.gpu_solver(groom, st, form="sweep")
    mat = orc.configure(groom, radius=st["radius"], density=st["density"], dtype=np.float32)
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)  # noqa: E731
    q0, qr = handle.get_orientations(), t(handle.get_rest_darboux())
    handle.close()
    im, lr, ks = t(mat["inv_mass"]), t(mat["l_rest"]), t(mat["k_stretch"])
    desc = vbd.Desc()
    lib.kami_vbd_desc_init(ctypes.byref(desc))
    desc.gravity[:] = st["gravity"]
    desc.num_itr, desc.max_h, desc.schedule, desc.wind_peak = st["num_itr"], st["max_h"], 0, 0.0
    out = []
    for extra in (0, 40):
        sb = groom.strand_begin.astype(np.int32).copy()
        sb[-1] += extra
        bufs = dict(strand_begin=t(sb), positions=t(groom.positions.astype(np.float32)),
                    velocities=t(helpers.random_velocities(groom, 0.2, seed=3)),
                    last_velocities=torch.zeros((groom.num_vertices, 3), device=dev), orientations=t(q0),
                    rest_darboux=qr, inv_mass=im, rest_length=lr, stretch_stiffness=ks)
        args = NoAllocArgs()
        args.num_vertices, args.num_strands = groom.num_vertices, groom.num_strands
        for name, ten in bufs.items():
            setattr(args, name, ten.data_ptr())
        args.clock[:] = (np.float32(st["max_h"]), 0.0, 0.0)
        assert step_noalloc(ctypes.byref(desc), ctypes.byref(args), 1 / 60, None) == 0
        torch.cuda.synchronize()
        out.append((bufs["positions"].cpu().numpy(), bufs["orientations"].cpu().numpy()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert float(np.abs(out[0][0] - groom.positions).max()) > 1e-4
