"""CPU tests of the C-ABI library: it loads, exports every declared symbol, and rejects bad input
on the host before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from kamisimulator_b200 import synth, vbd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fname in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fname.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fname)).read()
            names += re.findall(r"^\s*(?:const\s+)?[a-z_]+\*?\s+\**(kami_\w+)\s*\(", text, re.M)
    return names


def test_library_exports_every_declared_symbol():
    lib = vbd.load_library()
    names = declared_symbols()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    assert set(vbd.EXPORTED) <= set(names)


def test_version_and_defaults():
    assert "sm_100a" in vbd.version()
    lib = vbd.load_library()
    d = vbd.Desc()
    assert lib.kami_vbd_desc_init(ctypes.byref(d)) == 0
    # JsonParams() defaults (StableCosseratRodsSolver.h:86-111), Sim defaults (YBSimulator.cu:81-111)
    assert d.num_itr == 8
    assert d.velocity_decay == pytest.approx(0.05)
    assert d.radius == pytest.approx(4e-5)
    assert d.density == pytest.approx(1300.0)
    assert d.young == pytest.approx(5.0)
    assert d.damping == pytest.approx(1e-6)
    assert d.max_h == pytest.approx(4e-4)
    assert d.wind_peak == 0.0
    assert d.pin_roots == 1


def _create(desc):
    lib = vbd.load_library()
    h = ctypes.c_void_p()
    rc = lib.kami_vbd_create(ctypes.byref(desc) if desc is not None else None, ctypes.byref(h))
    return rc, lib.kami_vbd_last_error_string().decode()


def _desc(groom, keep):
    lib = vbd.load_library()
    d = vbd.Desc()
    lib.kami_vbd_desc_init(ctypes.byref(d))
    sb = np.ascontiguousarray(groom.strand_begin, np.int32)
    pos = np.ascontiguousarray(groom.positions, np.float32)
    keep += [sb, pos]
    d.num_strands = groom.num_strands
    d.strand_begin = sb.ctypes.data
    d.positions = pos.ctypes.data
    return d


def test_host_side_errors():
    keep = []
    rc, msg = _create(None)
    assert rc == 1 and "null" in msg
    g = synth.cantilever(4, 8)
    d = _desc(g, keep)
    d.schedule = 7
    rc, msg = _create(d)
    assert rc == 1 and "schedule" in msg
    d = _desc(g, keep)
    d.num_itr = -1
    assert _create(d)[0] == 1
    d = _desc(g, keep)
    d.max_h = 0.0
    assert _create(d)[0] == 1
    # a one-vertex strand is a dangling segment (Sim::configure, YBSimulator.cu:185-186)
    g1 = synth.Groom(np.array([0, 1, 9], np.int32), g.positions[:9].copy(), np.ones(2, np.float32),
                     np.ones(2, np.float32))
    rc, msg = _create(_desc(g1, keep))
    assert rc == 5 and "dangling" in msg
    # zero-length segment (YBSimulator.cu:197)
    g2 = synth.cantilever(4, 8)
    g2.positions[3] = g2.positions[2]
    rc, msg = _create(_desc(g2, keep))
    assert rc == 5 and "zero-length" in msg
    # SDF descriptor checks
    d = _desc(g, keep)
    sd = vbd.SdfDesc()
    sd.dims[:] = (4, 4, 0)
    d.sdf = ctypes.pointer(sd)
    assert _create(d)[0] == 1


def test_null_handle_calls_fail_cleanly():
    lib = vbd.load_library()
    assert lib.kami_vbd_step(None, ctypes.c_float(0.01), None) == 1
    assert lib.kami_vbd_destroy(None) == 0
    n = ctypes.c_size_t()
    assert lib.kami_vbd_state_size(None, ctypes.byref(n)) == 1
    assert lib.kami_vbd_set_launch_mode(None, 0) == 1
    m = ctypes.c_int32()
    assert lib.kami_vbd_get_launch_mode(None, ctypes.byref(m)) == 1
    assert lib.kami_vbd_step_hair(None, ctypes.c_float(0.01), None, None, None, None) == 1
    assert lib.kami_vbd_strain_limit(None, ctypes.c_float(0.1), None) == 1
    assert lib.kami_vbd_set_tape_window(None, 0, 1) == 1
    assert lib.kami_vbd_restore_tape_window(None, None, 0, vbd.MEM_DEVICE) == 1
    # host registration checks its arguments before any CUDA call
    assert lib.kami_host_register(None, 64) == 1
    assert lib.kami_host_register(ctypes.c_void_p(4096), 0) == 1
    assert lib.kami_host_unregister(None) == 1


def test_batch_rejects_grooms_with_different_solver_settings():
    """The check runs on the host before any device work, so it needs no GPU (1 = KAMI_ERR_INVALID_ARGUMENT)."""
    g0, g1 = synth.cantilever(2, 8), synth.cantilever(3, 6)
    descs = (vbd.Desc * 2)()
    lib = vbd.load_library()
    keep = []
    for d, g in zip(descs, (g0, g1)):
        sb = np.ascontiguousarray(g.strand_begin, np.int32)
        pos = np.ascontiguousarray(g.positions, np.float32)
        keep += [sb, pos]
        assert lib.kami_vbd_desc_init(ctypes.byref(d)) == 0
        d.num_strands, d.strand_begin, d.positions = g.num_strands, sb.ctypes.data, pos.ctypes.data
    descs[1].num_itr = descs[0].num_itr + 1
    h = ctypes.c_void_p()
    assert lib.kami_vbd_batch_create(2, descs, ctypes.byref(h)) == 1
    assert "groom 1 differs from groom 0 in num_itr" in lib.kami_vbd_last_error_string().decode()
    assert lib.kami_vbd_batch_create(0, descs, ctypes.byref(h)) == 1
    descs[1].num_itr = descs[0].num_itr
    descs[1].strand_begin = None
    assert lib.kami_vbd_batch_create(2, descs, ctypes.byref(h)) == 1


def _desc_for(g, lib, keep):
    d = vbd.Desc()
    assert lib.kami_vbd_desc_init(ctypes.byref(d)) == 0
    sb = np.ascontiguousarray(g.strand_begin, np.int32)
    pos = np.ascontiguousarray(g.positions, np.float32)
    keep += [sb, pos]
    d.num_strands, d.strand_begin, d.positions = g.num_strands, sb.ctypes.data, pos.ctypes.data
    return d


def test_hair_hair_settings_are_checked_on_the_host():
    """1 = INVALID_ARGUMENT, 5 = GEOMETRY, 6 = UNSUPPORTED; no device is touched."""
    lib = vbd.load_library()
    keep = []
    h = ctypes.c_void_p()
    g = synth.cantilever(2, 8)
    d = _desc_for(g, lib, keep)
    d.hair_hair = 1
    d.form = vbd.FORMS["fused"]
    assert lib.kami_vbd_create(ctypes.byref(d), ctypes.byref(h)) == 6
    assert "sweep form" in lib.kami_vbd_last_error_string().decode()
    d.form = vbd.FORMS["auto"]
    d.detection_scaler = 1.0  # Sim::uploadMeta: "Detection scaler must be greater than 1."
    assert lib.kami_vbd_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d.detection_scaler = 1.2
    d.barrier_thickness = 0.011  # 2 x 5 mm segments < 2 r + barrier
    assert lib.kami_vbd_create(ctypes.byref(d), ctypes.byref(h)) == 5
    assert "longer segments" in lib.kami_vbd_last_error_string().decode()


def test_desc_defaults_for_hair_hair():
    d = vbd.Desc()
    assert vbd.load_library().kami_vbd_desc_init(ctypes.byref(d)) == 0
    assert d.hair_hair == 0 and d.detection_period == 1 and d.step_limit == 1 and d.velocity_radius == 1
    assert d.barrier_thickness == pytest.approx(2 * 0.95 * 4e-5)  # StableCosseratRodsSolver.cpp:176-180
    assert d.k_collision == pytest.approx(1e-5) and d.k_friction == pytest.approx(5.0)
    assert d.friction_coeff == pytest.approx(0.1) and d.detection_scaler == pytest.approx(1.2)


def test_noalloc_rejects_bad_dt_before_touching_a_device():
    """A NaN or infinite dt, or one needing more than KAMI_MAX_SUBSTEPS substeps of max_h, is an
    argument error found on the host; the (never dereferenced) array pointers need only be non-null."""
    from tests.helpers import NoAllocArgs, bind_noalloc

    lib, step_noalloc = bind_noalloc()
    d = vbd.Desc()
    lib.kami_vbd_desc_init(ctypes.byref(d))
    d.schedule = 0
    d.max_h = 1e-9
    a = NoAllocArgs()
    a.num_vertices, a.num_strands = 64, 2
    for name in ("strand_begin", "positions", "velocities", "last_velocities", "orientations", "rest_darboux",
                 "inv_mass", "rest_length", "stretch_stiffness"):
        setattr(a, name, 256)
    for dt in (float("nan"), float("inf"), -float("inf"), 1.0):  # 1 s / 1 ns = 1e9 substeps
        assert step_noalloc(ctypes.byref(d), ctypes.byref(a), dt, None) == 1, dt
        msg = lib.kami_vbd_last_error_string().decode()
        assert "finite" in msg or "substeps" in msg, msg


def test_connection_indices_are_checked_before_any_device_work():
    """connection_index entries must be -1 or another vertex of the groom; a tie cannot run on the
    fused form (1 = KAMI_ERR_INVALID_ARGUMENT, 6 = KAMI_ERR_UNSUPPORTED)."""
    g = synth.cantilever(2, 8)
    keep = []
    for bad in (8 * 2, -2):
        d = _desc(g, keep)
        conn = np.full(g.num_vertices, -1, np.int32)
        conn[3] = bad
        keep.append(conn)
        d.connection_index = conn.ctypes.data
        rc, msg = _create(d)
        assert rc == 1 and "connection_index[3]" in msg, msg
    conn = np.full(g.num_vertices, -1, np.int32)
    conn[5] = 5  # tied to itself
    keep.append(conn)
    d = _desc(g, keep)
    d.connection_index = conn.ctypes.data
    assert _create(d)[0] == 1
    conn = np.full(g.num_vertices, -1, np.int32)
    conn[7], conn[15] = 15, 7
    keep.append(conn)
    d = _desc(g, keep)
    d.connection_index = conn.ctypes.data
    d.form = 2  # KAMI_FORM_FUSED
    rc, msg = _create(d)
    assert rc == 6 and "connection" in msg, msg
