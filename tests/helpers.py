"""Shared set-up for the tests: one settings dict drives both the CPU oracle and the GPU solver."""
import ctypes

import numpy as np

from kamisimulator_b200 import synth

POS_TOL = 1e-5  # m, per step
TWIST_TOL = 1e-5  # rad, per step


def oracle_sim(groom, settings, dtype=np.float32, velocities=None):
    from oracle.oracle import OracleSim

    s = dict(settings)
    form = s.pop("form", None)  # the oracle has a single form
    del form
    return OracleSim(groom, dtype=dtype, velocities=velocities, **s)


def gpu_solver(groom, settings, form="auto", velocities=None):
    from kamisimulator_b200.vbd import Solver

    s = dict(settings)
    s.pop("num_threads", None)
    s.setdefault("form", form)
    return Solver(groom, velocities=velocities, **s)


def soft_settings(**kw):
    """Soft, fast-moving rods so that a 1e-5 m bound constrains every term of the update."""
    s = dict(num_itr=6, max_h=1.0 / 60.0, gravity=(0.3, -0.4, -9.81), radius=40e-6, density=1300.0, damping=1e-6,
             velocity_decay=0.05, schedule="colour2")
    s.update(kw)
    return s


def soft_groom(num_strands=96, lengths=(8, 40), seed=11, young_scale=1e-4):
    rng = np.random.default_rng(seed)
    lens = rng.integers(lengths[0], lengths[1] + 1, num_strands)
    g = synth.groom_strands(rng, lens)
    g.strand_young = (g.strand_young * young_scale).astype(np.float32)
    g.strand_dev = rng.uniform(0.05, 1.0, num_strands).astype(np.float32)
    return g


def random_velocities(groom, scale=0.3, seed=7):
    rng = np.random.default_rng(seed)
    v = rng.normal(0.0, scale, (groom.num_vertices, 3)).astype(np.float32)
    v[groom.strand_begin[:-1]] = 0.0
    return v


class NoAllocArgs(ctypes.Structure):
    """kami_vbd_noalloc_args (include/kami_vbd.h)."""
    _fields_ = [("num_vertices", ctypes.c_int64), ("num_strands", ctypes.c_int32),
                ("strand_begin", ctypes.c_void_p), ("positions", ctypes.c_void_p), ("velocities", ctypes.c_void_p),
                ("last_velocities", ctypes.c_void_p), ("orientations", ctypes.c_void_p),
                ("rest_darboux", ctypes.c_void_p), ("inv_mass", ctypes.c_void_p), ("rest_length", ctypes.c_void_p),
                ("stretch_stiffness", ctypes.c_void_p), ("clock", ctypes.c_float * 3)]


def bind_noalloc():
    """The library and its kami_vbd_step_noalloc entry point with argument types set."""
    from kamisimulator_b200 import vbd

    lib = vbd.load_library()
    fn = lib.kami_vbd_step_noalloc
    fn.argtypes = [ctypes.POINTER(vbd.Desc), ctypes.POINTER(NoAllocArgs), ctypes.c_float, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib, fn
