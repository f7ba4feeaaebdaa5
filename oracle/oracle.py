"""ctypes front-end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (oracle/kami_oracle.cpp) restates the reference's Stable Cosserat Rods
VBD step on the CPU, in FP32 or FP64.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use this module, always as the checker.

``OracleSim`` mirrors YarnBall::Sim as StableCosseratRodsSolver drives it
(src/solvers/StableCosseratRods/StableCosseratRodsSolver.cpp:112-234):
construct from curves, configure, setYoung, pin roots, then advance(dt) + SDF pass.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libkami_oracle.so")
_lib = None

SCHEDULES = {"colour2": 0, "jacobi": 1}

HAS_PREV, HAS_NEXT, HAS_NEXT_ORIENTATION, FIX_ORIENTATION = 1, 2, 4, 8


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("gravity", ctypes.c_float * 3),
        ("damping", ctypes.c_float),
        ("velocity_decay", ctypes.c_float),
        ("acceleration_ratio", ctypes.c_float),
        ("ext_mult", ctypes.c_float),
        ("wind_peak", ctypes.c_float),
        ("wind_y_freq", ctypes.c_float),
        ("wind_z_freq", ctypes.c_float),
        ("wind_time_freq", ctypes.c_float),
        ("wind_sharpness", ctypes.c_float),
        ("num_itr", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("max_h", ctypes.c_float),
        ("sdf_enabled", ctypes.c_int32),
        ("sdf_dims", ctypes.c_int32 * 3),
        ("sdf_min", ctypes.c_float * 3),
        ("sdf_max", ctypes.c_float * 3),
        ("sdf_threshold", ctypes.c_float),
        ("sdf_phi", ctypes.c_void_p),
        ("sdf_grad", ctypes.c_void_p),
        ("body_rot", ctypes.c_float * 4),
        ("body_trans", ctypes.c_float * 3),
        ("num_threads", ctypes.c_int32),
        ("hair_hair", ctypes.c_int32),
        ("radius", ctypes.c_float),
        ("barrier_thickness", ctypes.c_float),
        ("k_collision", ctypes.c_float),
        ("k_friction", ctypes.c_float),
        ("friction_coeff", ctypes.c_float),
        ("detection_scaler", ctypes.c_float),
        ("detection_period", ctypes.c_int32),
        ("step_limit", ctypes.c_int32),
        ("velocity_radius", ctypes.c_int32),
        ("connection", ctypes.c_void_p),
    ]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        for suffix, ct in (("f32", ctypes.c_float), ("f64", ctypes.c_double)):
            fn = getattr(lib, f"oracle_configure_{suffix}")
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                           ctypes.c_float, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                           ctypes.c_float, ctypes.c_int32] + [ctypes.c_void_p] * 6
            fn = getattr(lib, f"oracle_advance_{suffix}")
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int64, ctypes.c_int32] + [ctypes.c_void_p] * 11 + [
                ctypes.c_float]
        lib.oracle_num_threads.restype = ctypes.c_int
        lib.oracle_sdf_bake_f64.restype = ctypes.c_int
        lib.oracle_sdf_bake_f64.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32] + [ctypes.c_void_p] * 6
        lib.oracle_sag_free_f32.restype = ctypes.c_int
        lib.oracle_sag_free_f32.argtypes = [ctypes.c_int32] + [ctypes.c_void_p] * 8 + [ctypes.c_int32]
        lib.oracle_resample_cmr.restype = ctypes.c_int64
        lib.oracle_resample_cmr.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_void_p,
                                            ctypes.c_int64]
        lib.oracle_flop_count.restype = None
        lib.oracle_flop_count.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_strain_limit_f32.restype = None
        lib.oracle_strain_limit_f32.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                                                ctypes.c_void_p]
        lib.oracle_sdf_points_f64.restype = ctypes.c_int
        lib.oracle_sdf_points_f64.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                              ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def configure(groom, radius=40e-6, density=1300.0, stiffness_mode=0, k_stretch=3e3, k_bend=6e-4, pin_roots=True,
              dtype=np.float32):
    """Per-vertex material arrays exactly as Sim::configure + setYoung produce them."""
    lib = load()
    nv = groom.num_vertices
    ns = groom.num_strands
    sb = np.ascontiguousarray(groom.strand_begin, np.int32)
    pos = np.ascontiguousarray(groom.positions, np.float32)
    young = np.ascontiguousarray(groom.strand_young, np.float32)
    dev = np.ascontiguousarray(groom.strand_dev, np.float32)
    out = dict(inv_mass=np.zeros(nv, dtype), l_rest=np.zeros(nv, dtype), k_stretch=np.zeros(nv, dtype),
               flags=np.zeros(nv, np.uint32), q=np.zeros((nv, 4), dtype), q_rest=np.zeros((nv, 4), dtype))
    fn = lib.oracle_configure_f32 if dtype == np.float32 else lib.oracle_configure_f64
    rc = fn(nv, ns, _p(sb), _p(pos), radius, density, stiffness_mode, _p(young), _p(dev), k_stretch, k_bend,
            int(pin_roots), _p(out["inv_mass"]), _p(out["l_rest"]), _p(out["k_stretch"]), _p(out["flags"]),
            _p(out["q"]), _p(out["q_rest"]))
    if rc != 0:
        raise ValueError(f"oracle configure failed with code {rc}")
    return out


class OracleSim:
    """YarnBall::Sim + the SDF pass, restated on the CPU in FP32 or FP64."""

    def __init__(self, groom, *, num_itr=10, max_h=None, gravity=(0.0, 0.0, -9.81), radius=40e-6, density=1300.0,
                 damping=1e-6, velocity_decay=0.05, acceleration_ratio=1.0, ext_mult=1.0, wind=(0.0, 0.0, 0.0, 0.0, 3.0),
                 schedule="colour2", sdf=None, body_rot=(0.0, 0.0, 0.0, 1.0), body_trans=(0.0, 0.0, 0.0),
                 stiffness_mode=0, k_stretch=3e3, k_bend=6e-4, pin_roots=True, dtype=np.float32, num_threads=0,
                 velocities=None, hair_hair=False, barrier_thickness=7.6e-5, k_collision=1e-5, k_friction=5.0,
                 friction_coeff=0.1, detection_scaler=1.2, detection_period=1, step_limit=None, velocity_radius=True,
                 connection_index=None):
        """hair_hair: the hair-hair collision path (EnableHairHairColl); step_limit defaults to it, as
        StableCosseratRodsSolver sets useStepSizeLimit = EnableHairHairColl (.cpp:184).
        connection_index: per vertex the vertex it is tied to by a connection spring, or -1."""
        self.dtype = dtype
        self.lib = load()
        self.groom = groom
        self.nv = groom.num_vertices
        self.ns = groom.num_strands
        self.sb = np.ascontiguousarray(groom.strand_begin, np.int32)
        m = configure(groom, radius, density, stiffness_mode, k_stretch, k_bend, pin_roots, dtype)
        self.inv_mass, self.l_rest, self.k_stretch = m["inv_mass"], m["l_rest"], m["k_stretch"]
        self.flags, self.q, self.q_rest = m["flags"], m["q"], m["q_rest"]
        self.x = np.ascontiguousarray(groom.positions, dtype).copy()
        self.v = np.zeros((self.nv, 3), dtype) if velocities is None else np.ascontiguousarray(velocities, dtype).copy()
        self.v_last = np.zeros((self.nv, 3), dtype)
        max_h = 4e-4 if max_h is None else max_h
        # meta.h starts at maxH (YBSimulator.cu:85), lastH is taken from it on the first advance
        # h, lastH, time, substep counter (Sim::stepCounter, step.cpp:52)
        self.clock = np.array([np.float32(max_h), 0.0, 0.0, 0.0], np.float64)
        p = OracleParams()
        p.gravity[:] = gravity
        p.damping, p.velocity_decay, p.acceleration_ratio, p.ext_mult = damping, velocity_decay, acceleration_ratio, ext_mult
        p.wind_peak, p.wind_y_freq, p.wind_z_freq, p.wind_time_freq, p.wind_sharpness = wind
        p.num_itr = num_itr
        p.schedule = SCHEDULES[schedule]
        p.max_h = max_h
        p.num_threads = num_threads
        self._sdf_keep = None
        if sdf is not None:
            phi = np.ascontiguousarray(sdf.phi, np.float32)
            grad = np.ascontiguousarray(sdf.grad, np.float32)
            self._sdf_keep = (phi, grad)
            p.sdf_enabled = 1
            p.sdf_dims[:] = sdf.dims
            p.sdf_min[:] = sdf.grid_min
            p.sdf_max[:] = sdf.grid_max
            p.sdf_threshold = sdf.threshold
            p.sdf_phi = phi.ctypes.data
            p.sdf_grad = grad.ctypes.data
        p.body_rot[:] = body_rot
        p.body_trans[:] = body_trans
        p.hair_hair = int(bool(hair_hair))
        p.radius = radius
        p.barrier_thickness, p.k_collision, p.k_friction = barrier_thickness, k_collision, k_friction
        p.friction_coeff, p.detection_scaler, p.detection_period = friction_coeff, detection_scaler, detection_period
        p.step_limit = int(bool(hair_hair if step_limit is None else step_limit))
        p.velocity_radius = int(bool(velocity_radius))
        self._conn_keep = None
        if connection_index is not None:
            self._conn_keep = np.ascontiguousarray(connection_index, np.int32)
            p.connection = self._conn_keep.ctypes.data
        self.params = p

    def set_body_transform(self, rot, trans):
        self.params.body_rot[:] = rot
        self.params.body_trans[:] = trans

    def advance(self, dt):
        fn = self.lib.oracle_advance_f32 if self.dtype == np.float32 else self.lib.oracle_advance_f64
        rc = fn(ctypes.byref(self.params), self.nv, self.ns, _p(self.sb), _p(self.inv_mass), _p(self.l_rest),
                _p(self.k_stretch), _p(self.flags), _p(self.q_rest), _p(self.x), _p(self.v), _p(self.v_last),
                _p(self.q), _p(self.clock), dt)
        if rc == 4:
            raise RuntimeError("a segment has more than 16 contacts (MAX_COLLISIONS_PER_SEGMENT exceeded)")
        if rc != 0:
            raise RuntimeError(f"oracle advance failed with code {rc}")

    def state(self):
        return dict(x=self.x.copy(), v=self.v.copy(), v_last=self.v_last.copy(), q=self.q.copy(),
                    clock=self.clock.copy())

    def load_state(self, st):
        self.x[...] = st["x"]
        self.v[...] = st["v"]
        self.v_last[...] = st["v_last"]
        self.q[...] = st["q"]
        self.clock[...] = st["clock"]


def strain_limit(x, strand_begin, rest_lengths, strain_error=0.1):
    """The SDF solver's StrainLimiting (cudaSDFCollision.cu:176-199) on packed strands, FP32: returns
    the corrected positions (rest_lengths[i]: rest length of the segment starting at vertex i)."""
    lib = load()
    out = np.ascontiguousarray(x, np.float32).copy()
    sb = np.ascontiguousarray(strand_begin, np.int32)
    l0 = np.ascontiguousarray(rest_lengths, np.float32)
    lib.oracle_strain_limit_f32(len(sb) - 1, _p(sb), _p(l0), float(strain_error), _p(out))
    return out


def twist_angles(q_ref, q_new):
    """Twist of q_new relative to q_ref about the material axis e_x: 2 atan2(dq.xyz . e_x, dq.w), dq = q_ref^-1 q_new."""
    a = np.asarray(q_ref, np.float64)
    b = np.asarray(q_new, np.float64)
    ax, ay, az, aw = -a[:, 0], -a[:, 1], -a[:, 2], a[:, 3]
    bx, by, bz, bw = b[:, 0], b[:, 1], b[:, 2], b[:, 3]
    # (conj(a) * b).x and .w
    dx = aw * bx + bw * ax + (ay * bz - by * az)
    dw = aw * bw - (ax * bx + ay * by + az * bz)
    ang = 2.0 * np.arctan2(dx, dw)
    return (ang + np.pi) % (2.0 * np.pi) - np.pi


def sdf_bake(vertices, triangles, dims, grid_min, grid_max):
    """FP64 body SDF of a closed triangle mesh on the grid nodes grid_min + ds (i, j, k):
    (phi [nz, ny, nx], grad [nz, ny, nx, 3])."""
    lib = load()
    v = np.ascontiguousarray(vertices, np.float32)
    t = np.ascontiguousarray(triangles, np.int32)
    d = np.asarray(dims, np.int32)
    lo = np.asarray(grid_min, np.float32)
    hi = np.asarray(grid_max, np.float32)
    nx, ny, nz = (int(a) for a in dims)
    phi = np.zeros((nz, ny, nx), np.float64)
    grad = np.zeros((nz, ny, nx, 3), np.float64)
    rc = lib.oracle_sdf_bake_f64(v.shape[0], _p(v), t.shape[0], _p(t), _p(d), _p(lo), _p(hi), _p(phi), _p(grad))
    if rc != 0:
        raise RuntimeError("oracle SDF bake failed")
    return phi, grad


def sdf_points(vertices, triangles, points):
    """FP64 signed distance to a closed triangle mesh at float32-rounded points [..., 3]."""
    lib = load()
    v = np.ascontiguousarray(vertices, np.float32)
    t = np.ascontiguousarray(triangles, np.int32)
    p = np.ascontiguousarray(np.asarray(points, np.float32), np.float64).reshape(-1, 3)
    out = np.zeros(p.shape[0], np.float64)
    lib.oracle_sdf_points_f64(v.shape[0], _p(v), t.shape[0], _p(t), p.shape[0], _p(p), _p(out))
    return out.reshape(np.asarray(points).shape[:-1])


def sag_free(groom, material, gravity, iterations):
    """Sim::SagFree restated (FP32 material): returns new (l_rest, q, q_rest); `material` is
    configure(..., dtype=float32) with roots pinned."""
    lib = load()
    sb = np.ascontiguousarray(groom.strand_begin, np.int32)
    pos = np.ascontiguousarray(groom.positions, np.float32)
    g = np.asarray(gravity, np.float32)
    lr = np.array(material["l_rest"], np.float32)
    q = np.array(material["q"], np.float32)
    qr = np.array(material["q_rest"], np.float32)
    im = np.ascontiguousarray(material["inv_mass"], np.float32)
    ks = np.ascontiguousarray(material["k_stretch"], np.float32)
    lib.oracle_sag_free_f32(groom.num_strands, _p(sb), _p(pos), _p(g), _p(im), _p(ks), _p(lr), _p(q), _p(qr), iterations)
    return lr, q, qr


def resample_cmr(points, target):
    """Resample::resampleCMR(curve, 1, n - 2, target) restated: the resampled strand (float32 [m, 3])."""
    lib = load()
    p = np.ascontiguousarray(points, np.float32)
    cap = 5 * p.shape[0] + 16
    out = np.zeros((cap, 3), np.float32)
    # the target is a float setting (JsonParams::ResampleLen) widened to double, as BuildYarnBallHair passes it
    n = lib.oracle_resample_cmr(_p(p), p.shape[0], float(np.float32(target)), _p(out), cap)
    if n < 0:
        raise ValueError("a strand needs at least 4 points")
    return out[:min(n, cap)].copy()


def flop_count():
    """(position, orientation) FLOPs of one update of the reference algorithm -- cosseratItr for an
    interior vertex and quaternionLambdaItr for a segment with both neighbours -- counted by running
    the oracle's templated updates on an op-counting scalar (+ - * / sqrt count one; an FMA two)."""
    lib = load()
    a, b = ctypes.c_int64(), ctypes.c_int64()
    lib.oracle_flop_count(ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value
