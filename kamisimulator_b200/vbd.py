"""Python binding of the solver's C ABI (include/kami_vbd.h) through ctypes.

``Solver`` mirrors the calls KamiSimulator makes on its StableCosseratRods solver
(src/solvers/Solver.h:61-84, StableCosseratRodsSolver.cpp:33-277): construct from a
groom and settings, ``step(dt)`` per internal step, ``set``/``get`` positions and
velocities for Upload/DownloadHair.  Arrays cross the boundary as float32 numpy
arrays (host) or torch CUDA tensors (device).  There is no CPU path: without the
compiled library every call raises.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libkami_vbd.so")

KAMI_OK = 0
STATUS_NAMES = {0: "KAMI_OK", 1: "KAMI_ERR_INVALID_ARGUMENT", 2: "KAMI_ERR_CUDA", 3: "KAMI_ERR_OUT_OF_MEMORY",
                4: "KAMI_ERR_NONFINITE", 5: "KAMI_ERR_GEOMETRY", 6: "KAMI_ERR_UNSUPPORTED", 7: "KAMI_ERR_TIMEOUT",
                8: "KAMI_ERR_STATE", 9: "KAMI_ERR_CONTACTS", 10: "KAMI_ERR_IO"}
SCHEDULES = {"colour2": 0, "jacobi": 1}
FORMS = {"auto": 0, "sweep": 1, "fused": 2}
MEM_HOST, MEM_DEVICE = 0, 1

# Every symbol declared in include/kami_vbd.h.
EXPORTED = [
    "kami_vbd_desc_init", "kami_vbd_create", "kami_vbd_destroy", "kami_vbd_get_sizes",
    "kami_vbd_set_positions_velocities", "kami_vbd_get_positions_velocities", "kami_vbd_get_orientations",
    "kami_vbd_set_orientations", "kami_vbd_get_rest_darboux", "kami_vbd_set_rest_darboux",
    "kami_vbd_set_body_transform", "kami_vbd_step", "kami_vbd_synchronize", "kami_vbd_state_size",
    "kami_vbd_get_state", "kami_vbd_set_state", "kami_vbd_last_error_string", "kami_vbd_version",
    "kami_vbd_step_n", "kami_vbd_set_tuning", "kami_vbd_get_tuning", "kami_vbd_autotune",
    "kami_vbd_tape_reserve", "kami_vbd_get_tile_count", "kami_vbd_set_tape_window", "kami_vbd_step_record", "kami_vbd_backward", "kami_vbd_get_rest_darboux_grad",
    "kami_vbd_zero_rest_darboux_grad", "kami_vbd_batch_create", "kami_vbd_batch_count", "kami_vbd_batch_groom_range",
    "kami_vbd_batch_step", "kami_vbd_set_hair_layout", "kami_vbd_upload_hair", "kami_vbd_download_hair",
    "kami_usc_info", "kami_usc_read", "kami_usc_write", "kami_sdf_bake", "kami_vbd_sag_free",
    "kami_hair_subdivide", "kami_hair_resample", "kami_vbd_step_host", "kami_vbd_get_tiles_per_group",
    "kami_vbd_set_launch_mode", "kami_vbd_get_launch_mode", "kami_vbd_step_hair", "kami_host_register",
    "kami_host_unregister", "kami_vbd_strain_limit", "kami_vbd_restore_tape_window",
]


class KamiError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class SdfDesc(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int32 * 3), ("grid_min", ctypes.c_float * 3), ("grid_max", ctypes.c_float * 3),
                ("threshold", ctypes.c_float), ("phi", ctypes.c_void_p), ("grad", ctypes.c_void_p)]


class Desc(ctypes.Structure):
    _fields_ = [
        ("num_strands", ctypes.c_int32),
        ("strand_begin", ctypes.c_void_p),
        ("positions", ctypes.c_void_p),
        ("velocities", ctypes.c_void_p),
        ("radius", ctypes.c_float),
        ("density", ctypes.c_float),
        ("stiffness_mode", ctypes.c_int32),
        ("young", ctypes.c_float),
        ("deviation", ctypes.c_float),
        ("strand_young", ctypes.c_void_p),
        ("strand_deviation", ctypes.c_void_p),
        ("k_stretch", ctypes.c_float),
        ("k_bend", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
        ("damping", ctypes.c_float),
        ("velocity_decay", ctypes.c_float),
        ("acceleration_ratio", ctypes.c_float),
        ("external_force_multiplier", ctypes.c_float),
        ("wind_peak", ctypes.c_float),
        ("wind_y_freq", ctypes.c_float),
        ("wind_z_freq", ctypes.c_float),
        ("wind_time_freq", ctypes.c_float),
        ("wind_sharpness", ctypes.c_float),
        ("num_itr", ctypes.c_int32),
        ("max_h", ctypes.c_float),
        ("schedule", ctypes.c_int32),
        ("form", ctypes.c_int32),
        ("pin_roots", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("sdf", ctypes.POINTER(SdfDesc)),
        ("slots_per_lane", ctypes.c_int32),
        ("warps_per_block", ctypes.c_int32),
        ("hair_hair", ctypes.c_int32),
        ("barrier_thickness", ctypes.c_float),
        ("k_collision", ctypes.c_float),
        ("k_friction", ctypes.c_float),
        ("friction_coeff", ctypes.c_float),
        ("detection_scaler", ctypes.c_float),
        ("detection_period", ctypes.c_int32),
        ("step_limit", ctypes.c_int32),
        ("velocity_radius", ctypes.c_int32),
        ("sag_free_itr", ctypes.c_int32),
        ("connection_index", ctypes.c_void_p),
    ]


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads the compiled library; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"the CUDA solver library {path} is missing; build it with __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    sig = {
        "kami_vbd_desc_init": [ctypes.POINTER(Desc)],
        "kami_vbd_create": [ctypes.POINTER(Desc), ctypes.POINTER(vp)],
        "kami_vbd_batch_create": [i32, ctypes.POINTER(Desc), ctypes.POINTER(vp)],
        "kami_vbd_batch_count": [vp, ctypes.POINTER(i32)],
        "kami_vbd_batch_groom_range": [vp, i32, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i64),
                                       ctypes.POINTER(i64)],
        "kami_vbd_batch_step": [vp, f32, i32, vp, vp],
        "kami_vbd_set_hair_layout": [vp, i32, i32, vp],
        "kami_vbd_upload_hair": [vp, vp, vp, i32],
        "kami_vbd_download_hair": [vp, vp, vp, i32],
        "kami_sdf_bake": [vp, i32, vp, i32, vp, vp, vp, vp, vp, i32, i32],
        "kami_vbd_sag_free": [vp, i32],
        "kami_hair_subdivide": [i32, vp, i32, vp, vp, i32, vp, vp, vp, i32],
        "kami_hair_resample": [i32, vp, i32, vp, f32, i32],
        "kami_usc_info": [ctypes.c_char_p, ctypes.POINTER(i32), ctypes.POINTER(i64), ctypes.POINTER(i32)],
        "kami_usc_read": [ctypes.c_char_p, i32, vp, vp],
        "kami_usc_write": [ctypes.c_char_p, i32, vp, i32, vp],
        "kami_vbd_destroy": [vp],
        "kami_vbd_get_sizes": [vp, ctypes.POINTER(i64), ctypes.POINTER(i32), ctypes.POINTER(i32)],
        "kami_vbd_set_positions_velocities": [vp, vp, vp, i32],
        "kami_vbd_get_positions_velocities": [vp, vp, vp, i32],
        "kami_vbd_get_orientations": [vp, vp, i32],
        "kami_vbd_set_orientations": [vp, vp, i32],
        "kami_vbd_get_rest_darboux": [vp, vp, i32],
        "kami_vbd_set_rest_darboux": [vp, vp, i32],
        "kami_vbd_set_body_transform": [vp, vp, vp],
        "kami_vbd_step": [vp, f32, vp],
        "kami_vbd_step_host": [vp, f32, vp, vp, vp, vp],
        "kami_vbd_get_tiles_per_group": [vp, ctypes.POINTER(i32)],
        "kami_vbd_synchronize": [vp],
        "kami_vbd_strain_limit": [vp, f32, vp],
        "kami_vbd_state_size": [vp, ctypes.POINTER(ctypes.c_size_t)],
        "kami_vbd_get_state": [vp, vp, ctypes.c_size_t, i32],
        "kami_vbd_set_state": [vp, vp, ctypes.c_size_t, i32],
        "kami_vbd_step_n": [vp, f32, i32, vp, vp],
        "kami_vbd_set_tuning": [vp, i32, i32, i32, i32],
        "kami_vbd_get_tuning": [vp, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32)],
        "kami_vbd_set_launch_mode": [vp, i32],
        "kami_vbd_step_hair": [vp, f32, vp, vp, vp, vp],
        "kami_host_register": [vp, ctypes.c_size_t],
        "kami_host_unregister": [vp],
        "kami_vbd_get_launch_mode": [vp, ctypes.POINTER(i32)],
        "kami_vbd_autotune": [vp, f32, i32, ctypes.POINTER(i32), ctypes.POINTER(ctypes.c_double)],
        "kami_vbd_tape_reserve": [vp, i32, i64],
        "kami_vbd_get_tile_count": [vp, ctypes.POINTER(i64)],
        "kami_vbd_set_tape_window": [vp, i64, i64],
        "kami_vbd_restore_tape_window": [vp, vp, ctypes.c_size_t, i32],
        "kami_vbd_step_record": [vp, f32, vp],
        "kami_vbd_backward": [vp, vp, vp, vp, vp, i32, vp],
        "kami_vbd_get_rest_darboux_grad": [vp, vp, i32],
        "kami_vbd_zero_rest_darboux_grad": [vp],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.kami_vbd_last_error_string.restype = ctypes.c_char_p
    lib.kami_vbd_last_error_string.argtypes = []
    lib.kami_vbd_version.restype = ctypes.c_char_p
    lib.kami_vbd_version.argtypes = []
    _lib = lib
    return lib


def _check(rc):
    if rc != KAMI_OK:
        msg = _lib.kami_vbd_last_error_string().decode()
        raise KamiError(rc, msg)


def _ptr(a):
    """Host numpy array or torch tensor -> (pointer, memory kind)."""
    if a is None:
        return None, MEM_HOST
    if hasattr(a, "data_ptr"):
        if a.is_cuda:
            return ctypes.c_void_p(a.data_ptr()), MEM_DEVICE
        return ctypes.c_void_p(a.data_ptr()), MEM_HOST
    return a.ctypes.data_as(ctypes.c_void_p), MEM_HOST


def torch_float32():
    import torch

    return torch.float32


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


class Solver:
    """One StableCosseratRods solver instance on the GPU (a YarnBall::Sim plus its SDF pass)."""

    def __init__(self, groom, *, num_itr=8, max_h=4e-4, gravity=(0.0, -9.8, 0.0), radius=4e-5, density=1300.0,
                 damping=1e-6, velocity_decay=0.05, acceleration_ratio=1.0, ext_mult=1.0,
                 wind=(0.0, 1.0, 0.7, 0.4, 3.0), schedule="colour2", form="auto", sdf=None, stiffness_mode=0,
                 young=5.0, deviation=1.0, per_strand=True, k_stretch=3e3, k_bend=6e-4, pin_roots=True,
                 velocities=None, device=-1, slots_per_lane=0, warps_per_block=0, hair_hair=False,
                 barrier_thickness=None, k_collision=None, k_friction=None, friction_coeff=None,
                 detection_scaler=None, detection_period=None, step_limit=None, velocity_radius=None,
                 sag_free_itr=0, connection_index=None):
        """groom: one groom (kami_vbd_create) or a list of grooms (kami_vbd_batch_create, one handle
        stepping all of them; velocities and connection_index are then None or lists with one entry
        per groom).  connection_index: per vertex, the vertex of the same groom it is tied to by a
        connection spring (Vertex::connectionIndex), or -1."""
        self.lib = load_library()
        self._h = None
        self._tape_rollout = None  # the autograd rollout whose steps the tape holds (autograd.py)
        grooms = list(groom) if isinstance(groom, (list, tuple)) else [groom]
        if velocities is None or not isinstance(groom, (list, tuple)):
            velocities = [velocities] * len(grooms)
        if connection_index is None or not isinstance(groom, (list, tuple)):
            connection_index = [connection_index] * len(grooms)
        keep = []
        sdf_ptr = None
        if sdf is not None:
            phi = np.ascontiguousarray(sdf.phi, np.float32)
            grad = np.ascontiguousarray(sdf.grad, np.float32)
            sd_ = SdfDesc()
            sd_.dims[:] = sdf.dims
            sd_.grid_min[:] = sdf.grid_min
            sd_.grid_max[:] = sdf.grid_max
            sd_.threshold = sdf.threshold
            sd_.phi = phi.ctypes.data
            sd_.grad = grad.ctypes.data
            keep += [phi, grad, sd_]
            sdf_ptr = ctypes.pointer(sd_)
        descs = (Desc * len(grooms))()
        for d, g, v, ci in zip(descs, grooms, velocities, connection_index):
            sb = np.ascontiguousarray(g.strand_begin, np.int32)
            pos = _f32(g.positions)
            vel = None if v is None else _f32(v)
            sy = np.ascontiguousarray(g.strand_young, np.float32) if per_strand else None
            sd = np.ascontiguousarray(g.strand_dev, np.float32) if per_strand else None
            keep += [sb, pos, vel, sy, sd]
            _check(self.lib.kami_vbd_desc_init(ctypes.byref(d)))
            d.num_strands = g.num_strands
            d.strand_begin = sb.ctypes.data
            d.positions = pos.ctypes.data
            d.velocities = vel.ctypes.data if vel is not None else None
            d.radius, d.density = radius, density
            d.stiffness_mode = stiffness_mode
            d.young, d.deviation = young, deviation
            d.strand_young = sy.ctypes.data if sy is not None else None
            d.strand_deviation = sd.ctypes.data if sd is not None else None
            d.k_stretch, d.k_bend = k_stretch, k_bend
            d.gravity[:] = gravity
            d.damping, d.velocity_decay, d.acceleration_ratio = damping, velocity_decay, acceleration_ratio
            d.external_force_multiplier = ext_mult
            d.wind_peak, d.wind_y_freq, d.wind_z_freq, d.wind_time_freq, d.wind_sharpness = wind
            d.num_itr = num_itr
            d.max_h = max_h
            d.schedule = SCHEDULES[schedule]
            d.form = FORMS[form]
            d.pin_roots = int(pin_roots)
            d.device = device
            d.slots_per_lane = slots_per_lane
            d.warps_per_block = warps_per_block
            d.sdf = sdf_ptr
            d.hair_hair = int(bool(hair_hair))
            d.sag_free_itr = int(sag_free_itr)
            if ci is not None:
                ci = np.ascontiguousarray(ci, np.int32)
                if ci.shape != (g.num_vertices,):
                    raise ValueError("connection_index needs one entry per vertex")
                keep.append(ci)
                d.connection_index = ci.ctypes.data
            for name, val in (("barrier_thickness", barrier_thickness), ("k_collision", k_collision),
                              ("k_friction", k_friction), ("friction_coeff", friction_coeff),
                              ("detection_scaler", detection_scaler), ("detection_period", detection_period),
                              ("step_limit", step_limit), ("velocity_radius", velocity_radius)):
                if val is not None:
                    setattr(d, name, val)
        h = ctypes.c_void_p()
        if isinstance(groom, (list, tuple)):
            _check(self.lib.kami_vbd_batch_create(len(grooms), descs, ctypes.byref(h)))
        else:
            _check(self.lib.kami_vbd_create(ctypes.byref(descs[0]), ctypes.byref(h)))
        self._h = h
        nv, ns, c = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
        _check(self.lib.kami_vbd_get_sizes(h, ctypes.byref(nv), ctypes.byref(ns), ctypes.byref(c)))
        self.num_vertices, self.num_strands, self.slots_per_lane = nv.value, ns.value, c.value
        ng = ctypes.c_int32()
        _check(self.lib.kami_vbd_batch_count(h, ctypes.byref(ng)))
        self.num_grooms = ng.value
        self.max_h = float(np.float32(max_h))
        self.num_itr = int(num_itr)
        del keep

    def substeps(self, dt):
        """Substeps of one step of dt, ceil(dt / max_h) in float as kami_vbd_step takes them."""
        return max(1, math.ceil(np.float32(dt) / np.float32(self.max_h)))

    def groom_range(self, groom):
        """(first strand, strands, first vertex, vertices) of one groom of a batch handle."""
        s0, ns, v0, nv = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        _check(self.lib.kami_vbd_batch_groom_range(self._h, groom, ctypes.byref(s0), ctypes.byref(ns),
                                                   ctypes.byref(v0), ctypes.byref(nv)))
        return s0.value, ns.value, v0.value, nv.value

    def sag_free(self, iterations=1):
        """kami_vbd_sag_free: sag-free rest lengths and rest angles under the handle's gravity."""
        _check(self.lib.kami_vbd_sag_free(self._h, iterations))

    def set_hair_layout(self, hair_strands, max_verts, strand_refs=None):
        """The padded Hair arrays ([hair_strands][max_verts] xyz) the solver reads and writes;
        strand_refs[s]: the Hair strand of solver strand s (None: the identity)."""
        refs = None if strand_refs is None else np.ascontiguousarray(strand_refs, np.int32)
        _check(self.lib.kami_vbd_set_hair_layout(self._h, hair_strands, max_verts,
                                                 None if refs is None else refs.ctypes.data_as(ctypes.c_void_p)))

    def upload_hair(self, x=None, v=None):
        """UploadHair from padded arrays (numpy host arrays or torch CUDA tensors)."""
        if x is not None and not hasattr(x, "data_ptr"):
            x = _f32(x)
        if v is not None and not hasattr(v, "data_ptr"):
            v = _f32(v)
        px, mx = _ptr(x)
        pv, mv = _ptr(v)
        _check(self.lib.kami_vbd_upload_hair(self._h, px, pv, mx if x is not None else mv))

    def step_hair(self, dt, x_in=None, v_in=None, x_out=None, v_out=None):
        """kami_vbd_step_hair on padded Hair arrays (host float32, (hair_strands, max_verts, 3)):
        upload (if x_in), step, download (if x_out), in one launch when the arrays are page-locked."""
        p = [_ptr(a)[0] for a in (x_in, v_in, x_out, v_out)]
        _check(self.lib.kami_vbd_step_hair(self._h, ctypes.c_float(dt), *p))

    def download_hair(self, x=None, v=None):
        """DownloadHair into padded arrays, in place (entries the solver does not own are kept)."""
        px, mx = _ptr(x)
        pv, mv = _ptr(v)
        _check(self.lib.kami_vbd_download_hair(self._h, px, pv, mx if x is not None else mv))

    def batch_step(self, dt, n, body_transforms=None, stream=None):
        """kami_vbd_batch_step: every groom of the handle, n steps."""
        s = None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        bt = None if body_transforms is None else _f32(body_transforms, (-1, 7))
        if bt is not None and bt.shape[0] != n:
            raise ValueError("body_transforms needs one row per step")
        _check(self.lib.kami_vbd_batch_step(self._h, ctypes.c_float(dt), n,
                                            None if bt is None else bt.ctypes.data_as(ctypes.c_void_p), s))

    # -- lifecycle
    def close(self):
        if self._h is not None:
            self.lib.kami_vbd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- stepping
    def step(self, dt, stream=None):
        s = None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        _check(self.lib.kami_vbd_step(self._h, ctypes.c_float(dt), s))

    def step_n(self, dt, n, body_transforms=None, stream=None):
        """n steps of dt; body_transforms: (n, 7) rotation xyzw + translation per step, or None."""
        s = None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        bt = None
        if body_transforms is not None:
            bt = _f32(body_transforms, (n, 7))
        _check(self.lib.kami_vbd_step_n(self._h, ctypes.c_float(dt), n,
                                        bt.ctypes.data_as(ctypes.c_void_p) if bt is not None else None, s))

    def set_tuning(self, slots_per_lane=0, warps_per_block=0, steps_per_launch=0, register_cap=0):
        _check(self.lib.kami_vbd_set_tuning(self._h, slots_per_lane, warps_per_block, steps_per_launch, register_cap))
        self.slots_per_lane = self.get_tuning()[0]

    def get_tuning(self):
        c, w, f, r = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _check(self.lib.kami_vbd_get_tuning(self._h, ctypes.byref(c), ctypes.byref(w), ctypes.byref(f),
                                            ctypes.byref(r)))
        return c.value, w.value, f.value, r.value

    def set_launch_mode(self, mode):
        """kami_vbd_set_launch_mode: 0 (hardware-scheduled tile grid) or 1 (persistent resident CTAs)."""
        _check(self.lib.kami_vbd_set_launch_mode(self._h, int(mode)))

    def get_launch_mode(self):
        m = ctypes.c_int32()
        _check(self.lib.kami_vbd_get_launch_mode(self._h, ctypes.byref(m)))
        return m.value

    def autotune(self, dt, trial_steps=16):
        """Returns ((slots_per_lane, warps_per_block, steps_per_launch, register_cap), vertex-iters/s)."""
        best = (ctypes.c_int32 * 4)()
        rate = ctypes.c_double()
        _check(self.lib.kami_vbd_autotune(self._h, ctypes.c_float(dt), trial_steps, best, ctypes.byref(rate)))
        self.slots_per_lane = best[0]
        return tuple(best), rate.value

    def synchronize(self):
        _check(self.lib.kami_vbd_synchronize(self._h))

    def strain_limit(self, strain_error=0.1, stream=None):
        """kami_vbd_strain_limit: the SDF solver's strain limiting (cudaSDFCollision.cu:176-199), run
        after a step as SDFBodyCollisionSolver::SolveNextStep runs it after its SDF pass (default
        StrainError 0.1, SDFBodyCollisionSolver.h:26)."""
        s = None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        _check(self.lib.kami_vbd_strain_limit(self._h, ctypes.c_float(strain_error), s))

    def set_body_transform(self, rot, trans):
        r = (ctypes.c_float * 4)(*rot)
        t = (ctypes.c_float * 3)(*trans)
        _check(self.lib.kami_vbd_set_body_transform(self._h, r, t))

    # -- boundary data
    def set_positions_velocities(self, x=None, v=None):
        if x is not None and not hasattr(x, "data_ptr"):
            x = _f32(x, (-1, 3))
        if v is not None and not hasattr(v, "data_ptr"):
            v = _f32(v, (-1, 3))
        px, mx = _ptr(x)
        pv, mv = _ptr(v)
        mem = mx if x is not None else mv
        _check(self.lib.kami_vbd_set_positions_velocities(self._h, px, pv, mem))

    def get_positions_velocities(self, x_out=None, v_out=None):
        if x_out is None and v_out is None:
            x_out = np.empty((self.num_vertices, 3), np.float32)
            v_out = np.empty((self.num_vertices, 3), np.float32)
        px, mx = _ptr(x_out)
        pv, mv = _ptr(v_out)
        _check(self.lib.kami_vbd_get_positions_velocities(self._h, px, pv, mx if x_out is not None else mv))
        return x_out, v_out

    def step_host(self, dt, x, v, x_out=None, v_out=None):
        """One frame from host arrays to host arrays (kami_vbd_step_host): upload positions and
        velocities, step, download; pipelined over strand groups.  x_out / v_out default to x / v
        (updated in place).  Pinned torch CPU tensors let the copies run asynchronously."""
        x_out = x if x_out is None else x_out
        v_out = v if v_out is None else v_out
        for a in (x, v, x_out, v_out):
            if hasattr(a, "data_ptr"):
                if a.is_cuda or a.dtype != torch_float32() or not a.is_contiguous():
                    raise ValueError("step_host takes contiguous float32 host arrays")
            elif a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("step_host takes contiguous float32 host arrays")
            n = a.numel() if hasattr(a, "numel") else a.size
            if n != 3 * self.num_vertices:
                raise ValueError(f"step_host arrays hold 3 x {self.num_vertices} floats, got {n}")
        ptrs = [_ptr(a)[0] for a in (x, v, x_out, v_out)]
        _check(self.lib.kami_vbd_step_host(self._h, ctypes.c_float(dt), *ptrs))
        return x_out, v_out

    def get_orientations(self, out=None):
        out = np.empty((self.num_vertices, 4), np.float32) if out is None else out
        p, m = _ptr(out)
        _check(self.lib.kami_vbd_get_orientations(self._h, p, m))
        return out

    def set_orientations(self, q):
        q = q if hasattr(q, "data_ptr") else _f32(q, (-1, 4))
        p, m = _ptr(q)
        _check(self.lib.kami_vbd_set_orientations(self._h, p, m))

    def get_rest_darboux(self, out=None):
        out = np.empty((self.num_vertices, 4), np.float32) if out is None else out
        p, m = _ptr(out)
        _check(self.lib.kami_vbd_get_rest_darboux(self._h, p, m))
        return out

    def set_rest_darboux(self, qr):
        qr = qr if hasattr(qr, "data_ptr") else _f32(qr, (-1, 4))
        p, m = _ptr(qr)
        _check(self.lib.kami_vbd_set_rest_darboux(self._h, p, m))

    def state_size(self):
        n = ctypes.c_size_t()
        _check(self.lib.kami_vbd_state_size(self._h, ctypes.byref(n)))
        return n.value

    def get_state(self):
        buf = np.empty(self.state_size() // 4, np.float32)
        _check(self.lib.kami_vbd_get_state(self._h, buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes, MEM_HOST))
        return buf

    def set_state(self, buf):
        buf = np.ascontiguousarray(buf, np.float32)
        _check(self.lib.kami_vbd_set_state(self._h, buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes, MEM_HOST))

    def get_state_into(self, out):
        """Snapshot into a preallocated buffer (numpy, or a torch CUDA tensor for a device copy)."""
        p, m = _ptr(out)
        nbytes = out.numel() * out.element_size() if hasattr(out, "numel") else out.nbytes
        _check(self.lib.kami_vbd_get_state(self._h, p, nbytes, m))
        return out

    def set_state_from(self, buf):
        p, m = _ptr(buf)
        nbytes = buf.numel() * buf.element_size() if hasattr(buf, "numel") else buf.nbytes
        _check(self.lib.kami_vbd_set_state(self._h, p, nbytes, m))

    # -- differentiable stepping
    def tape_reserve(self, max_steps, max_tiles=0):
        _check(self.lib.kami_vbd_tape_reserve(self._h, max_steps, max_tiles))

    def tape_bytes_per_substep(self, tiles=None):
        """Device bytes one recorded substep of `tiles` warp tiles (all by default) takes on the tape:
        (num_itr + 1) * 32 + 48 B per slot, as kami_vbd_tape_reserve allocates them."""
        tiles = self.tile_count() if tiles is None else tiles
        return ((self.num_itr + 1) * 32 + 48) * 32 * self.slots_per_lane * tiles

    def tile_count(self):
        n = ctypes.c_int64()
        _check(self.lib.kami_vbd_get_tile_count(self._h, ctypes.byref(n)))
        return n.value

    def tiles_per_group(self):
        """Tiles a strand may run on across (1 when every strand fits one tile)."""
        k = ctypes.c_int32()
        _check(self.lib.kami_vbd_get_tiles_per_group(self._h, ctypes.byref(k)))
        return k.value

    def set_tape_window(self, tile_begin, tile_end):
        _check(self.lib.kami_vbd_set_tape_window(self._h, tile_begin, tile_end))

    def restore_tape_window_from(self, buf):
        """set_state_from for the strands of the tape window only (and the step clock): a whole-groom
        state buffer, of which only the window's strands are read when it is a CUDA tensor."""
        p, m = _ptr(buf)
        nbytes = buf.numel() * buf.element_size() if hasattr(buf, "numel") else buf.nbytes
        _check(self.lib.kami_vbd_restore_tape_window(self._h, p, nbytes, m))

    def step_record(self, dt, stream=None):
        s = None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        _check(self.lib.kami_vbd_step_record(self._h, ctypes.c_float(dt), s))

    def backward(self, gx, gv, gvl, gq):
        """In place: adjoint of the state after the recorded steps -> adjoint before them."""
        ptrs = [_ptr(a) for a in (gx, gv, gvl, gq)]
        _check(self.lib.kami_vbd_backward(self._h, ptrs[0][0], ptrs[1][0], ptrs[2][0], ptrs[3][0], ptrs[0][1], None))

    def get_rest_darboux_grad(self, out=None):
        out = np.empty((self.num_vertices, 4), np.float32) if out is None else out
        p, m = _ptr(out)
        _check(self.lib.kami_vbd_get_rest_darboux_grad(self._h, p, m))
        return out

    def zero_rest_darboux_grad(self):
        _check(self.lib.kami_vbd_zero_rest_darboux_grad(self._h))

    def split_state(self, buf):
        nv = self.num_vertices
        return dict(x=buf[:3 * nv].reshape(nv, 3), v=buf[3 * nv:6 * nv].reshape(nv, 3),
                    v_last=buf[6 * nv:9 * nv].reshape(nv, 3), q=buf[9 * nv:13 * nv].reshape(nv, 4),
                    clock=buf[13 * nv:13 * nv + 3])


def version():
    return load_library().kami_vbd_version().decode()


def read_usc(path, max_verts=0):
    """A USC-HairSalon .data file: (vertex count per strand int32 [S], xyz float32) with xyz packed
    [V, 3] (max_verts = 0) or padded [S, max_verts, 3] like KamiSimulator's Hair arrays."""
    lib = load_library()
    ns, nv, mx = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int32()
    _check(lib.kami_usc_info(os.fsencode(path), ctypes.byref(ns), ctypes.byref(nv), ctypes.byref(mx)))
    counts = np.zeros(ns.value, np.int32)
    shape = (ns.value, max_verts, 3) if max_verts > 0 else (nv.value, 3)
    xyz = np.zeros(shape, np.float32)
    _check(lib.kami_usc_read(os.fsencode(path), max_verts, counts.ctypes.data_as(ctypes.c_void_p),
                             xyz.ctypes.data_as(ctypes.c_void_p)))
    return counts, xyz


def write_usc(path, counts, xyz, max_verts=0):
    """Writes a USC-HairSalon .data file from packed ([V, 3]) or padded ([S, max_verts, 3]) xyz."""
    lib = load_library()
    c = np.ascontiguousarray(counts, np.int32)
    a = np.ascontiguousarray(xyz, np.float32)
    _check(lib.kami_usc_write(os.fsencode(path), c.shape[0], c.ctypes.data_as(ctypes.c_void_p), max_verts,
                              a.ctypes.data_as(ctypes.c_void_p)))


def bake_sdf(vertices, triangles, dims, grid_min, grid_max, threshold=1e-3, device=-1):
    """kami_sdf_bake on the GPU: an SDFGrid-like object (dims, grid_min, grid_max, phi [nz, ny, nx],
    grad [nz, ny, nx, 3], threshold) ready for Solver(..., sdf=...)."""
    from types import SimpleNamespace

    lib = load_library()
    v = np.ascontiguousarray(vertices, np.float32)
    t = np.ascontiguousarray(triangles, np.int32)
    d = np.asarray(dims, np.int32)
    lo = np.asarray(grid_min, np.float32)
    hi = np.asarray(grid_max, np.float32)
    nx, ny, nz = (int(a) for a in dims)
    phi = np.zeros((nz, ny, nx), np.float32)
    grad = np.zeros((nz, ny, nx, 3), np.float32)
    c = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _check(lib.kami_sdf_bake(c(v), v.shape[0], c(t), t.shape[0], c(d), c(lo), c(hi), c(phi), c(grad), MEM_HOST, device))
    return SimpleNamespace(dims=tuple(int(a) for a in dims), grid_min=tuple(float(a) for a in lo),
                           grid_max=tuple(float(a) for a in hi), phi=phi, grad=grad, threshold=threshold)


def hair_subdivide(counts, xyz, mul, vxyz=None, device=-1):
    """DivideHair on padded [S, max_verts, 3] arrays: returns (counts, xyz[, vxyz]) with rows of
    (max_verts - 1) * mul + 1 (zeros past each strand's end)."""
    lib = load_library()
    c = np.ascontiguousarray(counts, np.int32)
    x = np.ascontiguousarray(xyz, np.float32)
    ns, mv = x.shape[0], x.shape[1]
    out_mv = (mv - 1) * mul + 1
    oc = np.zeros(ns, np.int32)
    ox = np.zeros((ns, out_mv, 3), np.float32)
    v = None if vxyz is None else np.ascontiguousarray(vxyz, np.float32)
    ov = None if v is None else np.zeros_like(ox)
    p = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _check(lib.kami_hair_subdivide(ns, p(c), mv, p(x), p(v), mul, p(oc), p(ox), p(ov), device))
    return (oc, ox) if v is None else (oc, ox, ov)


def hair_resample(counts, xyz, target_len, device=-1):
    """BuildYarnBallHair's resampling on padded [S, max_verts, 3] arrays: returns new (counts, xyz)."""
    lib = load_library()
    c = np.array(counts, np.int32)
    x = np.array(xyz, np.float32)
    _check(lib.kami_hair_resample(x.shape[0], c.ctypes.data_as(ctypes.c_void_p), x.shape[1],
                                  x.ctypes.data_as(ctypes.c_void_p), ctypes.c_float(target_len), device))
    return c, x
