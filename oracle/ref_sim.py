"""ctypes front-end of oracle/_ref/libkami_ref.so -- TEST INFRASTRUCTURE ONLY.

The library is KamiSimulator's own YarnBall Sim and SDF kernel compiled from the reference
sources (oracle/ref/Makefile) with a thin C driver (oracle/ref/ref_driver.cu).  It needs a CUDA
device.  Tests use it to pin the CPU oracle to the reference itself."""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libkami_ref.so")
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
        lib.ref_create.restype = vp
        lib.ref_create.argtypes = [i64, i32, vp, vp, f32, f32, f32, f32, vp, f32, i32, f32, i32]
        lib.ref_destroy.argtypes = [vp]
        lib.ref_material.argtypes = [vp] + [vp] * 6
        lib.ref_set_state.argtypes = [vp] + [vp] * 5
        lib.ref_advance.argtypes = [vp, f32]
        lib.ref_sag_free.argtypes = [vp, i32, vp, i32]
        lib.ref_sag_free.restype = ctypes.c_int
        lib.ref_step_hair_hair.argtypes = [vp, f32, f32]
        lib.ref_step_hair_hair.restype = ctypes.c_int
        lib.ref_download.argtypes = [vp, vp, vp, vp]
        lib.ref_sdf_project.argtypes = [i64, vp, vp, vp, vp, vp, vp, f32, vp, vp, vp, vp]
        lib.ref_strain_limit.argtypes = [i32, vp, vp, f32, vp]
        lib.ref_set_connections.argtypes = [vp, vp]
        for n in ("ref_material", "ref_set_state", "ref_advance", "ref_download", "ref_sdf_project", "ref_strain_limit",
                  "ref_set_connections"):
            getattr(lib, n).restype = ctypes.c_int
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefSim:
    """The reference's YarnBall::Sim (Jacobi kernels, racy at block boundaries)."""

    def __init__(self, groom, *, young, deviation=1.0, radius=40e-6, density=1300.0, gravity=(0.0, 0.0, -9.81),
                 velocity_decay=0.05, num_itr=10, max_h=4e-4, pin_roots=True):
        self.lib = load()
        self.nv = groom.num_vertices
        sb = np.ascontiguousarray(groom.strand_begin, np.int32)
        pos = np.ascontiguousarray(groom.positions, np.float32)
        g = np.asarray(gravity, np.float32)
        self.h = self.lib.ref_create(self.nv, groom.num_strands, _p(sb), _p(pos), radius, density, young, deviation,
                                     _p(g), velocity_decay, num_itr, max_h, int(pin_roots))
        if not self.h:
            raise RuntimeError("reference Sim construction failed")

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def material(self):
        nv = self.nv
        out = dict(inv_mass=np.zeros(nv, np.float32), l_rest=np.zeros(nv, np.float32),
                   k_stretch=np.zeros(nv, np.float32), flags=np.zeros(nv, np.uint32), q=np.zeros((nv, 4), np.float32),
                   q_rest=np.zeros((nv, 4), np.float32))
        self.lib.ref_material(self.h, _p(out["inv_mass"]), _p(out["l_rest"]), _p(out["k_stretch"]), _p(out["flags"]),
                              _p(out["q"]), _p(out["q_rest"]))
        return out

    def set_state(self, x, v, v_last, q, clock):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (x, v, v_last, q, clock)]
        if self.lib.ref_set_state(self.h, *[_p(a) for a in arrs]) != 0:
            raise RuntimeError("ref_set_state failed")

    def sag_free(self, strand_begin, iterations):
        """Sim::SagFree on the reference's host arrays (roots = first vertex of each strand)."""
        sb = np.ascontiguousarray(strand_begin, np.int32)
        self.lib.ref_sag_free(self.h, sb.shape[0] - 1, _p(sb), iterations)

    def step_hair_hair(self, dt, barrier_thickness):
        """One substep of the reference's hair-hair path with its own kernels, detection over every
        segment pair (the reference's LBVH cannot run as shipped); returns its error word."""
        rc = self.lib.ref_step_hair_hair(self.h, dt, barrier_thickness)
        if rc < 0:
            raise RuntimeError("ref_step_hair_hair failed")
        return rc

    def advance(self, dt):
        if self.lib.ref_advance(self.h, dt) != 0:
            raise RuntimeError("ref_advance failed")

    def set_connections(self, connection_index):
        """Vertex::connectionIndex of every vertex (-1: none)."""
        c = np.ascontiguousarray(connection_index, np.int32)
        if self.lib.ref_set_connections(self.h, _p(c)) != 0:
            raise RuntimeError("ref_set_connections failed")

    def download(self):
        x = np.zeros((self.nv, 3), np.float32)
        v = np.zeros((self.nv, 3), np.float32)
        q = np.zeros((self.nv, 4), np.float32)
        self.lib.ref_download(self.h, _p(x), _p(v), _p(q))
        return x, v, q


def sdf_project(pos, vel, local_idx, sdf, rot=(0.0, 0.0, 0.0, 1.0), trans=(0.0, 0.0, 0.0)):
    """One pass of the reference's SDFHeadCollision kernel; returns new (pos, vel)."""
    lib = load()
    p = np.ascontiguousarray(pos, np.float32).copy()
    v = np.ascontiguousarray(vel, np.float32).copy()
    li = np.ascontiguousarray(local_idx, np.int32)
    dims = np.asarray(sdf.dims, np.int32)
    gmin = np.asarray(sdf.grid_min, np.float32)
    gmax = np.asarray(sdf.grid_max, np.float32)
    phi = np.ascontiguousarray(sdf.phi, np.float32)
    grad = np.ascontiguousarray(sdf.grad, np.float32)
    r = np.asarray(rot, np.float32)
    t = np.asarray(trans, np.float32)
    rc = lib.ref_sdf_project(p.shape[0], _p(p), _p(v), _p(li), _p(dims), _p(gmin), _p(gmax), sdf.threshold, _p(phi),
                             _p(grad), _p(r), _p(t))
    if rc != 0:
        raise RuntimeError("ref_sdf_project failed")
    return p, v


def strain_limit(x, strand_begin, rest_lengths, strain_error=0.1):
    """One pass of the reference's StrainLimiting kernel (cudaSDFCollision.cu:176-199) on packed
    strands; returns the corrected positions."""
    lib = load()
    out = np.ascontiguousarray(x, np.float32).copy()
    sb = np.ascontiguousarray(strand_begin, np.int32)
    l0 = np.ascontiguousarray(rest_lengths, np.float32)
    if lib.ref_strain_limit(len(sb) - 1, _p(sb), _p(l0), float(strain_error), _p(out)) != 0:
        raise RuntimeError("ref_strain_limit failed")
    return out


CPU_LIB_PATH = os.path.join(_HERE, "_ref", "libkami_ref_cpu.so")


def cpu_available():
    """The reference's CPU parts built from source (SDF bake, strand resampler); no GPU needed."""
    return os.path.exists(CPU_LIB_PATH)


_cpu = None


def _sdf_lib():
    global _cpu
    if _cpu is None:
        lib = ctypes.CDLL(CPU_LIB_PATH)
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        lib.ref_sdf_signed_distance.argtypes = [i32, vp, i32, vp, i64, vp, vp]
        lib.ref_sdf_bake.argtypes = [i32, vp, i32, vp, vp, vp, vp, vp, vp]
        lib.ref_resample_cmr.argtypes = [vp, i32, ctypes.c_double, vp, i64]
        lib.ref_resample_cmr.restype = i64
        _cpu = lib
    return _cpu


def resample_cmr(points, target):
    """Resample::resampleCMR(curve, 1, n - 2, target) of the reference, compiled from source.  It
    corrupts the heap when a pass yields 8 samples or fewer (resample.h:78-79): call it only for
    strands whose resampled length is well above that."""
    p = np.ascontiguousarray(points, np.float32)
    cap = 5 * p.shape[0] + 16
    out = np.zeros((cap, 3), np.float32)
    # the target is a float setting (JsonParams::ResampleLen) widened to double, as BuildYarnBallHair passes it
    n = _sdf_lib().ref_resample_cmr(_p(p), p.shape[0], float(np.float32(target)), _p(out), cap)
    return out[:min(n, cap)].copy()


def sdf_signed_distance(vertices, triangles, points):
    """Discregrid's TriangleMeshDistance::signed_distance, compiled from the reference's sources."""
    v = np.ascontiguousarray(vertices, np.float32)
    t = np.ascontiguousarray(triangles, np.int32)
    p = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    out = np.zeros(p.shape[0], np.float64)
    _sdf_lib().ref_sdf_signed_distance(v.shape[0], _p(v), t.shape[0], _p(t), p.shape[0], _p(p), _p(out))
    return out


def sdf_bake(vertices, triangles, dims, grid_min, grid_max):
    """The reference's bake: Kami::SDF::Init (cubic Lagrange grid of Discregrid's distance at
    resolution dims) sampled at the grid nodes as PNMesh::StoreSDFQueries does; (phi, grad)."""
    v = np.ascontiguousarray(vertices, np.float32)
    t = np.ascontiguousarray(triangles, np.int32)
    d = np.asarray(dims, np.int32)
    lo = np.asarray(grid_min, np.float32)
    hi = np.asarray(grid_max, np.float32)
    nx, ny, nz = (int(a) for a in dims)
    phi = np.zeros((nz, ny, nx), np.float32)
    grad = np.zeros((nz, ny, nx, 3), np.float32)
    _sdf_lib().ref_sdf_bake(v.shape[0], _p(v), t.shape[0], _p(t), _p(d), _p(lo), _p(hi), _p(phi), _p(grad))
    return phi, grad
