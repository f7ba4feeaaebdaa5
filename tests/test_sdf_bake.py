"""Body SDF bake: the FP64 oracle against the reference's own code built from source on the CPU
(oracle/_ref/libkami_ref_cpu.so: Kami::SDF over Discregrid, utilities/Geometry.cpp:5-35, and
PNMesh::StoreSDFQueries' node loop), and the host-side checks of kami_sdf_bake."""
import ctypes

import numpy as np
import pytest

from kamisimulator_b200 import synth, vbd
from oracle import oracle as orc
from oracle import ref_sim

needs_ref = pytest.mark.skipif(not ref_sim.cpu_available(), reason="oracle/_ref not built (needs the reference sources)")
MESHES = {"icosphere": lambda: synth.icosphere(3), "torus": lambda: synth.torus()}


def _nodes(dims, lo, hi):
    nx, ny, nz = dims
    ds = (np.asarray(hi, np.float64) - np.asarray(lo, np.float64)) / np.asarray(dims)
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return np.stack([lo[0] + ds[0] * ix, lo[1] + ds[1] * iy, lo[2] + ds[2] * iz], -1), ds


@needs_ref
@pytest.mark.parametrize("mesh", sorted(MESHES))
def test_oracle_distance_equals_discregrid(mesh):
    """Exact signed distance and sign (TriangleMeshDistance::signed_distance) at every node of a
    grid over the mesh's box padded by 20 %, and at random points."""
    V, T = MESHES[mesh]()
    lo, hi = synth.mesh_bounds(V)
    pad = 0.2 * (np.asarray(hi) - np.asarray(lo))
    lo, hi = tuple(np.asarray(lo) - pad), tuple(np.asarray(hi) + pad)
    dims = (21, 24, 19)
    phi, _ = orc.sdf_bake(V, T, dims, lo, hi)
    pts, _ = _nodes(dims, np.float32(lo), np.float32(hi))
    ref = ref_sim.sdf_signed_distance(V, T, pts.reshape(-1, 3)).reshape(phi.shape)
    assert (phi < 0).any() and (phi > 0).any()
    np.testing.assert_allclose(phi, ref, rtol=0, atol=1e-12)


@needs_ref
@pytest.mark.parametrize("mesh", sorted(MESHES))
def test_reference_grid_is_a_resampling_of_the_exact_distance(mesh):
    """The reference's grid resamples the distance through a cubic Lagrange grid over the mesh box
    padded by 0.1 m, so near the surface it is the exact distance up to that resampling error
    (measured up to ~0.3 node spacings on the torus at 24^3); the outside gradients follow the same
    rule (radial from the grid centre) exactly."""
    V, T = MESHES[mesh]()
    lo, hi = synth.mesh_bounds(V)
    dims = (24, 24, 24)
    phi, grad = orc.sdf_bake(V, T, dims, lo, hi)
    rphi, rgrad = ref_sim.sdf_bake(V, T, dims, lo, hi)
    ds = (np.asarray(hi) - np.asarray(lo)).min() / 24
    near = np.abs(phi) < 2 * ds
    assert np.abs(phi - rphi)[near].max() <= 0.5 * ds
    assert np.mean(np.sign(phi[near]) == np.sign(rphi[near])) >= 0.98
    pts, _ = _nodes(dims, np.float32(lo), np.float32(hi))
    centre = (np.asarray(lo, np.float64) + np.asarray(hi, np.float64)) / 2
    off_centre = np.linalg.norm(pts - centre, axis=-1) > 1e-6  # the radial direction is 0/0 at the centre
    out = (phi >= 0) & (rphi >= 0) & np.isfinite(rgrad).all(-1) & off_centre
    np.testing.assert_allclose(grad[out], rgrad[out], atol=1e-6)


def test_oracle_matches_the_analytic_torus():
    """Distance to a torus, (sqrt(x^2 + y^2) - R)^2 + z^2 = r^2, within its tessellation error."""
    V, T = synth.torus(0.06, 0.025, 96, 48)
    lo, hi = (-0.1, -0.1, -0.04), (0.1, 0.1, 0.04)
    dims = (20, 20, 8)
    phi, grad = orc.sdf_bake(V, T, dims, lo, hi)
    p, _ = _nodes(dims, np.float32(lo), np.float32(hi))
    exact = np.sqrt((np.hypot(p[..., 0], p[..., 1]) - 0.06) ** 2 + p[..., 2] ** 2) - 0.025
    chord = 0.025 * (1 - np.cos(np.pi / 48)) + 0.085 * (1 - np.cos(np.pi / 96))
    assert np.abs(phi - exact).max() <= 2 * chord
    inside = phi < -1e-3
    assert np.allclose(np.linalg.norm(grad[inside], axis=-1), 1.0, atol=1e-9)


def test_bake_rejects_bad_meshes_on_the_host():
    """1 = INVALID_ARGUMENT, 5 = GEOMETRY; no device is touched."""
    lib = vbd.load_library()
    V, T = synth.icosphere(1)
    dims = np.array([4, 4, 4], np.int32)
    lo = np.array([-0.1] * 3, np.float32)
    hi = np.array([0.1] * 3, np.float32)
    phi = np.zeros(64, np.float32)
    grad = np.zeros(192, np.float32)
    c = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    bad = T.copy()
    bad[3, 1] = V.shape[0]
    assert lib.kami_sdf_bake(c(V), V.shape[0], c(bad), T.shape[0], c(dims), c(lo), c(hi), c(phi), c(grad), 0, -1) == 1
    flat = T.copy()
    flat[0] = [0, 0, 1]
    assert lib.kami_sdf_bake(c(V), V.shape[0], c(flat), T.shape[0], c(dims), c(lo), c(hi), c(phi), c(grad), 0, -1) == 5
    assert lib.kami_sdf_bake(c(V), V.shape[0], c(T), T.shape[0], c(dims), c(hi), c(lo), c(phi), c(grad), 0, -1) == 1
    Vn = V.copy()
    Vn[2, 0] = np.nan
    assert lib.kami_sdf_bake(c(Vn), V.shape[0], c(T), T.shape[0], c(dims), c(lo), c(hi), c(phi), c(grad), 0, -1) == 1
