"""Seeded synthetic grooms and body SDF grids for the solver's workloads.

The reference ships no hair or head data for this path (its USC-HairSalon `.data`
files and head meshes are downloaded separately), so every workload is generated
here from a fixed seed:

* ``cantilever``: straight horizontal rods, the geometry of the reference's
  cantilever harness (src/solvers/CantileverTestSolver.cpp:18-104): 64 rods x 32
  vertices, 5 mm segments, roots 1 cm apart on the y axis, rods along +x.
* ``groom``: strands rooted uniformly on the upper (z > 0) hemisphere of a 0.09 m
  head sphere, growing along the outward normal with a helical curl (radius
  U[0, 8] mm, pitch U[1, 3] cm), segment length 2 mm x U[0.9, 1.1], per-strand
  Young's modulus log-uniform in [1, 5] GPa.
* ``batched grooms``: many independent grooms with log-uniform strand counts and
  uniform-integer vertex counts per strand.
* ``sphere_sdf`` / ``capsule_union_sdf``: signed-distance grids sampled at the
  node positions the reference uses (node (i, j, k) at grid_min + ds * (i, j, k),
  ds = (grid_max - grid_min) / dims, src/PNMesh.cpp:118-146), stored x-fastest.

Positions are float32 metres; strands are contiguous, described by CSR offsets
``strand_begin`` (length S + 1).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Groom:
    strand_begin: np.ndarray  # int32 [S + 1]
    positions: np.ndarray  # float32 [V, 3]
    strand_young: np.ndarray  # float32 [S], GPa
    strand_dev: np.ndarray  # float32 [S], bend deviation coefficient

    @property
    def num_strands(self) -> int:
        return int(self.strand_begin.shape[0] - 1)

    @property
    def num_vertices(self) -> int:
        return int(self.positions.shape[0])

    def strand_lengths(self) -> np.ndarray:
        return np.diff(self.strand_begin)


@dataclasses.dataclass
class SDFGrid:
    dims: tuple  # (nx, ny, nz)
    grid_min: tuple
    grid_max: tuple
    phi: np.ndarray  # float32 [nz, ny, nx]
    grad: np.ndarray  # float32 [nz, ny, nx, 3]
    threshold: float

    def node_positions(self, z0: int = 0, z1: int | None = None) -> np.ndarray:
        nx, ny, nz = self.dims
        z1 = nz if z1 is None else z1
        return _node_positions(self.dims, self.grid_min, self.grid_max, z0, z1)


def _node_positions(dims, gmin, gmax, z0, z1):
    nx, ny, nz = dims
    gmin = np.asarray(gmin, np.float32)
    ds = (np.asarray(gmax, np.float32) - gmin) / np.asarray(dims, np.float32)
    iz, iy, ix = np.meshgrid(np.arange(z0, z1), np.arange(ny), np.arange(nx), indexing="ij")
    p = np.stack([ix, iy, iz], axis=-1).astype(np.float32)
    return gmin + ds * p


def cantilever(num_rods: int = 64, verts_per_rod: int = 32, segment: float = 5e-3, spacing: float = 1e-2,
               young: float = 3.9) -> Groom:
    """Straight rods along +x, roots at (0, spacing * k, 0)."""
    k = np.arange(num_rods, dtype=np.float32)
    j = np.arange(verts_per_rod, dtype=np.float32)
    pos = np.zeros((num_rods, verts_per_rod, 3), np.float32)
    pos[:, :, 0] = segment * j[None, :]
    pos[:, :, 1] = spacing * k[:, None]
    sb = (np.arange(num_rods + 1) * verts_per_rod).astype(np.int32)
    return Groom(sb, pos.reshape(-1, 3), np.full(num_rods, young, np.float32), np.ones(num_rods, np.float32))


def _orthonormal_frames(n: np.ndarray):
    """Two unit vectors perpendicular to each row of n (rows unit length)."""
    helper = np.where(np.abs(n[:, 2:3]) < 0.9, np.array([[0.0, 0.0, 1.0]]), np.array([[1.0, 0.0, 0.0]]))
    t1 = np.cross(n, helper)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(n, t1)
    return t1, t2


def groom_strands(rng: np.random.Generator, lengths: np.ndarray, head_radius: float = 0.09,
                  seg_len: float = 2e-3, seg_jitter: float = 0.1, curl_radius_max: float = 8e-3,
                  pitch_range=(1e-2, 3e-2), young_range=(1.0, 5.0)) -> Groom:
    """Curly strands of the given vertex counts rooted on the upper head hemisphere."""
    lengths = np.asarray(lengths, np.int64)
    S = lengths.shape[0]
    # uniform on the upper hemisphere: z = cos(theta) uniform in (0, 1]
    z = rng.uniform(0.0, 1.0, S)
    phi = rng.uniform(0.0, 2.0 * math.pi, S)
    rxy = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    n = np.stack([rxy * np.cos(phi), rxy * np.sin(phi), z], axis=1)
    t1, t2 = _orthonormal_frames(n)
    curl_r = rng.uniform(0.0, curl_radius_max, S)
    pitch = rng.uniform(pitch_range[0], pitch_range[1], S)
    theta0 = rng.uniform(0.0, 2.0 * math.pi, S)
    young = np.exp(rng.uniform(math.log(young_range[0]), math.log(young_range[1]), S))
    V = int(lengths.sum())
    sb = np.zeros(S + 1, np.int64)
    np.cumsum(lengths, out=sb[1:])
    strand_of = np.repeat(np.arange(S), lengths)
    local = np.arange(V) - sb[strand_of]
    seg = seg_len * rng.uniform(1.0 - seg_jitter, 1.0 + seg_jitter, V)
    seg[sb[1:] - 1] = 0.0  # no segment after a tip
    # axial advance per segment so that the helix arc length matches the segment length
    slope = np.sqrt(1.0 + (2.0 * math.pi * curl_r / pitch) ** 2)
    dz = seg / slope[strand_of]
    excl = np.cumsum(dz) - dz  # exclusive prefix sum over all vertices
    axial = excl - excl[sb[:-1]][strand_of]  # ... restarted at each strand root
    axial[local == 0] = 0.0
    ang = theta0[strand_of] + 2.0 * math.pi * axial / pitch[strand_of]
    r = curl_r[strand_of]
    off = (r * (np.cos(ang) - np.cos(theta0[strand_of])))[:, None] * t1[strand_of] + \
          (r * (np.sin(ang) - np.sin(theta0[strand_of])))[:, None] * t2[strand_of]
    pos = head_radius * n[strand_of] + axial[:, None] * n[strand_of] + off
    return Groom(sb.astype(np.int32), pos.astype(np.float32), young.astype(np.float32), np.ones(S, np.float32))


def groom(num_strands: int = 10_000, verts_per_strand: int = 64, seed: int = 2) -> Groom:
    rng = np.random.default_rng(seed)
    return groom_strands(rng, np.full(num_strands, verts_per_strand))


def batched_grooms(num_grooms: int = 64, strands_range=(500, 20_000), verts_range=(16, 128), seed: int = 3,
                   strand_scale: float = 1.0) -> list:
    """Independent grooms: strand count log-uniform, vertices per strand uniform integer."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(num_grooms):
        s = int(round(math.exp(rng.uniform(math.log(strands_range[0]), math.log(strands_range[1]))) * strand_scale))
        s = max(1, s)
        lens = rng.integers(verts_range[0], verts_range[1] + 1, s)
        out.append(groom_strands(rng, lens))
    return out


def concat_grooms(grooms: list) -> Groom:
    sbs, pos, young, dev = [np.zeros(1, np.int64)], [], [], []
    off = 0
    for g in grooms:
        sbs.append(g.strand_begin[1:].astype(np.int64) + off)
        off += g.num_vertices
        pos.append(g.positions)
        young.append(g.strand_young)
        dev.append(g.strand_dev)
    return Groom(np.concatenate(sbs).astype(np.int32), np.concatenate(pos), np.concatenate(young),
                 np.concatenate(dev))


# ---- hair-hair contact scenes ---------------------------------------------------------------------

def bar_and_drape(verts: int = 25, segment: float = 1e-3, gap: float = 3e-4, bar_young: float = 5.0,
                  drape_young: float = 1e-6) -> Groom:
    """A stiff strand along x (root at -x) and a soft strand along y, `gap` above it, crossing it at
    the middle: under gravity the soft strand falls onto the stiff one."""
    half = segment * (verts - 1) / 2
    t = np.linspace(-half, half, verts)
    a = np.stack([t, np.zeros(verts), np.zeros(verts)], 1)
    b = np.stack([np.zeros(verts), t, np.full(verts, gap)], 1)
    return Groom(strand_begin=np.array([0, verts, 2 * verts], np.int32),
                 positions=np.concatenate([a, b]).astype(np.float32),
                 strand_young=np.array([bar_young, drape_young], np.float32), strand_dev=np.ones(2, np.float32))


def tangle(num_strands: int = 24, verts: int = 24, segment: float = 1e-3, layer: float = 2e-4, seed: int = 0,
           young: float = 1e-5) -> Groom:
    """Horizontal strands through a common vertical axis, each `layer` above the previous one, in
    random directions: falling under gravity they pile onto each other (many crossing contacts)."""
    rng = np.random.default_rng(seed)
    half = segment * (verts - 1) / 2
    pos = []
    for k in range(num_strands):
        th = rng.uniform(0, 2 * np.pi)
        d = np.array([np.cos(th), np.sin(th), 0.0])
        c = np.array([rng.uniform(-2e-3, 2e-3), rng.uniform(-2e-3, 2e-3), k * layer])
        pos.append(c + (np.arange(verts)[:, None] * segment - half) * d)
    return Groom(strand_begin=np.arange(num_strands + 1, dtype=np.int32) * verts,
                 positions=np.concatenate(pos).astype(np.float32),
                 strand_young=np.full(num_strands, young, np.float32), strand_dev=np.ones(num_strands, np.float32))


def contact_fence(num_posts: int = 20, spacing: float = 3e-5, verts: int = 8, segment: float = 1e-3) -> Groom:
    """`num_posts` parallel strands `spacing` apart and one strand across all of them: its middle
    segment touches every post, more than the 16 contacts a segment can hold."""
    half = segment * (verts - 1) / 2
    t = np.arange(verts) * segment - half
    pos = []
    for k in range(num_posts):
        x = (k - (num_posts - 1) / 2) * spacing
        pos.append(np.stack([np.full(verts, x), t, np.zeros(verts)], 1))
    pos.append(np.stack([t, np.zeros(verts), np.full(verts, 4e-5)], 1))
    n = num_posts + 1
    return Groom(strand_begin=np.arange(n + 1, dtype=np.int32) * verts, positions=np.concatenate(pos).astype(np.float32),
                 strand_young=np.full(n, 1.0, np.float32), strand_dev=np.ones(n, np.float32))


# ---- body meshes for the SDF bake ----------------------------------------------------------------

def icosphere(subdivisions: int = 3, radius: float = 0.09, centre=(0.0, 0.0, 0.0)):
    """Closed triangle mesh of a sphere (vertices float32 [V, 3], triangles int32 [T, 3], outward
    counter-clockwise winding)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    for _ in range(subdivisions):
        cache, nf = {}, []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    V = np.asarray(verts) * radius + np.asarray(centre)
    return V.astype(np.float32), np.asarray(f, np.int32)


def torus(major: float = 0.06, minor: float = 0.025, n_major: int = 32, n_minor: int = 16, centre=(0.0, 0.0, 0.0)):
    """Closed, non-convex triangle mesh of a torus around the z axis (outward winding)."""
    u = np.arange(n_major) * 2 * np.pi / n_major
    w = np.arange(n_minor) * 2 * np.pi / n_minor
    U, W = np.meshgrid(u, w, indexing="ij")
    x = (major + minor * np.cos(W)) * np.cos(U)
    y = (major + minor * np.cos(W)) * np.sin(U)
    z = minor * np.sin(W)
    V = np.stack([x, y, z], -1).reshape(-1, 3) + np.asarray(centre)
    tris = []
    for i in range(n_major):
        for j in range(n_minor):
            a, b = i * n_minor + j, ((i + 1) % n_major) * n_minor + j
            c, d = ((i + 1) % n_major) * n_minor + (j + 1) % n_minor, i * n_minor + (j + 1) % n_minor
            tris += [(a, b, c), (a, c, d)]
    return V.astype(np.float32), np.asarray(tris, np.int32)


def mesh_bounds(vertices):
    """The mesh's bounding box: the grid StoreSDFQueries samples (PNMesh.cpp:117-121)."""
    v = np.asarray(vertices, np.float32)
    return tuple(float(a) for a in v.min(0)), tuple(float(a) for a in v.max(0))


def sphere_sdf(n: int = 128, radius: float = 0.09, half_extent: float = 0.2, threshold: float = 1e-3) -> SDFGrid:
    dims = (n, n, n)
    gmin = (-half_extent,) * 3
    gmax = (half_extent,) * 3
    p = _node_positions(dims, gmin, gmax, 0, n).astype(np.float64)
    d = np.linalg.norm(p, axis=-1)
    phi = (d - radius).astype(np.float32)
    grad = (p / np.maximum(d, 1e-12)[..., None]).astype(np.float32)
    return SDFGrid(dims, gmin, gmax, phi, grad, threshold)


def capsule_union_sdf(n: int = 256, num_capsules: int = 12, radius_range=(0.02, 0.08), half_extent: float = 0.3,
                      threshold: float = 1e-3, seed: int = 5) -> SDFGrid:
    """Union (min) of random capsules; the gradient is that of the closest capsule."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-0.15, 0.15, (num_capsules, 3))
    b = a + rng.normal(0.0, 0.08, (num_capsules, 3))
    r = rng.uniform(radius_range[0], radius_range[1], num_capsules)
    dims = (n, n, n)
    gmin = (-half_extent,) * 3
    gmax = (half_extent,) * 3
    phi = np.empty((n, n, n), np.float32)
    grad = np.empty((n, n, n, 3), np.float32)
    chunk = max(1, (1 << 21) // (n * n))
    for z0 in range(0, n, chunk):
        z1 = min(n, z0 + chunk)
        p = _node_positions(dims, gmin, gmax, z0, z1).reshape(-1, 3).astype(np.float64)
        best = np.full(p.shape[0], np.inf)
        bgrad = np.zeros_like(p)
        for c in range(num_capsules):
            ab = b[c] - a[c]
            t = np.clip(((p - a[c]) @ ab) / (ab @ ab), 0.0, 1.0)
            closest = a[c] + t[:, None] * ab
            dv = p - closest
            dist = np.linalg.norm(dv, axis=1)
            d = dist - r[c]
            m = d < best
            best[m] = d[m]
            bgrad[m] = dv[m] / np.maximum(dist[m], 1e-12)[:, None]
        phi[z0:z1] = best.reshape(z1 - z0, n, n)
        grad[z0:z1] = bgrad.reshape(z1 - z0, n, n, 3)
    return SDFGrid(dims, gmin, gmax, phi, grad, threshold)


def head_rotation(t: float, amplitude_deg: float = 30.0, freq_hz: float = 1.0):
    """Body quaternion (x, y, z, w) for a sinusoidal yaw about the vertical (z) axis."""
    ang = math.radians(amplitude_deg) * math.sin(2.0 * math.pi * freq_hz * t)
    return (0.0, 0.0, math.sin(0.5 * ang), math.cos(0.5 * ang))


# Solver settings of each workload.  Units: seconds, metres, kg/m^3, GPa.
WORKLOADS = {
    "cantilever_64x32": dict(num_itr=10, dt=1.0 / 60.0, frames=100, gravity=(0.0, 0.0, -9.81), sdf=None),
    "groom_10k_x64": dict(num_itr=20, dt=1.0 / 120.0, frames=200, gravity=(0.0, 0.0, -9.81), sdf="sphere128"),
    "batched_64_grooms": dict(num_itr=20, dt=1.0 / 120.0, frames=120, gravity=(0.0, 0.0, -9.81), sdf="sphere128"),
    "adjoint_2k_x48": dict(num_itr=20, dt=1.0 / 120.0, frames=60, gravity=(0.0, 0.0, -9.81), sdf="sphere128"),
    "large_8x100k_x100": dict(num_itr=30, dt=1.0 / 120.0, frames=240, gravity=(0.0, 0.0, -9.81), sdf="capsules256"),
}

COMMON = dict(radius=40e-6, density=1300.0, damping=1e-6, velocity_decay=0.05, acceleration_ratio=1.0,
              ext_mult=1.0)
