"""CPU tests of the oracle: hand-derived values, invariants and an independent numpy restatement."""
import math

import numpy as np
import pytest

from kamisimulator_b200 import synth
from oracle import oracle as orc
from tests import helpers


def test_configure_matches_hand_formulas():
    """Sim::configure + setYoung (YBSimulator.cu:161-320) on the 64x32 cantilever, by hand."""
    g = synth.cantilever()
    m = orc.configure(g, radius=40e-6, density=1300.0, dtype=np.float64)
    l = 5e-3
    r = 40e-6
    mass_mid = (2 * l) * r * r * math.pi * 1300.0 / 2
    mass_tip = l * r * r * math.pi * 1300.0 / 2
    assert m["inv_mass"][0] == 0.0  # root pinned
    # positions are float32, so segment lengths carry ~1e-6 relative rounding
    assert m["inv_mass"][1] == pytest.approx(1 / mass_mid, rel=1e-5)
    assert m["inv_mass"][31] == pytest.approx(1 / mass_tip, rel=1e-5)
    mmrad = r * 1000
    ss = 3.9 * math.pi * mmrad ** 2
    assert m["k_stretch"][5] == pytest.approx(ss, rel=1e-6)
    bt = ss * mmrad ** 2 * 0.25 / l ** 2
    assert np.linalg.norm(m["q_rest"][5]) == pytest.approx(bt, rel=1e-5)
    # straight +x rods: identity orientations and rest Darboux along w
    np.testing.assert_allclose(m["q"][:31], np.tile([0, 0, 0, 1.0], (31, 1)), atol=1e-12)
    # flags: root has next + next orientation, interior all three, last-but-one no next orientation, tip fixed
    assert m["flags"][0] == orc.HAS_NEXT | orc.HAS_NEXT_ORIENTATION
    assert m["flags"][1] == orc.HAS_PREV | orc.HAS_NEXT | orc.HAS_NEXT_ORIENTATION
    assert m["flags"][30] == orc.HAS_PREV | orc.HAS_NEXT
    assert m["flags"][31] == orc.HAS_PREV | orc.FIX_ORIENTATION
    assert m["flags"][-1] == orc.HAS_PREV  # the last vertex of the whole set is not marked fixed
    assert m["l_rest"][31] == pytest.approx(1.0 / g.num_vertices)


def test_configure_rejects_bad_geometry():
    g = synth.cantilever(4, 8)
    g.positions[9] = g.positions[8]  # zero-length segment
    with pytest.raises(ValueError):
        orc.configure(g)


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_rest_state_stays_at_rest(schedule):
    g = synth.cantilever(8, 16)
    s = orc.OracleSim(g, num_itr=10, max_h=1 / 60, gravity=(0, 0, 0), schedule=schedule, dtype=np.float64)
    x0 = s.x.copy()
    for _ in range(5):
        s.advance(1 / 60)
    np.testing.assert_allclose(s.x, x0, atol=1e-14)
    assert np.abs(s.v).max() < 1e-12


def test_zero_iterations_is_the_predict_and_finish():
    """With no VBD iterations a step is x += dx0, v = dx0/h (1 - decay h) (iteration.cu:8-74)."""
    g = synth.cantilever(4, 8)
    v0 = helpers.random_velocities(g, 0.5).astype(np.float64)
    s = orc.OracleSim(g, num_itr=0, max_h=1 / 60, gravity=(0.1, 0.2, -9.81), dtype=np.float64, velocities=v0,
                      pin_roots=False)
    x0 = s.x.copy()
    h = float(np.float32(1 / 60))
    s.advance(1 / 60)
    # first step: v_last = 0, lastH = max_h, a = v0 / lastH, s = clamp(a.g / |g|^2, 0, 1)
    gv = np.array([0.1, 0.2, -9.81])
    acc = v0 / float(np.float32(1 / 60))
    sc = np.clip(acc @ gv / (gv @ gv), 0, 1)
    dx = h * v0 + (h * h * sc)[:, None] * gv
    np.testing.assert_allclose(s.x, x0 + dx, atol=1e-12)
    np.testing.assert_allclose(s.v, dx / h * (1 - 0.05 * h), atol=1e-10)
    np.testing.assert_allclose(s.v_last, v0, atol=0)


def test_translation_invariance():
    g = helpers.soft_groom(24, (6, 20))
    # on a 2^-20 m grid the offset below is exact in float32, so both grooms have the same geometry
    g.positions = (np.round(g.positions.astype(np.float64) * 2 ** 20) / 2 ** 20).astype(np.float32)
    v = helpers.random_velocities(g)
    set_ = helpers.soft_settings(gravity=(0.0, 0.0, -9.81))
    a = helpers.oracle_sim(g, set_, np.float64, v)
    g2 = synth.Groom(g.strand_begin, (g.positions + np.array([0.25, -1.5, 3.0], np.float32)), g.strand_young, g.strand_dev)
    b = helpers.oracle_sim(g2, set_, np.float64, v)
    for _ in range(4):
        a.advance(1 / 60)
        b.advance(1 / 60)
    da = a.x - g.positions.astype(np.float64)
    db = b.x - g2.positions.astype(np.float64)
    np.testing.assert_allclose(da, db, atol=1e-9)
    np.testing.assert_allclose(a.q, b.q, atol=1e-9)


@pytest.mark.parametrize("schedule", ["colour2", "jacobi"])
def test_unit_quaternions_and_fp32_vs_fp64(schedule):
    g = helpers.soft_groom(40, (6, 30))
    v = helpers.random_velocities(g)
    st = helpers.soft_settings(schedule=schedule)
    a = helpers.oracle_sim(g, st, np.float32, v)
    b = helpers.oracle_sim(g, st, np.float64, v)
    for _ in range(3):
        a.advance(1 / 60)
        b.advance(1 / 60)
    np.testing.assert_allclose(np.linalg.norm(a.q, axis=1), 1.0, atol=1e-5)
    assert np.abs(a.x - b.x).max() < 1e-5
    assert np.abs(orc.twist_angles(b.q, a.q)).max() < 1e-5


def _quat_mul(l, r):
    x = l[..., 3] * r[..., 0] + r[..., 3] * l[..., 0] + (l[..., 1] * r[..., 2] - r[..., 1] * l[..., 2])
    y = l[..., 3] * r[..., 1] + r[..., 3] * l[..., 1] + (l[..., 2] * r[..., 0] - r[..., 2] * l[..., 0])
    z = l[..., 3] * r[..., 2] + r[..., 3] * l[..., 2] + (l[..., 0] * r[..., 1] - r[..., 0] * l[..., 1])
    w = l[..., 3] * r[..., 3] - (l[..., 0] * r[..., 0] + l[..., 1] * r[..., 1] + l[..., 2] * r[..., 2])
    return np.stack([x, y, z, w], -1)


def _conj(q):
    return q * np.array([-1, -1, -1, 1.0])


def _numpy_step(groom, m, x, v, vl, q, h, last_h, grav, num_itr, damping=1e-6, decay=0.05):
    """Independent vectorised restatement of one colour2 substep (iteration.cu, cosserat.cu), FP64."""
    sb = groom.strand_begin
    nv = groom.num_vertices
    local = np.arange(nv) - np.repeat(sb[:-1], np.diff(sb))
    im, lr, ks, fl, qr = m["inv_mass"], m["l_rest"], m["k_stretch"], m["flags"], m["q_rest"]
    ext = np.asarray(grav, np.float64)
    dx = h * v
    free = im != 0
    y = v.copy()
    y[free] = dx[free] + h * h * ext
    acc = (v - vl) / last_h
    s = np.clip(acc @ ext / (ext @ ext), 0, 1)
    dx[free] += (h * h * s[free])[:, None] * ext
    vl = v.copy()
    damp = damping / h
    nxt = (fl & orc.HAS_NEXT) != 0
    prv = (fl & orc.HAS_PREV) != 0
    e = np.zeros_like(x)
    e[:-1] = x[1:] - x[:-1]

    def d3(qq):
        return np.stack([qq[:, 3] ** 2 + qq[:, 0] ** 2 - qq[:, 1] ** 2 - qq[:, 2] ** 2,
                         2 * (qq[:, 0] * qq[:, 1] + qq[:, 3] * qq[:, 2]),
                         2 * (qq[:, 0] * qq[:, 2] - qq[:, 3] * qq[:, 1])], 1)

    for _ in range(num_itr):
        for colour in (0, 1):
            sel = free & ((local & 1) == colour)
            idx = np.nonzero(sel)[0]
            a = 1.0 / (im[idx] * h * h)
            f = a[:, None] * (y[idx] - dx[idx])
            H = np.zeros((idx.size, 3, 3)) + a[:, None, None]
            D = d3(q)
            for which, sign in ((nxt, 1), (prv, -1)):
                ok = which[idx]
                j = idx[ok] if sign == 1 else idx[ok] - 1  # segment start
                invl = 1.0 / lr[j]
                c = (e[j] + dx[j + 1] - dx[j]) * invl[:, None] - D[j]
                k = ks[j] * invl
                d = k * invl
                f[ok] += sign * k[:, None] * c - (damp * d)[:, None] * dx[idx[ok]]
                H[ok] += (d * (1 + damp))[:, None, None] * np.eye(3)
            dx[idx] += np.linalg.solve(H, f[..., None])[..., 0]
        for colour in (0, 1):
            sel = nxt & ((fl & orc.FIX_ORIENTATION) == 0) & ((local & 1) == colour)
            idx = np.nonzero(sel)[0]
            V = -2 * ks[idx, None] * (e[idx] + dx[idx + 1] - dx[idx]) / lr[idx, None]
            b = np.zeros((idx.size, 4))
            okp = prv[idx]
            ip = idx[okp]
            phi = np.where(np.sum(_quat_mul(_conj(q[ip - 1]), q[ip]) * qr[ip - 1], 1) > 0, 1.0, -1.0)
            b[okp] += phi[:, None] * _quat_mul(q[ip - 1], qr[ip - 1])
            okn = (fl[idx] & orc.HAS_NEXT_ORIENTATION) != 0
            iN = idx[okn]
            phi = np.where(np.sum(_quat_mul(_conj(q[iN]), q[iN + 1]) * qr[iN], 1) > 0, 1.0, -1.0)
            b[okn] += phi[:, None] * _quat_mul(q[iN + 1], _conj(qr[iN]))
            lam = np.linalg.norm(V, axis=1) + np.linalg.norm(b, axis=1)
            Vq = np.concatenate([V, np.zeros((idx.size, 1))], 1)
            ex = np.tile([1.0, 0, 0, 0], (idx.size, 1))
            r = _quat_mul(_quat_mul(Vq, b), ex) + lam[:, None] * b
            q[idx] = r / np.linalg.norm(r, axis=1, keepdims=True)
    v = v.copy()
    v[free] = dx[free] / h * (1 - decay * h)
    return x + dx, v, vl, q


def test_oracle_matches_independent_numpy_restatement():
    g = helpers.soft_groom(12, (5, 14), seed=4)
    v0 = helpers.random_velocities(g, 0.4, seed=5).astype(np.float64)
    grav = (0.3, -0.4, -9.81)
    s = orc.OracleSim(g, num_itr=4, max_h=1 / 60, gravity=grav, radius=40e-6, dtype=np.float64, velocities=v0)
    m = dict(inv_mass=s.inv_mass, l_rest=s.l_rest, k_stretch=s.k_stretch, flags=s.flags, q_rest=s.q_rest)
    x, v, vl, q = s.x.copy(), s.v.copy(), s.v_last.copy(), s.q.copy()
    h = float(np.float32(1 / 60))
    last_h = h
    for step in range(3):
        s.advance(1 / 60)
        x, v, vl, q = _numpy_step(g, m, x, v, vl, q, h, last_h, grav, 4)
        np.testing.assert_allclose(s.x, x, atol=1e-11, err_msg=f"step {step}")
        np.testing.assert_allclose(s.v, v, atol=1e-8)
        np.testing.assert_allclose(s.q, q, atol=1e-7)


def test_sdf_projects_inside_points_to_the_shell():
    """A vertex inside the sphere lands on |p + ds/2| = R + threshold: the reference interpolates
    from idx - 0.5 (cudaSDFCollision.cu:140-142), i.e. it reads phi half a cell up each axis."""
    sdf = synth.sphere_sdf(128, radius=0.09, half_extent=0.2, threshold=1e-3)
    ds = 0.4 / 128
    rng = np.random.default_rng(1)
    n = 50
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    pos = np.zeros((n, 2, 3), np.float32)
    pos[:, 0] = 0.15 * dirs  # root outside, skipped by the pass
    pos[:, 1] = 0.08 * dirs
    g = synth.Groom(np.arange(0, 2 * n + 1, 2, dtype=np.int32), pos.reshape(-1, 3), np.full(n, 1.0, np.float32),
                    np.ones(n, np.float32))
    s = orc.OracleSim(g, num_itr=0, max_h=1 / 60, gravity=(0, 0, 0), sdf=sdf, dtype=np.float64)
    s.v[1::2] = 0.2 * dirs  # outward velocity is kept along the tangent only
    s.advance(1 / 60)
    p = s.x[1::2]
    r = np.linalg.norm(p + ds / 2, axis=1)
    np.testing.assert_allclose(r, 0.09 + 1e-3, atol=2e-4)
    np.testing.assert_allclose(s.x[0::2], pos[:, 0], atol=1e-7)  # roots untouched


def test_golden_fixture_regression():
    """The committed FP64 cantilever trajectory (tests/golden/make_golden.py) still reproduces."""
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "oracle_cantilever_f64.npz")
    ref = np.load(path)
    g = synth.cantilever(int(ref["num_rods"]), int(ref["verts"]), young=float(ref["young"]))
    g.strand_dev[:] = float(ref["deviation"])
    s = orc.OracleSim(g, num_itr=int(ref["num_itr"]), max_h=1 / 60, gravity=tuple(ref["gravity"]),
                      radius=float(ref["radius"]), schedule=str(ref["schedule"]), dtype=np.float64)
    for f in range(int(ref["frames"])):
        s.advance(1 / 60)
    np.testing.assert_allclose(s.x, ref["x"], atol=1e-12)
    np.testing.assert_allclose(s.q, ref["q"], atol=1e-12)


# ---- pins against KamiSimulator's own code, run on a GPU (tests/golden/make_ref_fixtures.py) ----
def _ref_pins():
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_pins.npz"))


@pytest.mark.parametrize("case", ["cant", "groom"])
def test_configure_matches_reference_fixture(case):
    ref = _ref_pins()
    if case == "cant":
        g = synth.cantilever()
    else:
        g = synth.groom(100, 64, seed=2)
        g.strand_young[:] = 2.0
    o = orc.configure(g, dtype=np.float32)
    np.testing.assert_array_equal(o["flags"], ref[f"{case}_flags"])
    for k in ("inv_mass", "l_rest", "k_stretch", "q", "q_rest"):
        np.testing.assert_allclose(o[k], ref[f"{case}_{k}"], rtol=5e-7, atol=1e-7, err_msg=k)  # <= 4 ulp


def test_jacobi_trajectories_match_reference_fixture():
    """The reference's Jacobi kernels race at block boundaries (run-to-run spread ~3e-8 m here)."""
    ref = _ref_pins()
    g = synth.groom(100, 64, seed=2)
    g.strand_young[:] = 2.0
    s = orc.OracleSim(g, num_itr=20, max_h=1 / 120, schedule="jacobi")
    for f in range(3):
        s.advance(1 / 120)
        assert np.abs(s.x - ref["jgroom_x"][f]).max() < 1e-6
        assert np.abs(orc.twist_angles(ref["jgroom_q"][f], s.q)).max() < 1e-5
    g = synth.cantilever(8, 16, young=1e-3)
    s = orc.OracleSim(g, num_itr=10, max_h=1 / 60, schedule="jacobi")
    for f in range(6):
        s.advance(1 / 60)
        assert np.abs(s.x - ref["jsoft_x"][f]).max() < 1e-6
        assert np.abs(orc.twist_angles(ref["jsoft_q"][f], s.q)).max() < 1e-5


@pytest.mark.parametrize("name", ["sphere", "capsules"])
def test_sdf_pass_matches_reference_fixture(name):
    ref = _ref_pins()
    sdf = synth.sphere_sdf(32) if name == "sphere" else synth.capsule_union_sdf(24, num_capsules=5)
    p, v, li = ref[f"sdf_{name}_p"], ref[f"sdf_{name}_v"], ref[f"sdf_{name}_li"]
    # 250 strands of 8 particles: local index = position in the strand, as in the fixture
    g = synth.Groom(np.arange(0, p.shape[0] + 1, 8, dtype=np.int32), p, np.ones(p.shape[0] // 8, np.float32),
                    np.ones(p.shape[0] // 8, np.float32))
    assert np.array_equal(li, np.arange(p.shape[0]) % 8)
    s = orc.OracleSim(g, num_itr=0, max_h=1.0, gravity=(0, 0, 0), sdf=sdf, pin_roots=False, velocity_decay=0.0)
    s.set_body_transform(tuple(ref[f"sdf_{name}_rot"]), tuple(ref[f"sdf_{name}_tr"]))
    s.advance(1e-3)  # zero velocity, zero gravity: positions unchanged, then the SDF pass
    assert np.mean(np.any(ref[f"sdf_{name}_pout"] != p, axis=1)) > 0.01
    np.testing.assert_allclose(s.x, ref[f"sdf_{name}_pout"], atol=1e-6)


def test_flop_count_pins_the_roofline_constant():
    # the FP32 roofline in bench.py divides by the reference algorithm's FLOPs per vertex-iteration;
    # the constant there must be the oracle's count
    import ast
    import os

    pos, ori = orc.flop_count()
    assert (pos, ori) == (242, 250)
    src = open(os.path.join(os.path.dirname(os.path.dirname(__file__)), "bench.py")).read()
    consts = {n.targets[0].id: n.value.value for n in ast.parse(src).body
              if isinstance(n, ast.Assign) and isinstance(n.targets[0], ast.Name) and isinstance(n.value, ast.Constant)}
    assert consts["REFERENCE_FLOP_PER_VERTEX_ITER"] == pos + ori


@pytest.mark.parametrize("wind", [(0.0, 1.0, 0.7, 0.4, 3.0), (6.0, 1.0, 0.7, 0.4, 3.0), (6.0, 1.0, 0.7, 0.4, 2.5)])
def test_fp64_autograd_restatement_follows_the_fp64_oracle(wind):
    """oracle/torch_ref.py, the FP64 reference of the adjoint tests, against the FP64 oracle over 6
    frames: SDF on, and wind off, with an odd integer sharpness and with a fractional one."""
    import torch

    from oracle.torch_ref import TorchVBD

    g = helpers.soft_groom(24, (6, 20), seed=31, young_scale=1e-3)
    v0 = helpers.random_velocities(g, 0.15, seed=32)
    sdf = synth.sphere_sdf(48, threshold=2e-3)
    st = dict(num_itr=5, max_h=1 / 60, gravity=(0.3, -0.4, -9.81), radius=40e-6)
    o = orc.OracleSim(g, dtype=np.float64, wind=wind, sdf=sdf, velocities=v0, **st)
    m = orc.configure(g, radius=st["radius"], dtype=np.float64)
    tv = TorchVBD(g, m, num_itr=5, max_h=1 / 60, gravity=st["gravity"], sdf=sdf, wind=wind)
    state = (torch.tensor(g.positions.astype(np.float64)), torch.tensor(v0.astype(np.float64)),
             torch.zeros(g.num_vertices, 3, dtype=torch.float64), torch.tensor(m["q"]), float(np.float32(1 / 60)))
    qr = torch.tensor(m["q_rest"])
    for _ in range(6):
        state = tv.step(state, qr, 1 / 60)
        o.advance(1 / 60)
    # the oracle rounds the wind's cosine argument to float, as the reference does
    np.testing.assert_allclose(state[0].numpy(), o.x, rtol=0, atol=1e-9)
    np.testing.assert_allclose(state[3].numpy(), o.q, rtol=0, atol=1e-8)


def test_strain_limiting_restatement_on_a_hand_case():
    """StrainLimiting (cudaSDFCollision.cu:176-199): from the root, a segment whose length is off its
    rest length by more than StrainError x l0 gets its far vertex pulled along the segment to l0; the
    next segment is then measured from the corrected vertex.  Segments inside the tolerance stay."""
    x = np.array([[0, 0, 0], [0, 0, 1.5], [0, 0, 2.0], [0, 0, 3.05],
                  [1, 0, 0], [1, 0, 0.5], [1, 0.6, 0.5]], np.float32)
    sb = np.array([0, 4, 7], np.int32)
    l0 = np.array([1, 1, 1, 0, 1, 0.5, 0], np.float32)
    out = orc.strain_limit(x, sb, l0, 0.1)
    # strand 0: 1.5 -> 1 (vertex 1 to z = 1); vertex 2 is then 1.0 from it (kept); 1.05 is within 10 % (kept)
    np.testing.assert_allclose(out[:4], [[0, 0, 0], [0, 0, 1], [0, 0, 2], [0, 0, 3.05]], atol=1e-6)
    # strand 1: 0.5 against 1 -> vertex 5 pushed out to z = 1; the 0.6 segment is then measured from there
    assert abs(np.linalg.norm(out[5] - out[4]) - 1.0) < 1e-6
    np.testing.assert_allclose(out[5], [1, 0, 1], atol=1e-6)
    d6 = np.linalg.norm(out[6] - out[5])
    assert abs(d6 - 0.5) < 1e-6  # |(1, 0.6, 0.5) - (1, 0, 1)| = 0.781 > 1.1 x 0.5: pulled to 0.5
    # a tolerance that covers every strain changes nothing
    np.testing.assert_array_equal(orc.strain_limit(x, sb, l0, 10.0), x)
