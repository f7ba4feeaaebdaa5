"""The C++ Solver plugin (kamisimulator_b200/plugin): KamiSimulator's solver calls
(Construct(settings json), SolveNextStep(dt), DownloadHair) on a Hair-like padded strand array."""
import json
import os
import subprocess

import numpy as np
import pytest

from kamisimulator_b200 import synth
from tests import helpers

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "kamisimulator_b200", "lib", "kami_solver_driver")

# the keys and values of the reference's scripts/json/StCossRods.json
REFERENCE_SETTINGS = {
    "EnableResample": True, "EnableSDF": True, "EnableHairHairColl": False, "UseYoungsModule": True, "NumItr": 32,
    "SagFreeItr": 1, "SubdivCoeff": 3, "StretchK": 3e3, "BendK": 6e-4, "YoungsModule": 5,
    "StiffnessDeviationCoeff": 1, "CurveRadius": 4e-5, "Density": 1.3e6, "ResampleLen": 1e-3,
    "VelocityDecay": 0.05, "ExternalForceMultiplier": 1, "WindPeak": 40, "WindYFreq": 1, "WindZFreq": 0.7,
    "WindTimeFreq": 0.4, "WindSharpness": 3.0,
}


def write_hair(path, groom, pad_to=None):
    counts = np.diff(groom.strand_begin).astype(np.uint32)
    mv = int(pad_to or counts.max())
    arr = np.zeros((groom.num_strands, mv, 3), np.float32)
    for s in range(groom.num_strands):
        a, b = groom.strand_begin[s], groom.strand_begin[s + 1]
        arr[s, : b - a] = groom.positions[a:b]
    with open(path, "wb") as f:
        f.write(np.array([groom.num_strands, mv], np.uint32).tobytes())
        f.write(counts.tobytes())
        f.write(arr.tobytes())
    return counts, mv


def read_out(path, ns, mv):
    data = np.fromfile(path, np.float32)
    n = ns * mv * 3
    return data[:n].reshape(ns, mv, 3), data[n:2 * n].reshape(ns, mv, 3)


def test_descriptor_from_reference_settings(tmp_path):
    # strands of 3 vertices are skipped, as StableCosseratRodsSolver::BuildYarnBallHair does
    lens = np.array([10, 3, 12, 2, 8])
    g = synth.groom_strands(np.random.default_rng(0), lens)
    write_hair(tmp_path / "hair.bin", g)
    (tmp_path / "s.json").write_text(json.dumps(REFERENCE_SETTINGS))
    out = subprocess.run([DRIVER, "--dry-run", str(tmp_path / "s.json"), str(tmp_path / "hair.bin")],
                         capture_output=True, text=True, check=True).stdout
    d = json.loads(out)
    assert d["num_strands"] == 3 and d["num_vertices"] == 30
    assert d["num_itr"] == 32
    assert d["radius"] == pytest.approx(0.05 * 4e-5)  # StableCosseratRodsSolver.cpp:177-179
    assert d["density"] == pytest.approx(1.3e6)
    assert d["young"] == pytest.approx(5.0) and d["deviation"] == pytest.approx(1.0) and d["stiffness_mode"] == 0
    assert d["wind_peak"] == pytest.approx(40.0) and d["velocity_decay"] == pytest.approx(0.05)
    assert d["max_h"] == pytest.approx(4e-4)  # Sim::maxH
    assert d["gravity"] == pytest.approx([0.0, -9.8, 0.0])
    assert d["sag_free_itr"] == 1


def test_invalid_settings_are_rejected(tmp_path):
    g = synth.cantilever(2, 8)
    write_hair(tmp_path / "hair.bin", g)
    (tmp_path / "s.json").write_text(json.dumps({"Schedule": "gauss-seidel"}))
    r = subprocess.run([DRIVER, "--dry-run", str(tmp_path / "s.json"), str(tmp_path / "hair.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "Schedule" in r.stderr
    # features of the reference this solver does not build are refused, not ignored
    (tmp_path / "scene.json").write_text("{}")
    for bad, word in (({"YBJsonPath": str(tmp_path / "scene.json")}, "YBJsonPath"),
                      ({"UseStrainLimiting": True, "StrainError": -0.1}, "StrainError")):
        (tmp_path / "s.json").write_text(json.dumps(bad))
        r = subprocess.run([DRIVER, "--dry-run", str(tmp_path / "s.json"), str(tmp_path / "hair.bin")],
                           capture_output=True, text=True)
        assert r.returncode == 1 and word in r.stderr, r.stderr
    # a YBJsonPath that names no file falls back to the Hair, as in the reference (IsFileExist)
    (tmp_path / "s.json").write_text(json.dumps({"YBJsonPath": str(tmp_path / "missing.json")}))
    subprocess.run([DRIVER, "--dry-run", str(tmp_path / "s.json"), str(tmp_path / "hair.bin")], check=True,
                   capture_output=True)


def test_strain_limiting_settings(tmp_path):
    """The SDF solver's UseStrainLimiting and StrainError (SDFBodyCollisionSolver.cpp:36-37), off and
    0.1 by default (SDFBodyCollisionSolver.h:26-27)."""
    g = synth.cantilever(2, 8)
    write_hair(tmp_path / "hair.bin", g)
    for settings, on, err in (({}, 0, 0.1), ({"UseStrainLimiting": True}, 1, 0.1),
                              ({"UseStrainLimiting": True, "StrainError": 0.05}, 1, 0.05)):
        (tmp_path / "s.json").write_text(json.dumps(settings))
        out = subprocess.run([DRIVER, "--dry-run", str(tmp_path / "s.json"), str(tmp_path / "hair.bin")],
                             capture_output=True, text=True, check=True).stdout
        d = json.loads(out)
        assert d["strain_limiting"] == on and d["strain_error"] == pytest.approx(err)


def test_sag_free_setting(tmp_path):
    g = synth.cantilever(2, 8)
    write_hair(tmp_path / "hair.bin", g)
    (tmp_path / "s.json").write_text(json.dumps({"SagFreeItr": 3}))
    out = subprocess.run([DRIVER, "--dry-run", str(tmp_path / "s.json"), str(tmp_path / "hair.bin")],
                         capture_output=True, text=True, check=True).stdout
    assert json.loads(out)["sag_free_itr"] == 3


def test_hair_hair_settings(tmp_path):
    g = synth.cantilever(2, 8)
    write_hair(tmp_path / "hair.bin", g)
    (tmp_path / "s.json").write_text(json.dumps({"EnableHairHairColl": True, "CurveRadius": 5e-5}))
    out = subprocess.run([DRIVER, "--dry-run", str(tmp_path / "s.json"), str(tmp_path / "hair.bin")],
                         capture_output=True, text=True, check=True).stdout
    d = json.loads(out)
    assert d["hair_hair"] == 1 and d["step_limit"] == 1
    assert d["barrier_thickness"] == pytest.approx(2 * 0.95 * 5e-5)  # StableCosseratRodsSolver.cpp:180


@pytest.mark.gpu
def test_plugin_steps_match_the_c_abi_and_the_oracle(tmp_path):
    g = helpers.soft_groom(40, (6, 30), seed=12)
    counts, mv = write_hair(tmp_path / "hair.bin", g, pad_to=40)
    settings = {"NumItr": 6, "UseYoungsModule": True, "YoungsModule": 1e-4, "StiffnessDeviationCoeff": 0.5,
                "CurveRadius": 40e-6 / 0.05, "Density": 1300, "VelocityDecay": 0.05, "WindPeak": 0,
                "EnableSDF": False, "MaxTimeStep": 1 / 60, "Gravity": [0.3, -0.4, -9.81],
                "SubdivCoeff": 1, "EnableResample": False}
    (tmp_path / "s.json").write_text(json.dumps(settings))
    steps = 5
    subprocess.run([DRIVER, str(tmp_path / "s.json"), str(tmp_path / "hair.bin"), str(steps), str(1 / 60),
                    str(tmp_path / "out.bin")], check=True, capture_output=True)
    pos, _ = read_out(tmp_path / "out.bin", g.num_strands, mv)
    packed = np.concatenate([pos[s, : counts[s]] for s in range(g.num_strands)])
    st = dict(num_itr=6, max_h=1 / 60, gravity=(0.3, -0.4, -9.81), radius=40e-6, velocity_decay=0.05)
    g.strand_young[:] = 1e-4
    g.strand_dev[:] = 0.5
    s = helpers.gpu_solver(g, st)
    o = helpers.oracle_sim(g, st, np.float32)
    for _ in range(steps):
        s.step(1 / 60)
        o.advance(1 / 60)
    x, _ = s.get_positions_velocities()
    s.close()
    # the plugin's radius is 0.05 x CurveRadius in float, within an ulp of the 40 um given to the C ABI here
    np.testing.assert_allclose(packed, x, atol=1e-6)
    assert np.abs(packed - o.x).max() <= helpers.POS_TOL
    assert np.abs(packed - g.positions).max() > 1e-4  # the strands moved


@pytest.mark.gpu
def test_plugin_strain_limiting_after_each_step(tmp_path):
    """UseStrainLimiting: every SolveNextStep is followed by the SDF solver's strain limiting, as
    SDFBodyCollisionSolver::SolveNextStep runs it after its SDF pass (SDFBodyCollisionSolver.cpp:186);
    the same as kami_vbd_step then kami_vbd_strain_limit through the C ABI."""
    g = helpers.soft_groom(40, (6, 30), seed=12)
    counts, mv = write_hair(tmp_path / "hair.bin", g, pad_to=40)
    settings = {"NumItr": 6, "UseYoungsModule": True, "YoungsModule": 1e-4, "StiffnessDeviationCoeff": 0.5,
                "CurveRadius": 40e-6 / 0.05, "Density": 1300, "VelocityDecay": 0.05, "WindPeak": 0,
                "EnableSDF": True, "UseStrainLimiting": True, "StrainError": 0.002, "MaxTimeStep": 1 / 60,
                "Gravity": [0.3, -0.4, -9.81], "SubdivCoeff": 1, "EnableResample": False}
    (tmp_path / "s.json").write_text(json.dumps(settings))
    steps = 5
    subprocess.run([DRIVER, str(tmp_path / "s.json"), str(tmp_path / "hair.bin"), str(steps), str(1 / 60),
                    str(tmp_path / "out.bin")], check=True, capture_output=True)
    pos, _ = read_out(tmp_path / "out.bin", g.num_strands, mv)
    packed = np.concatenate([pos[s, : counts[s]] for s in range(g.num_strands)])
    st = dict(num_itr=6, max_h=1 / 60, gravity=(0.3, -0.4, -9.81), radius=40e-6, velocity_decay=0.05)
    g.strand_young[:] = 1e-4
    g.strand_dev[:] = 0.5
    limited, free = helpers.gpu_solver(g, st), helpers.gpu_solver(g, st)
    for _ in range(steps):
        limited.step(1 / 60)
        limited.strain_limit(0.002)
        free.step(1 / 60)
    x, _ = limited.get_positions_velocities()
    xf, _ = free.get_positions_velocities()
    limited.close()
    free.close()
    np.testing.assert_allclose(packed, x, atol=1e-6)
    assert np.abs(x - xf).max() > 1e-5  # the limit changed the motion


@pytest.mark.gpu
def test_plugin_reads_and_writes_usc_data_files(tmp_path):
    """The driver loads a USC-HairSalon .data file into a Hair of 100 vertices per strand (skipping
    strands under 4 vertices), steps it, and exports the Hair as .data: the same result as the
    binary Hair path."""
    from kamisimulator_b200 import vbd

    g = helpers.soft_groom(30, (2, 40), seed=14)
    counts = np.diff(g.strand_begin).astype(np.int32)
    vbd.write_usc(tmp_path / "in.data", counts, g.positions)
    write_hair(tmp_path / "hair.bin", g, pad_to=100)
    settings = {"NumItr": 6, "UseYoungsModule": True, "YoungsModule": 1e-4, "CurveRadius": 40e-6 / 0.05,
                "WindPeak": 0, "EnableSDF": False, "MaxTimeStep": 1 / 60, "Gravity": [0.3, -0.4, -9.81],
                "SubdivCoeff": 1, "EnableResample": False}
    (tmp_path / "s.json").write_text(json.dumps(settings))
    for src, dst in (("in.data", "out.data"), ("hair.bin", "out.bin")):
        subprocess.run([DRIVER, str(tmp_path / "s.json"), str(tmp_path / src), "4", str(1 / 60), str(tmp_path / dst)],
                       check=True, capture_output=True)
    c, xd = vbd.read_usc(tmp_path / "out.data", max_verts=100)
    xb, _ = read_out(tmp_path / "out.bin", g.num_strands, 100)
    np.testing.assert_array_equal(c, counts)
    for s in range(g.num_strands):
        np.testing.assert_array_equal(xd[s, :counts[s]], xb[s, :counts[s]])
    moved = [s for s in range(g.num_strands) if counts[s] >= 4]
    assert max(np.abs(xd[s, :counts[s]] - g.positions[g.strand_begin[s]:g.strand_begin[s + 1]]).max()
               for s in moved) > 1e-4


@pytest.mark.gpu
def test_plugin_subdivides_and_resamples_the_hair(tmp_path):
    """With the reference solver's defaults (SubdivCoeff 3, EnableResample at ResampleLen), Construct
    subdivides and resamples the Hair first: the result equals kami_hair_subdivide +
    kami_hair_resample followed by the C ABI."""
    from kamisimulator_b200 import vbd

    g = helpers.soft_groom(20, (6, 14), seed=15)
    counts, mv = write_hair(tmp_path / "hair.bin", g, pad_to=16)
    settings = {"NumItr": 6, "UseYoungsModule": True, "YoungsModule": 1e-4, "CurveRadius": 40e-6 / 0.05,
                "WindPeak": 0, "EnableSDF": False, "MaxTimeStep": 1 / 60, "Gravity": [0.3, -0.4, -9.81],
                "ResampleLen": 1.5e-3}
    (tmp_path / "s.json").write_text(json.dumps(settings))
    subprocess.run([DRIVER, str(tmp_path / "s.json"), str(tmp_path / "hair.bin"), "3", str(1 / 60),
                    str(tmp_path / "out.bin")], check=True, capture_output=True)
    padded = np.zeros((g.num_strands, 16, 3), np.float32)
    for s in range(g.num_strands):
        padded[s, :counts[s]] = g.positions[g.strand_begin[s]:g.strand_begin[s + 1]]
    c3, x3 = vbd.hair_subdivide(counts, padded, 3)
    cr, xr = vbd.hair_resample(c3, x3, 1.5e-3)
    assert (cr != c3).any()
    keep = [s for s in range(g.num_strands) if cr[s] >= 4]
    pos = np.concatenate([xr[s, :cr[s]] for s in keep])
    gg = synth.Groom(strand_begin=np.concatenate([[0], np.cumsum([cr[s] for s in keep])]).astype(np.int32),
                     positions=pos, strand_young=np.full(len(keep), 1e-4, np.float32),
                     strand_dev=np.ones(len(keep), np.float32))
    st = dict(num_itr=6, max_h=1 / 60, gravity=(0.3, -0.4, -9.81), radius=np.float32(0.05) * np.float32(40e-6 / 0.05),
              velocity_decay=0.05)
    s = helpers.gpu_solver(gg, st, form="fused")
    for _ in range(3):
        s.step(1 / 60)
    x = s.get_positions_velocities()[0]
    s.close()
    out, _ = read_out(tmp_path / "out.bin", g.num_strands, (16 - 1) * 3 + 1)
    got = np.concatenate([out[s, :cr[s]] for s in keep])
    np.testing.assert_allclose(got, x, atol=1e-6)


def write_sdf(path, sdf):
    with open(path, "wb") as f:
        f.write(np.array(sdf.dims, np.int32).tobytes())
        f.write(np.array(sdf.grid_min, np.float32).tobytes())
        f.write(np.array(sdf.grid_max, np.float32).tobytes())
        f.write(np.ascontiguousarray(sdf.phi, np.float32).tobytes())
        f.write(np.ascontiguousarray(sdf.grad, np.float32).tobytes())


@pytest.mark.gpu
def test_plugin_runs_the_reference_default_settings(tmp_path):
    """The reference's own default settings (subdivision x3, resampling to 1 mm, one sag-free pass,
    NumItr 32, wind, the head SDF, Sim::maxH 4e-4 s, so 42 substeps per 1/60 s frame).  The resampled
    strands are longer than a tile of 128 slots and run on the fused form in groups of tiles; two
    frames of the plugin equal the same preprocessing and set-up through the C ABI."""
    from kamisimulator_b200 import vbd

    rng = np.random.default_rng(31)
    g = synth.groom_strands(rng, rng.integers(8, 31, 30), seg_len=6e-3)
    pad = 64  # resampled strands are capped at the Hair's row length, (64 - 1) * 3 + 1 after subdivision
    counts, mv = write_hair(tmp_path / "hair.bin", g, pad_to=pad)
    sdf = synth.sphere_sdf(64, threshold=1e-3)
    write_sdf(tmp_path / "sdf.bin", sdf)
    (tmp_path / "s.json").write_text(json.dumps(dict(REFERENCE_SETTINGS, SDFThreshold=1e-3)))
    subprocess.run([DRIVER, str(tmp_path / "s.json"), str(tmp_path / "hair.bin"), "2", str(1 / 60),
                    str(tmp_path / "out.bin"), str(tmp_path / "sdf.bin")], check=True, capture_output=True)
    padded = np.zeros((g.num_strands, pad, 3), np.float32)
    for s in range(g.num_strands):
        padded[s, :counts[s]] = g.positions[g.strand_begin[s]:g.strand_begin[s + 1]]
    c3, x3 = vbd.hair_subdivide(counts, padded, 3)
    cr, xr = vbd.hair_resample(c3, x3, 1e-3)
    assert cr.max() > 128  # longer than a tile
    keep = [s for s in range(g.num_strands) if cr[s] >= 4]
    pos = np.concatenate([xr[s, :cr[s]] for s in keep])
    gg = synth.Groom(strand_begin=np.concatenate([[0], np.cumsum([cr[s] for s in keep])]).astype(np.int32),
                     positions=pos, strand_young=np.full(len(keep), 5.0, np.float32),
                     strand_dev=np.ones(len(keep), np.float32))
    st = dict(num_itr=32, max_h=4e-4, gravity=(0.0, -9.8, 0.0), radius=np.float32(0.05) * np.float32(4e-5),
              density=1.3e6, velocity_decay=0.05, wind=(40.0, 1.0, 0.7, 0.4, 3.0), sdf=sdf, young=5.0,
              deviation=1.0, per_strand=False, sag_free_itr=1)
    s = helpers.gpu_solver(gg, st, form="auto")
    assert s.slots_per_lane == 4  # fused, in groups of tiles
    for _ in range(2):
        s.step(1 / 60)
    x = s.get_positions_velocities()[0]
    s.close()
    out, _ = read_out(tmp_path / "out.bin", g.num_strands, (pad - 1) * 3 + 1)
    got = np.concatenate([out[s, :cr[s]] for s in keep])
    assert np.isfinite(got).all()
    np.testing.assert_allclose(got, x, atol=1e-6)
