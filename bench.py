"""Benchmark of the Stable Cosserat Rods VBD step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload: the synthetic groom of 10,000 strands x 64 vertices (roots on the upper
hemisphere of a 0.09 m head sphere, helical curl, per-strand E log-uniform in [1, 5] GPa), 20 VBD
iterations per 1/120 s step, the head-sphere SDF on a 128^3 grid, colour2 schedule, FP32.
Metric: VBD vertex-iterations per second (vertices x iterations x steps / time), whole job.

`value` times the fused step kernel with the state resident in HBM; the 95 MB working set fits
the 126 MB L2, so a 256 MiB buffer is written between timed steps and only the step kernels are
timed (CUDA events on the launching stream).  `e2e` is the same metric through the C ABI with
host buffers: every frame is one kami_vbd_step_hair call on the plugin's page-locked padded Hair
arrays, which uploads positions/velocities (UploadHair), steps and writes them back (DownloadHair)
from one kernel, overlapping the PCIe traffic of one tile with the step of another (the plugin's
SolveNextStep + DownloadHair path); `packed_step_host_value` is kami_vbd_step_host on packed
arrays, and `three_calls_value` is the same frame as
kami_vbd_set_positions_velocities, kami_vbd_step, kami_vbd_get_positions_velocities in turn.  Extra
`forms` report the sweep form, the batched form on 64 uneven grooms against the same grooms as one
plain (fused, autotuned) handle each, and the other production forms; `trajectory` states the FP32
GPU trajectory's distance to an FP64 replay of the same update over 100 frames.  With N > 1 (torchrun) each rank steps its own groom
(weak scaling, no collective on the data path); times are maxima over ranks.

--impl reference times the CPU restatement of the reference's update (oracle/, Jacobi schedule =
the reference's cosseratItr/quaternionLambdaItr order) with every host thread on a bounded sample
of the same groom; the reference has no CPU implementation of this step of its own.
"""
from __future__ import annotations

import argparse
import math
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "groom_10k_x64"
DT = 1.0 / 120.0
NUM_ITR = 20
METRIC = "VBD vertex-iters/s"
UNIT = "vertex-iters/s"
BYTES_PER_VERTEX_STEP = 160  # fused kernel: 6 float4 loads + 4 float4 stores per vertex
# FLOPs of one vertex-iteration of the reference algorithm (cosseratItr 242 + quaternionLambdaItr
# 250), counted by the oracle's op-counting scalar; tests/test_oracle.py keeps this in step with it.
REFERENCE_FLOP_PER_VERTEX_ITER = 492
# Nominal FP32 peak of a B200: 148 SMs x 128 FMA lanes x 2 FLOP x 1965 MHz.
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
FALLBACK_HBM_GBS = 6650.0


def settings():
    from kamisimulator_b200 import synth

    return dict(num_itr=NUM_ITR, max_h=DT, gravity=(0.0, 0.0, -9.81), radius=40e-6, density=1300.0,
                velocity_decay=0.05, damping=1e-6, sdf=synth.sphere_sdf(128, threshold=1e-3))


def config_dict(extra=None):
    c = {"workload": f"{WORKLOAD}: 10,000 strands x 64 vertices, {NUM_ITR} VBD iterations, dt 1/120 s, "
                     "head-sphere SDF 128^3, colour2 schedule",
         "strands": 10000, "verts_per_strand": 64, "num_itr": NUM_ITR, "dt": DT, "sdf_grid": [128, 128, 128],
         "l2": "flushed between timed steps (256 MiB write), working set 95 MB < L2"}
    if extra:
        c.update(extra)
    return c


def fp32_probe(device=0):
    """Measured FP32 FMA throughput of a GPU in TFLOP/s, (plain FFMA chains, packed FFMA2 chains), from
    the bench-only probe library (kamisimulator_b200/csrc/fp32_probe.cu)."""
    import ctypes

    lib = ctypes.CDLL(os.path.join(ROOT, "kamisimulator_b200", "lib", "libkami_fp32_probe.so"))
    lib.kami_fp32_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.kami_fp32_peak.restype = ctypes.c_int
    fma, fma2 = ctypes.c_double(), ctypes.c_double()
    rc = lib.kami_fp32_peak(device, ctypes.byref(fma), ctypes.byref(fma2))
    if rc != 0:
        raise RuntimeError(f"kami_fp32_peak failed with cudaError {rc}")
    return fma.value, fma2.value


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the fused step kernel from the committed ncu capture summary."""
    p = os.path.join(ROOT, "profiles", "fused_step_groom_10k_x64.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch"), d
    except Exception:
        return None, None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpus):
        self.gpus = gpus
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.12)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (getattr(self, "out", "") or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                idx = int(parts[0])
            except ValueError:
                continue
            if idx not in self.gpus:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                pass
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(value, world, device="cuda"):
    """Largest `value` over all ranks (the job's time is the slowest rank's); identity for one rank."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, vertices_per_rank, num_itr, steps, max_ms):
    """Whole-job vertex-iterations per second: every rank steps its own groom (weak scaling)."""
    return world * vertices_per_rank * num_itr * steps / (max_ms / 1e3)


def rank_groom(rank):
    """The groom a rank steps: every rank its own 10,000 x 64 groom of the headline generator, seeded
    by the rank (rank 0 is the headline groom), so that ranks share nothing but the clock."""
    from kamisimulator_b200 import synth

    return synth.groom(10_000, 64, seed=2 + rank)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# --------------------------------------------------------------------------------------------------
# reference arm: CPU restatement of the reference's update on every host thread
# --------------------------------------------------------------------------------------------------
def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from kamisimulator_b200 import synth
    from oracle.oracle import OracleSim, load

    lib = load()
    threads = lib.oracle_num_threads()
    full = synth.groom()
    st = settings()
    # calibrate on one full-size frame, then bound each timed step to a strand subset
    cal = OracleSim(full, schedule="jacobi", num_threads=threads, **st)
    t0 = time.perf_counter()
    cal.advance(DT)
    t_full = time.perf_counter() - t0
    budget = 100.0 / max(1, args.steps + args.warmup)
    strands = int(max(64, min(10000, 10000 * budget / max(t_full, 1e-6))))
    sub = synth.groom(strands, 64, seed=2)
    sim = OracleSim(sub, schedule="jacobi", num_threads=threads, **st)
    for _ in range(args.warmup):
        sim.advance(DT)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.advance(DT)
    el = time.perf_counter() - t0
    units = sub.num_vertices * NUM_ITR * args.steps
    value = units / el
    sample = (f"{strands} of the 10,000 strands (x 64 vertices) per step, jacobi schedule, FP32, "
              f"{args.steps} steps; full-size frame took {t_full:.3f} s")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps * (10000 / strands),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict({"sample_strands": strands,
                                   "schedule": "jacobi (the reference's cosseratItr / quaternionLambdaItr order)"}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------------------------------
def time_steps(solver, steps, stream, flush):
    import torch

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for k in range(steps):
        flush.fill_(k & 0xFF)
        starts[k].record(stream)
        solver.step(DT, stream=stream)
        ends[k].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in zip(starts, ends))


def cpu_baseline_sample():
    from kamisimulator_b200 import synth
    from oracle.oracle import OracleSim, load

    threads = load().oracle_num_threads()
    g = synth.groom()
    sim = OracleSim(g, schedule="colour2", num_threads=threads, **settings())
    frames, t0 = 0, time.perf_counter()
    while frames < 3 or (time.perf_counter() - t0 < 10.0 and frames < 60):
        sim.advance(DT)
        frames += 1
    el = time.perf_counter() - t0
    return {"value": g.num_vertices * NUM_ITR * frames / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{frames} full-size frames of the 10,000 x 64 groom, colour2 schedule, FP32 "
                      f"(oracle/kami_oracle.cpp, OpenMP)"}


def batched_timing(torch, stream, flush, num_grooms=64, per_groom_handles=True, tuning=None):
    """kami_vbd_batch_step over `num_grooms` uneven grooms (strands log-uniform [500, 20000], 16-128
    vertices) in one handle, against the same grooms as one plain drop-in handle each (form auto =
    fused, each autotuned) and as sweep-form handles, stepped one after another.  `tuning` fixes the
    batch's tile shape instead of autotuning it (profiling runs)."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.vbd import Solver

    st = settings()
    grooms = synth.batched_grooms(num_grooms)
    V = sum(gg.num_vertices for gg in grooms)
    b = Solver(grooms, form="fused", **st)  # kami_vbd_batch_create
    if tuning:
        b.set_tuning(*tuning)
        best = b.get_tuning()
    else:
        best, _ = b.autotune(DT, trial_steps=8)
    nb = 24
    b.batch_step(DT, nb, stream=stream)  # warm-up: captures the graph for n = nb
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.fill_(1)
    e0.record(stream)
    b.batch_step(DT, nb, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1)
    b.close()

    def per_groom(form, rounds):
        """The grooms as one handle each (the CantileverTestSolver pattern: one Sim per instance,
        stepped one after another, src/solvers/CantileverTestSolver.cpp:106-111)."""
        hs = [Solver(gg, form=form, **st) for gg in grooms]
        if form == "auto":  # the plain drop-in: fused, each handle autotuned on its own strands
            for hh in hs:
                hh.autotune(DT, trial_steps=4)
        for hh in hs:
            hh.step(DT, stream=stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(rounds):
            for hh in hs:
                hh.step(DT, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        for hh in hs:
            hh.close()
        return V * NUM_ITR * rounds / (ms / 1e3), ms / rounds

    vb = V * NUM_ITR * nb / (ms_b / 1e3)
    res = {"value": vb, "ms_per_step": ms_b / nb, "vertices": V, "grooms": num_grooms,
           "tuning": {"slots_per_lane": best[0], "warps_per_block": best[1], "steps_per_launch": best[2],
                      "register_cap": best[3]},
           "what": f"{num_grooms} grooms (strands log-uniform [500, 20000], 16-128 vertices) in one "
                   f"kami_vbd_batch_create handle, {nb} steps per kami_vbd_batch_step "
                   f"({'fixed' if tuning else 'autotuned'} tile shape, CUDA graph), against {num_grooms} handles "
                   "stepped one after another with kami_vbd_step: the plain drop-in (form auto = fused, each "
                   "handle autotuned) and the sweep form"}
    if per_groom_handles:
        vf, ms_f = per_groom("auto", 10)
        vp, ms_p = per_groom("sweep", 3)
        res.update({"plain_per_groom_fused_value": vf, "plain_fused_ms_per_step": ms_f,
                    "batched_over_plain_fused": vb / vf, "plain_per_groom_sweep_value": vp,
                    "plain_sweep_ms_per_step": ms_p, "batched_over_plain_sweep": vb / vp})
    return res


def extra_forms(args, torch, stream, flush):
    """Plain per-groom sweep form and strain limiting on the headline groom, batched vs plain per-groom
    handles on 64 uneven grooms, the adjoint, the SDF bake, hair-hair, long strands and the reference's
    default settings."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.vbd import Solver

    out = {}
    g = synth.groom()
    st = settings()
    s = Solver(g, form="sweep", **st)
    for _ in range(3):
        s.step(DT, stream=stream)
    n = max(20, args.steps // 20)
    ms = time_steps(s, n, stream, flush)
    out["plain_sweep"] = {"value": g.num_vertices * NUM_ITR * n / (ms / 1e3), "ms_per_step": ms / n,
                          "what": "same groom, the sweep form (the reference's sweep order: even and odd vertices, "
                                  "then even and odd segments per iteration, one launch per iteration over tiles "
                                  "in shared memory) replayed from a CUDA graph"}
    s.close()

    out["strain_limit"] = strain_limit_timing(torch, stream)

    out["batched_64_grooms"] = batched_timing(torch, stream, flush)
    out["adjoint_2k_x48"] = adjoint_timing(torch, stream)
    out["adjoint_fit"] = adjoint_fit(torch)
    out["sdf_bake_128"] = sdf_bake_timing()
    try:
        out["hair_hair_sweep"] = hair_hair_timing(torch, stream)
    except Exception as e:  # a contact-list overflow (KAMI_ERR_CONTACTS) is reported, not fatal
        out["hair_hair_sweep"] = {"error": str(e)}
    out["long_strands_3k_x200"] = long_strand_timing(torch, stream, flush)
    out["reference_default_settings"] = default_settings_timing(torch, stream)
    # the 80 M-vertex workload's kernels and body motion at a quarter of its size (bench.py --only large runs
    # all 8 instances)
    out["large_2x100k_x100"] = large_timing(torch, stream, frames=8, adjoint_frames=10, tape_gb=20.0, instances=2)
    return out


def trajectory_errors(frames=100, cut_strands=1000):
    """The FP32 GPU trajectory against an FP64 replay of the same update (the FP64 oracle, colour2
    schedule, same inputs) over `frames` frames, beside the FP32 oracle's: the cantilever of 64 rods
    x 32 vertices (10 iterations, dt 1/60 s, 1 substep) and a cut of the headline groom's generator
    (`cut_strands` x 64 vertices, 20 iterations, dt 1/120 s, the 128^3 head SDF).  Free-running: no
    state is shared after frame 0.  Positions in m (max over vertices), twists in rad (max over
    segments), each at the last frame and as the maximum over all frames."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.vbd import Solver
    from oracle.oracle import OracleSim, twist_angles

    cases = {
        "cantilever_64x32": (synth.cantilever(), dict(num_itr=10, max_h=1 / 60, gravity=(0.0, 0.0, -9.81),
                                                      radius=40e-6, density=1300.0, velocity_decay=0.05,
                                                      damping=1e-6), 1 / 60),
        f"groom_cut_{cut_strands}x64": (synth.groom(cut_strands, 64, seed=2), settings(), DT),
    }
    out = {}
    for name, (g, st, dt) in cases.items():
        o64 = OracleSim(g, dtype=np.float64, schedule="colour2", **st)
        o32 = OracleSim(g, dtype=np.float32, schedule="colour2", **st)
        free = OracleSim(g, dtype=np.float32, schedule="colour2", **dict(st, sdf=None)) if st.get("sdf") else None
        strand_of = np.repeat(np.arange(g.num_strands), np.diff(g.strand_begin))
        touched = np.zeros(g.num_strands, bool)
        s = Solver(g, form="auto", **st)
        worst = {"gpu_vs_fp64_m": 0.0, "gpu_vs_fp64_rad": 0.0, "gpu_vs_fp32_oracle_m": 0.0,
                 "gpu_vs_fp32_oracle_rad": 0.0, "fp32_oracle_vs_fp64_m": 0.0, "fp32_oracle_vs_fp64_rad": 0.0}
        last = {}
        for _ in range(frames):
            s.step(dt)
            o64.advance(dt)
            o32.advance(dt)
            if free is not None:  # strands the body touches: the FP32 oracle with and without it part
                free.advance(dt)
                d = np.zeros(g.num_strands)
                np.maximum.at(d, strand_of, np.abs(o32.x - free.x).max(1))
                touched |= d > 0
            x, _v = s.get_positions_velocities()
            q = s.get_orientations()
            last = {"gpu_vs_fp64_m": float(np.abs(x - o64.x).max()),
                    "gpu_vs_fp64_rad": float(np.abs(twist_angles(o64.q, q)).max()),
                    "gpu_vs_fp32_oracle_m": float(np.abs(x - o32.x).max()),
                    "gpu_vs_fp32_oracle_rad": float(np.abs(twist_angles(o32.q, q)).max()),
                    "fp32_oracle_vs_fp64_m": float(np.abs(o32.x - o64.x).max()),
                    "fp32_oracle_vs_fp64_rad": float(np.abs(twist_angles(o64.q, o32.q.astype(np.float64))).max())}
            worst = {k: max(worst[k], v) for k, v in last.items()}
        travel = float(np.abs(o64.x - g.positions).max())
        s.close()
        out[name] = {"frames": frames, "vertices": g.num_vertices, "num_itr": st["num_itr"], "dt": dt,
                     "last_frame": last, "max_over_frames": worst, "max_displacement_m": travel}
        if free is not None:
            e64 = np.zeros(g.num_strands)
            e32 = np.zeros(g.num_strands)
            np.maximum.at(e64, strand_of, np.abs(x - o64.x).max(1))
            np.maximum.at(e32, strand_of, np.abs(o32.x - o64.x).max(1))
            un = ~touched
            out[name]["strands_touched_by_the_body"] = int(touched.sum())
            out[name]["untouched_strands_last_frame"] = {
                "strands": int(un.sum()), "gpu_vs_fp64_m": float(e64[un].max()) if un.any() else None,
                "fp32_oracle_vs_fp64_m": float(e32[un].max()) if un.any() else None}
    out["what"] = ("FP32 GPU step (kami_vbd_step, colour2) against the FP64 oracle replay of the same update, "
                   "free-running over the frames, with the FP32 oracle's own FP64 gap beside it; on the groom, also "
                   "over the strands the head never touches (the body pass's branch and velocity fix make touched "
                   "strands depend on rounding)")
    return out


def default_settings_timing(torch, stream, frames=3):
    """The reference solver's default settings (scripts/json/StCossRods.json and the defaults of
    StableCosseratRodsSolver.h:86-110): strands resampled to 1 mm segments, NumItr 32, wind (peak 40,
    frequencies 1 / 0.7 / 0.4, sharpness 3), the head SDF, and YarnBall's Sim::maxH of 4e-4 s, so a
    1/60 s frame is 42 substeps.  6,000 strands of 100-300 vertices (10-30 cm); one kami_vbd_step per
    frame, autotuned tile shape, CUDA events around the frames."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.vbd import Solver

    rng = np.random.default_rng(12)
    g = synth.groom_strands(rng, rng.integers(100, 301, 6000), seg_len=1e-3)
    st = dict(num_itr=32, max_h=4e-4, gravity=(0.0, 0.0, -9.81), radius=40e-6, density=1300.0, velocity_decay=0.05,
              damping=1e-6, wind=(40.0, 1.0, 0.7, 0.4, 3.0), sdf=synth.sphere_sdf(128, threshold=1e-3))
    dt = 1.0 / 60.0
    s = Solver(g, form="auto", **st)
    tuned, _ = s.autotune(dt, trial_steps=2)
    s.step(dt, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(frames):
        s.step(dt, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / frames
    s.get_positions_velocities()  # raises if a frame went non-finite
    s.close()
    substeps = math.ceil(dt / 4e-4 - 1e-6)
    return {"value": g.num_vertices * 32 * substeps / (ms / 1e3), "unit": UNIT, "ms_per_frame": ms,
            "substeps_per_frame": substeps, "vertices": g.num_vertices,
            "tuning": dict(zip(("slots_per_lane", "warps_per_block", "steps_per_launch", "register_cap"), tuned)),
            "what": "6,000 strands of 100-300 vertices at 1 mm, NumItr 32, wind, head SDF, 42 substeps of 4e-4 s per "
                    "1/60 s frame: the reference solver's default settings"}


def long_strand_timing(torch, stream, flush, steps=200):
    """3,000 strands x 200 vertices (longer than a tile of 128 slots), the headline settings: the
    fused form in groups of 2 tiles (autotuned) against the sweep form, one step per call, L2
    flushed between timed steps."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.vbd import Solver

    g = synth.groom(3000, 200, seed=9)
    st = settings()
    res = {}
    for form in ("fused", "sweep"):
        s = Solver(g, form=form, **st)
        if form == "fused":
            res["tuning"] = dict(zip(("slots_per_lane", "warps_per_block", "steps_per_launch", "register_cap"),
                                     s.autotune(DT, trial_steps=8)[0]))
        for _ in range(3):
            s.step(DT, stream=stream)
        n = steps if form == "fused" else steps // 4
        ms = time_steps(s, n, stream, flush)
        res[form] = {"value": g.num_vertices * NUM_ITR * n / (ms / 1e3), "ms_per_step": ms / n}
        s.close()
    res["what"] = ("3,000 strands x 200 vertices, 20 iterations, dt 1/120 s, head-sphere SDF 128^3: fused form on groups "
                   "of tiles (a strand runs on across the warps of a CTA) vs the sweep form")
    return res


def sdf_bake_timing():
    """kami_sdf_bake of a 128^3 grid from a 20,480-triangle icosphere head (host arrays in and out,
    host-timed: pseudonormals, copies and the kernel), against the FP64 oracle on an 8^3 subset."""
    from kamisimulator_b200 import synth, vbd
    from oracle import oracle as orc

    import torch

    V, T = synth.icosphere(5, radius=0.09)
    lo, hi = (-0.15,) * 3, (0.15,) * 3
    vbd.bake_sdf(V, T, (16, 16, 16), lo, hi)  # warm-up (context, module)
    torch.cuda.synchronize()  # nothing of the legs before it runs inside the timed calls
    gpu_s = float("inf")
    for _ in range(3):  # best of three whole calls (host allocations and page faults vary between calls)
        t0 = time.perf_counter()
        vbd.bake_sdf(V, T, (128, 128, 128), lo, hi)
        gpu_s = min(gpu_s, time.perf_counter() - t0)
    t0 = time.perf_counter()
    orc.sdf_bake(V, T, (8, 8, 8), lo, hi)
    cpu_s = time.perf_counter() - t0
    pairs = 128 ** 3 * T.shape[0]
    return {"seconds": gpu_s, "node_triangle_tests_per_s": pairs / gpu_s,
            "cpu_oracle_node_triangle_tests_per_s": 8 ** 3 * T.shape[0] / cpu_s, "cpu_threads": orc.load().oracle_num_threads(),
            "what": "128^3 nodes x 20,480 triangles, exact signed distance + gradients, whole kami_sdf_bake call"}


def strain_limit_timing(torch, stream, calls=100):
    """The SDF solver's strain limiting (kami_vbd_strain_limit, StrainError 0.1) after each fused step of
    the headline groom: CUDA events around `calls` limits alone, then `calls` steps each followed by a
    limit (L2 not flushed)."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.vbd import Solver

    s = Solver(synth.groom(), form="fused", **settings())
    s.set_tuning(2, 4, 1, 120)
    for _ in range(3):
        s.step(DT, stream=stream)
        s.strain_limit(0.1, stream=stream)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    for _ in range(calls):
        s.strain_limit(0.1, stream=stream)
    e1.record(stream)
    for _ in range(calls):
        s.step(DT, stream=stream)
        s.strain_limit(0.1, stream=stream)
    e2.record(stream)
    torch.cuda.synchronize()
    s.close()
    return {"ms_per_call": e0.elapsed_time(e1) / calls, "step_and_limit_ms": e1.elapsed_time(e2) / calls,
            "what": "10,000 x 64 groom, StrainLimiting (StrainError 0.1) after each fused step, CUDA events over "
                    f"{calls} calls (L2 not flushed)"}


def hair_hair_timing(torch, stream, steps=50, h=4e-4):
    """The sweep form with hair-hair collision (detection every substep) on a 2,000 x 48 groom with
    its strands' roots on the head, at the reference's substep maxH = 4e-4 s (the velocity radius of
    the detection grows with the substep; at 1/120 s a dense groom exceeds 16 contacts per segment):
    vertex-iterations/s, CUDA events around kami_vbd_step."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.vbd import Solver

    g = synth.groom(2000, 48, seed=4)
    st = dict(settings(), radius=2e-6, max_h=h)
    s = Solver(g, form="sweep", hair_hair=True, barrier_thickness=7.6e-5, **st)
    free = Solver(g, form="sweep", **st)
    res = {}
    for name, solver in (("hair_hair", s), ("no_contacts", free)):
        for _ in range(10):
            solver.step(h, stream=stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            solver.step(h, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        res[name] = {"value": g.num_vertices * NUM_ITR * 1000.0 / ms, "ms_per_step": ms}
        solver.synchronize()
        solver.close()
    res["what"] = ("2,000 strands x 48 vertices, 20 iterations, substeps of 4e-4 s, head SDF; sweep form with and without "
                   "hair-hair collision (radius 2 um, barrier 76 um as the solver sets them at CurveRadius 40 um)")
    return res


def large_timing(torch, stream, frames=24, adjoint_frames=30, tape_gb=60.0, instances=8):
    """`instances` x 100,000 strands x 100 vertices (8 instances: 80 M vertices), union-of-12-capsules SDF on 256^3,
    head yawing +-30 deg at 1 Hz, 30 iterations, dt 1/120: kami_vbd_batch_step over `frames` frames with
    one body transform per frame (a sample of the 240-frame run).  Then the adjoint over the last
    `adjoint_frames` frames of the run (frames 210-239 of the head motion): a checkpointed rollout
    and its backward to d loss / d per-strand stiffness, the tape bounded to `tape_gb` by tile
    windows; host-timed (the backward is a host loop over windows and checkpoints)."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.vbd import Solver

    t0 = time.perf_counter()
    rng = np.random.default_rng(11)
    inst = [synth.groom_strands(rng, np.full(100_000, 100)) for _ in range(instances)]
    sdf = synth.capsule_union_sdf(256, num_capsules=12, radius_range=(0.02, 0.08))
    gen_s = time.perf_counter() - t0
    st = dict(num_itr=30, max_h=DT, gravity=(0.0, 0.0, -9.81), radius=40e-6, density=1300.0, velocity_decay=0.05,
              damping=1e-6, sdf=sdf)
    t0 = time.perf_counter()
    s = Solver(inst, form="fused", **st)  # kami_vbd_batch_create over the 8 instances
    create_s = time.perf_counter() - t0
    V = s.num_vertices
    counts = np.concatenate([np.diff(g.strand_begin) for g in inst])
    del inst
    best, _ = s.autotune(DT, trial_steps=4)
    bt = np.array([list(synth.head_rotation(f * DT)) + [0.0, 0.0, 0.0] for f in range(frames)], np.float32)
    s.batch_step(DT, frames, bt, stream=stream)  # warm-up, graph capture
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.batch_step(DT, frames, bt, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    s.synchronize()
    out = {"value": V * 30 * frames / (ms / 1e3), "ms_per_step": ms / frames, "vertices": V, "instances": instances,
           "frames_timed": frames,
           "tuning": dict(zip(("slots_per_lane", "warps_per_block", "steps_per_launch", "register_cap"), best)),
           "generate_s": gen_s, "create_s": create_s}
    out["adjoint"] = large_adjoint(torch, s, counts, adjoint_frames, tape_gb)
    s.close()
    return out


def large_adjoint(torch, s, counts, frames, tape_gb, k=10):
    from kamisimulator_b200 import synth
    from kamisimulator_b200.autograd import rollout_positions

    first = 240 - frames
    body = np.array([list(synth.head_rotation((first + f) * DT)) + [0.0, 0.0, 0.0] for f in range(frames)], np.float32)
    init = s.get_state_into(torch.empty(s.state_size() // 4, dtype=torch.float32, device="cuda"))
    unit = s.get_rest_darboux(torch.empty((s.num_vertices, 4), dtype=torch.float32, device="cuda"))
    strand_of = torch.repeat_interleave(torch.arange(len(counts), device="cuda"), torch.as_tensor(counts, device="cuda"))
    tiles = s.tile_count()
    slots_per_tile = 32 * s.get_tuning()[0]
    per_tile = k * ((30 + 1) * 32 + 48) * slots_per_tile  # tape bytes per tile for k recorded steps
    chunk = max(1, min(tiles, int(tape_gb * 1e9 // per_tile)))
    c = torch.randn((s.num_vertices, 3), device="cuda")
    scale = torch.ones(len(counts), device="cuda", requires_grad=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x = rollout_positions(scale, s, unit, strand_of, init, frames, DT, k, tiles_per_chunk=chunk, body_transforms=body)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    (c * x).sum().backward()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    finite = bool(torch.isfinite(scale.grad).all().item())
    return {"frames": frames, "checkpoint_every": k, "tiles": tiles, "tiles_per_window": chunk,
            "windows": -(-tiles // chunk), "tape_gb": chunk * per_tile / 1e9, "forward_s": t1 - t0,
            "backward_s": t2 - t1, "gradient_finite": finite,
            "what": f"d sum(c . x_239) / d per-strand stiffness over frames {first}-239, head motion replayed, every "
                    "segment recomputed window by window"}


def adjoint_fit(torch, iterations=150, frames=60, k=10, lr=0.1, lr_end=0.005):
    """Per-strand bend/twist stiffness fit on 2,000 strands x 48 vertices (20 iterations, dt 1/120 s,
    head-sphere SDF): the target is the rollout at the true stiffness after `frames` frames, the
    learnable scales start at truth x U[0.5, 2] (log-parameterised, Adam), the loss is the L2 distance
    of the positions after the rollout, with a checkpoint every `k` frames.  Reports the loss curve
    and how far the recovered scales are from 1 (the truth)."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.autograd import rollout_positions
    from kamisimulator_b200.vbd import Solver

    g = synth.groom(2000, 48, seed=4)
    solver = Solver(g, form="fused", **settings())
    unit = torch.tensor(solver.get_rest_darboux(), device="cuda")
    strand_of = torch.tensor(np.repeat(np.arange(g.num_strands), np.diff(g.strand_begin)), device="cuda")
    init = torch.tensor(solver.get_state(), device="cuda")
    with torch.no_grad():
        target = rollout_positions(torch.ones(g.num_strands, device="cuda"), solver, unit, strand_of, init, frames,
                                   DT, k)
    rng = np.random.default_rng(6)
    start = rng.uniform(0.5, 2.0, g.num_strands)
    logs = torch.tensor(np.log(start), dtype=torch.float32, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([logs], lr=lr)
    decay = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=(lr_end / lr) ** (1.0 / iterations))
    losses = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(iterations):
        opt.zero_grad()
        x = rollout_positions(torch.exp(logs), solver, unit, strand_of, init, frames, DT, k)
        loss = ((x - target) ** 2).sum()
        loss.backward()
        opt.step()
        decay.step()
        losses.append(loss.item())
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    err = np.abs(np.exp(logs.detach().cpu().numpy()) - 1.0)
    err0 = np.abs(start - 1.0)
    # strands whose final positions say something about their stiffness: doubling it moves them > 1 mm
    with torch.no_grad():
        x2 = rollout_positions(torch.full((g.num_strands,), 2.0, device="cuda"), solver, unit, strand_of, init,
                               frames, DT, k)
    moved = np.zeros(g.num_strands)
    np.maximum.at(moved, strand_of.cpu().numpy(), (x2 - target).norm(dim=1).cpu().numpy())
    ident = moved > 1e-3
    solver.close()
    return {"strands": g.num_strands, "verts_per_strand": 48, "frames": frames, "checkpoint_every": k,
            "adam_iterations": iterations, "lr": lr, "seconds_per_iteration": el / iterations,
            "loss_curve": [losses[i] for i in range(0, iterations, max(1, iterations // 12))] + [losses[-1]],
            "loss_first": losses[0], "loss_last": losses[-1],
            "scale_error_start": {"median": float(np.median(err0)), "p90": float(np.percentile(err0, 90))},
            "scale_error_end": {"median": float(np.median(err)), "p90": float(np.percentile(err, 90))},
            "identifiable_strands": int(ident.sum()),
            "identifiable_scale_error_start": {"median": float(np.median(err0[ident])) if ident.any() else None,
                                               "p90": float(np.percentile(err0[ident], 90)) if ident.any() else None},
            "identifiable_scale_error_end": {"median": float(np.median(err[ident])) if ident.any() else None,
                                             "p90": float(np.percentile(err[ident], 90)) if ident.any() else None},
            "what": "fit of per-strand stiffness scales (truth = 1) to the positions after a 60-frame rollout (Adam, "
                    "learning rate decayed exponentially); |scale - 1| over all strands and over the identifiable "
                    "ones (doubling their stiffness moves their final positions by more than 1 mm)"}


def adjoint_timing(torch, stream):
    """Device time per step of the forward step, the recorded forward and the adjoint (reverse) step
    on 2,000 strands x 48 vertices, plus one host-timed autograd round (60 steps, checkpoint 10)."""
    from kamisimulator_b200 import synth
    from kamisimulator_b200.autograd import rollout_positions
    from kamisimulator_b200.vbd import Solver

    g = synth.groom(2000, 48, seed=4)
    st = settings()
    solver = Solver(g, form="fused", **st)
    k = 10
    solver.tape_reserve(k, 0)
    init = solver.get_state()
    solver_tape_gb = solver.tape_bytes_per_substep() * 60 / 1e9

    def timed(fn):
        solver.set_state(init)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k

    gx = torch.randn((g.num_vertices, 3), device="cuda")
    zero3, zero4 = torch.zeros_like(gx), torch.zeros((g.num_vertices, 4), device="cuda")
    for _ in range(2):  # second pass is the measurement
        fwd = timed(lambda: [solver.step(DT, stream=stream) for _ in range(k)])
        rec = timed(lambda: [solver.step_record(DT, stream=stream) for _ in range(k)])
        args = (gx.clone(), zero3.clone(), zero3.clone(), zero4.clone())
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        solver.backward(*args)
        b.record(stream)
        torch.cuda.synchronize()
        adj = a.elapsed_time(b) / k
    unit = torch.tensor(solver.get_rest_darboux(), device="cuda")
    strand_of = torch.tensor(np.repeat(np.arange(g.num_strands), np.diff(g.strand_begin)), device="cuda")
    init_d = torch.tensor(init, device="cuda")
    frames = 60

    def autograd_round(budget):
        """Host time of the forward rollout and of its backward pass (60 frames, checkpoint every 10)."""
        scale = torch.ones(g.num_strands, device="cuda", requires_grad=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x = rollout_positions(scale, solver, unit, strand_of, init_d, frames, DT, k, tape_budget_bytes=budget)
        loss = (x ** 2).sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        return t1 - t0, time.perf_counter() - t1

    autograd_round(0)  # warm-up
    f_plain, b_recompute = autograd_round(0)
    autograd_round(None)
    f_tape, b_tape = autograd_round(None)
    solver.close()
    return {"forward_ms_per_step": fwd, "recorded_forward_ms_per_step": rec, "adjoint_ms_per_step": adj,
            "adjoint_over_forward": adj / fwd, "recorded_forward_over_forward": rec / fwd,
            "backward_with_recompute_over_forward": (rec + adj) / fwd,
            "autograd": {"frames": frames, "checkpoint_every": k,
                         "recompute_every_segment": {"forward_s": f_plain, "backward_s": b_recompute,
                                                     "backward_over_forward": b_recompute / f_plain},
                         "tape_recorded_in_forward": {"forward_s": f_tape, "backward_s": b_tape,
                                                      "backward_over_forward": b_tape / f_plain,
                                                      "forward_over_plain_forward": f_tape / f_plain,
                                                      "tape_gb": solver_tape_gb}},
            "what": "2,000 strands x 48 vertices, 20 iterations, dt 1/120, sphere SDF; device time per step of "
                    "kami_vbd_step, kami_vbd_step_record and kami_vbd_backward (10 recorded steps); autograd: host "
                    "time of a 60-frame rollout and of its backward pass, every segment recomputed from its "
                    "checkpoint (tape budget 0) or every segment recorded during the forward pass (default budget)"}


def run_ours(args):
    import torch

    world, rank, local = dist_setup()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    from kamisimulator_b200 import synth, vbd
    from kamisimulator_b200.vbd import Solver

    g = rank_groom(rank)
    st = settings()
    V = g.num_vertices
    solver = Solver(g, form="fused", device=local, **st)  # this rank's GPU (LOCAL_RANK)
    if args.tuning:  # a fixed tile shape (profiling runs: no autotune launches before the timed ones)
        solver.set_tuning(*[int(t) for t in args.tuning.split(",")])
        tuned = solver.get_tuning()
    else:
        tuned, _ = solver.autotune(DT, trial_steps=8)  # the library's autotuner; restores the state
    launch_mode = solver.get_launch_mode()  # 0: hardware-scheduled tile grid, 1: persistent
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        solver.step(DT, stream=stream)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    gpus = list(range(world)) if world > 1 else [local]
    with ClockSampler(gpus) as clk:
        barrier()
        step_ms = time_steps(solver, args.steps, stream, flush)
        barrier()
    max_ms = max_over_ranks(step_ms, world)
    value = job_throughput(world, V, NUM_ITR, args.steps, max_ms)
    ms_step = max_ms / args.steps

    # end to end through the C ABI with pinned host buffers: one kami_vbd_step_host call per frame
    # (one kernel reads the host arrays, steps the tiles and writes the host arrays back), and for
    # comparison the same frame as three calls (kami_vbd_set_positions_velocities, kami_vbd_step,
    # kami_vbd_get_positions_velocities)
    xh = torch.empty((V, 3), dtype=torch.float32, pin_memory=True)
    vh = torch.empty((V, 3), dtype=torch.float32, pin_memory=True)
    solver.get_positions_velocities(xh.numpy(), vh.numpy())
    e2e_steps = max(10, args.steps // 10)

    def e2e_run(frame):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            frame()
        e1.record(stream)
        torch.cuda.synchronize()
        return job_throughput(world, V, NUM_ITR, e2e_steps, max_over_ranks(e0.elapsed_time(e1), world))

    def three_calls():
        solver.set_positions_velocities(xh.numpy(), vh.numpy())
        solver.step(DT, stream=stream)
        solver.get_positions_velocities(xh.numpy(), vh.numpy())

    # the plugin's frame: its Hair (padded [strand][vertex] arrays, page-locked at Construct) uploaded,
    # stepped and downloaded by one kami_vbd_step_hair call (UploadHair, SolveNextStep, DownloadHair)
    solver.set_hair_layout(g.num_strands, 64)
    hx = torch.empty((g.num_strands, 64, 3), dtype=torch.float32, pin_memory=True)
    hv = torch.empty((g.num_strands, 64, 3), dtype=torch.float32, pin_memory=True)
    solver.download_hair(hx, hv)
    for _ in range(3):
        solver.step_hair(DT, hx, hv, hx, hv)
        solver.step_host(DT, xh, vh)
    e2e_value = e2e_run(lambda: solver.step_hair(DT, hx, hv, hx, hv))
    e2e_packed = e2e_run(lambda: solver.step_host(DT, xh, vh))
    e2e_three_calls = e2e_run(three_calls)
    solver.close()

    line = None
    if rank == 0:
        peak, peak_kind = hbm_peak()
        achieved = V * BYTES_PER_VERTEX_STEP / (ms_step / 1e3) / 1e9
        traffic, prof = ncu_traffic()
        prof = prof or {}
        per_gpu = value / world
        kernel_flop = prof.get("fp32_flop_per_vertex_iter")
        fp32_peak, fp32_source = FP32_PEAK_TFLOPS, "nominal FP32 (148 SMs x 128 FMA lanes x 2 x 1965 MHz)"
        probe = None
        try:
            probe = fp32_probe(0)  # after the timed region: FFMA and FFMA2 chains on this GPU
        except Exception as exc:  # the nominal figure stands in, and the line says so
            fp32_source += f" (probe failed: {exc})"
        if probe and max(probe) > 0:
            fp32_peak = max(probe)
            fp32_source = (f"measured: kami_fp32_peak FMA chains, {probe[0]:.1f} TFLOP/s FFMA and {probe[1]:.1f} "
                           f"TFLOP/s packed FFMA2 (the larger is the peak); nominal {FP32_PEAK_TFLOPS:.1f}")
        fp32 = {"bound": "fp32 issue", "unit": "TFLOP/s", "peak": fp32_peak, "peak_source": fp32_source,
                "reference_flop_per_vertex_iter": REFERENCE_FLOP_PER_VERTEX_ITER,
                "reference_equivalent": per_gpu * REFERENCE_FLOP_PER_VERTEX_ITER / 1e12,
                "kernel_flop_per_vertex_iter": kernel_flop,
                "achieved": per_gpu * kernel_flop / 1e12 if kernel_flop else None,
                "issue_active": prof.get("issue_active_pct", 0) / 100 or None,
                "source": "kernel FLOPs (2 FFMA + FMUL + FADD per thread) and issue-slot use from the committed ncu capture"}
        fp32["frac"] = fp32["achieved"] / fp32_peak if fp32["achieved"] else None
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_dict({"form": "fused", "per_gpu": "one 10,000 x 64 groom per GPU",
                                       "tuning": dict(zip(("slots_per_lane", "warps_per_block", "steps_per_launch",
                                                           "register_cap"), tuned)),
                                       "launch_mode": launch_mode}),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "kernel": "fused_step_kernel (colour2, one step per launch)",
                             "bytes_per_launch": V * BYTES_PER_VERTEX_STEP, "peak_source": peak_kind},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 24 * V, "d2h_bytes_per_step": 24 * V,
                        "steps": e2e_steps,
                        "call": "kami_vbd_step_hair on the plugin's page-locked padded Hair arrays (UploadHair + "
                                "SolveNextStep + DownloadHair in one launch, the plugin's frame path)",
                        "packed_step_host_value": e2e_packed, "three_calls_value": e2e_three_calls},
                "fp32": fp32, "gpu_launches": args.steps, "clocks": clk.summary()}
    if world == 1 and rank == 0 and not args.skip_extra:
        line["forms"] = extra_forms(args, torch, stream, flush)
        line["trajectory"] = trajectory_errors()
        line["cpu_baseline"] = cpu_baseline_sample()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-extra", action="store_true", help="only the headline timing (profiling runs)")
    ap.add_argument("--only", choices=["adjoint", "fit", "large", "hairhair", "bake", "long", "default", "trajectory",
                                       "strain", "batched"],
                    help="run a single extra measurement")
    ap.add_argument("--grooms", type=int, default=64,
                    help="--only batched: the number of grooms (a smaller batch of the same generator for profiling "
                         "runs skips the per-groom handles)")
    ap.add_argument("--tuning", help="fixed tile shape C,warps,steps_per_launch,register_cap instead of autotuning")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.only == "adjoint":
        import torch

        print(json.dumps(adjoint_timing(torch, torch.cuda.current_stream())), flush=True)
    elif args.only == "large":
        import torch

        print(json.dumps(large_timing(torch, torch.cuda.current_stream())), flush=True)
    elif args.only == "batched":
        import torch

        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        tuning = [int(t) for t in args.tuning.split(",")] if args.tuning else None
        print(json.dumps(batched_timing(torch, torch.cuda.current_stream(), flush, args.grooms,
                                        per_groom_handles=args.grooms == 64, tuning=tuning)), flush=True)
    elif args.only == "strain":
        import torch

        print(json.dumps(strain_limit_timing(torch, torch.cuda.current_stream())), flush=True)
    elif args.only == "hairhair":
        import torch

        print(json.dumps(hair_hair_timing(torch, torch.cuda.current_stream())), flush=True)
    elif args.only == "bake":
        print(json.dumps(sdf_bake_timing()), flush=True)
    elif args.only == "fit":
        import torch

        print(json.dumps(adjoint_fit(torch)), flush=True)
    elif args.only == "trajectory":
        print(json.dumps(trajectory_errors()), flush=True)
    elif args.only == "default":
        import torch

        print(json.dumps(default_settings_timing(torch, torch.cuda.current_stream())), flush=True)
    elif args.only == "long":
        import torch

        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        print(json.dumps(long_strand_timing(torch, torch.cuda.current_stream(), flush)), flush=True)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
