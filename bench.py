#!/usr/bin/env python3
"""Benchmark: bundle-adjustment time-to-converge and LM iterations/s on one B200 (or N replicas).

Workload (default): the 12M-observation global refinement: 3,000 cameras with per-camera
intrinsics (6-DoF pose + log f, k1, k2 per camera, D = 26,993) over a 245 x 245 ground plane, 2M
points with geometric track lengths (mean ~6, minimum 2; ~12.0M observations), pixel noise
N(0, 0.5^2), 5% outliers, Huber loss (1 px), matrix-free block-Jacobi PCG with forcing tolerance
1e-6, run to convergence (LM budget 200). Seeded synthetic data (no dataset exists for it). One
step = one complete solve of that problem. A second leg in the same line solves the 500-camera,
1.2M-observation problem to convergence in both precisions.

value  : LM iterations/s of the mixed-precision solve (FP32 Jacobians and products, FP64 everything
         the reference's acceptance depends on), problem resident in device memory
         (omvgba_plan_solve), summed over replicas, divided by the slowest rank's time.
e2e    : the same through omvgba_solve from host arrays (lowering, upload and download included).
fp64   : the plain FP64 solve of the same problem, for the mixed-vs-FP64 comparison at equal cost.
targets: whether the mixed solve is >= 2x the FP64 solve's speed, whether both converged, and whether
         their final costs agree to 1e-6 relative.
roofline: the matrix-free product's tile kernel (k_mv_tiles<float>, the dominant kernel of the
         PCG loop), timed alone with CUDA events on the plan's stream with L2 flushed before each launch.
cpu_baseline: the C++ restatement of the reference CPU solver (the oracle) on the first LM
         iteration of the same problem, all host threads; a single-thread sample on the
         500-camera problem beside it.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 launch under torch.distributed.run; every rank solves its own seeded replica.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "openmvg-rs_b200"))

METRIC = "BA time-to-converge (s) & LM iters/s, mixed vs FP64 GPU, same final cost"
UNIT = "LM iterations/s"
L2_BYTES = 126 * 1024 * 1024
FLUSH_BYTES = 512 * 1024 * 1024
# Workloads: plane3000 is the headline (the 12M-observation global refinement the mixed-precision
# target is stated on); plane500 is the single large 500-camera problem, also run as the second leg
# of the headline line.
WORKLOADS = {
    "plane500": dict(
        kwargs=dict(cameras=500, points=200_000, mean_track=6.5, extent=100.0),
        text=("plane500: 500 cameras with per-camera (f, k1, k2) over a 100x100 ground plane, 200k points, "
              "geometric tracks mean ~6 (1,184,956 observations at seed 11), noise 0.5 px, 5% outliers, "
              "Huber 1 px, block-Jacobi PCG tolerance 1e-6")),
    "plane3000": dict(
        kwargs=dict(cameras=3000, points=2_000_000, mean_track=6.5, extent=245.0),
        text=("plane3000: 3,000 cameras with per-camera (f, k1, k2) over a 245x245 ground plane (the plane500 "
              "camera density), 2M points, geometric tracks mean ~6 (~12M observations), noise 0.5 px, 5% "
              "outliers, Huber 1 px, matrix-free block-Jacobi PCG tolerance 1e-6")),
    "windows256": dict(
        kwargs=dict(),
        text=("windows256: 256 independent local-BA windows (5-40 calibrated cameras, 500-5,290 points, tracks "
              "2-10, 1,408,836 observations at seed 23), Huber 1 px, dense Cholesky steps per window, solved "
              "in one batched call")),
    "residual10m": dict(
        kwargs=dict(),
        text=("residual10m: radial-camera reprojection residual and its hand-written VJP over 10M observations "
              "(3,000 cameras from random rotations and translations in the unit box, 2M points at depths 2-50, "
              "FP32), forward + backward through the torch.autograd.Function")),
}
CPU_SAMPLE_ITERATIONS = {"plane500": 3, "plane3000": 1}
CPU_SAMPLE_WINDOWS = 32
DEFAULT_WORKLOAD = "plane3000"
SECOND_LEG = "plane500"
MAX_ITERATIONS = 200  # LM budget: every bench solve converges well inside it
TRAFFIC_SUMMARY = {"plane500": os.path.join(ROOT, "profiles", "k_mv_tiles_fp32_plane500.txt"),
                   "plane3000": os.path.join(ROOT, "profiles", "k_mv_tiles_fp32_plane3000.txt")}


def problem_for(rank: int, workload: str = DEFAULT_WORKLOAD):
    from openmvg_ba_cuda import synthetic
    return synthetic.plane_problem(seed=11 + rank, **WORKLOADS[workload]["kwargs"])


def sfm_refresh_leg(problem, steps: int, sample: int = 3000) -> dict:
    """The landmark reprojection-error refresh openmvg-sfm runs after a solve, over the workload's
    landmarks (every observation supporting, every view posed): end to end from host arrays through
    omvgba_sfm_refresh_reprojection (upload, kernel, download), against the oracle's restatement on
    the first `sample` landmarks on one host thread."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sfm_oracle  # the CPU baseline's restatement only
    from openmvg_ba_cuda.adjuster import CudaBundleAdjuster
    from openmvg_ba_cuda.sfm import LandmarkTracks, refresh_reprojection
    P = len(problem.points)
    order = np.argsort(problem.observation_point, kind="stable")
    offset = np.concatenate([[0], np.cumsum(np.bincount(problem.observation_point, minlength=P))]).astype(np.uint64)
    tracks = LandmarkTracks(points=problem.points, active=np.ones(P, np.uint8), track_offset=offset,
                            track_pose=problem.observation_pose[order].astype(np.uint32),
                            track_intrinsic=problem.observation_intrinsic[order].astype(np.uint32),
                            track_pixel=np.ascontiguousarray(problem.observation_pixel[order]),
                            track_support=np.ones(len(order), np.uint8))
    with CudaBundleAdjuster(0) as ba:
        refresh_reprojection(ba, problem.rotations, problem.centers, problem.intrinsics, tracks)  # warm-up
        t0 = time.perf_counter()
        for _ in range(steps):
            out = refresh_reprojection(ba, problem.rotations, problem.centers, problem.intrinsics, tracks)
        gpu_s = (time.perf_counter() - t0) / steps
    n = min(sample, P)
    sub = LandmarkTracks(points=tracks.points[:n], active=tracks.active[:n], track_offset=offset[:n + 1],
                         track_pose=tracks.track_pose, track_intrinsic=tracks.track_intrinsic,
                         track_pixel=tracks.track_pixel, track_support=tracks.track_support)
    t0 = time.perf_counter()
    sfm_oracle.refresh(problem.rotations, problem.centers, problem.intrinsics, sub, np.zeros(n))
    cpu_s = time.perf_counter() - t0
    obs = int(offset[-1])
    return {"kernel": "k_sfm_refresh", "landmarks": P, "observations": obs,
            "e2e_seconds": gpu_s, "e2e_observations_per_s": obs / gpu_s,
            "rejected_landmarks": out.rejected_landmarks, "removed_observations": out.removed_observations,
            "cpu_oracle_observations_per_s": int(offset[n]) / cpu_s, "cpu_sample": f"first {n} landmarks, 1 thread, pure Python"}


def solve_config(precision: int, max_iterations: int = 50, stream: int = 0):
    from openmvg_ba_cuda import SolveConfig, abi
    return SolveConfig(linear_solver=abi.SOLVER_ITERATIVE, precision=precision, pcg_relative_tolerance=1e-6,
                       max_iterations=max_iterations, stream=stream)


# ---- distributed plumbing (replicas: no data-path collective) -----------------------------------
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def aggregate(seconds: float, units: float, device=None) -> tuple[float, float]:
    """(max seconds over ranks, sum of units over ranks); identity without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return seconds, units
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


# ---- clocks sampled during the timed region -----------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        # the raw samples go to OMVGBA_CLOCKS_DIR (default: the temporary directory); the JSON line
        # carries their summary
        clock_dir = os.environ.get("OMVGBA_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(clock_dir, f"clocks_rank{device_index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device_index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": "nvidia-smi unavailable"}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        return summarize_clocks(open(self.path).read())


def summarize_clocks(text: str) -> dict:
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    sm, mx, power, reasons = [], [], [], set()
    for line in text.splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx.append(float(f[2]))
            power.append(float(f[3]))
        except ValueError:
            continue
        for name, val in zip(names, f[5:9]):
            if val.lower().startswith("active"):
                reasons.add(name)
    if not sm:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
            "samples": len(sm), "power_w_max": max(power)}


def measured_peak() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "of measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "of fallback"


def traffic_per_launch(observations: int, workload: str):
    """DRAM bytes per launch of k_mv_tiles<float> from the committed ncu summary of this workload
    (else the plane500 one), scaled to this problem's observation count when the capture ran on
    another size."""
    path = TRAFFIC_SUMMARY.get(workload)
    if not path or not os.path.exists(path):
        path = TRAFFIC_SUMMARY["plane500"]
    try:
        fields = {}
        for line in open(path):
            if ":" in line:
                k, v = line.split(":", 1)
                fields[k.strip()] = v.strip()
        per_launch = float(fields["dram_bytes_per_launch"])
        captured = float(fields["observations"])
        return per_launch * observations / captured
    except (OSError, KeyError, ValueError):
        return None


# ---- CPU baseline: the oracle (C++ restatement of the reference CPU solver) ----------------------
def cpu_sample(problem, iterations: int, threads: int | None = None) -> dict:
    """The oracle on the first `iterations` LM iterations of `problem`: value = iterations / the wall
    time of those iterations (the LM loop; set-up and the final certificate, which runs once after
    the loop, are left out of the rate and reported as whole-call seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from openmvg_ba_cuda import abi
    threads = threads or oracle.max_threads()
    oracle.set_threads(threads)
    oracle.set_certificate(False)
    try:
        cfg = solve_config(abi.PRECISION_FP64, max_iterations=iterations)
        t0 = time.perf_counter()
        sol = oracle.solve(problem, cfg)
        dt = time.perf_counter() - t0
        per = oracle.iteration_seconds()
    finally:
        oracle.set_certificate(True)
    its = len(per)
    loop = sum(per)
    return {"value": its / loop, "unit": UNIT, "cores": threads, "kind": "port", "seconds": loop, "iterations": its,
            "call_seconds": dt, "pcg_iterations": int(sol.report.get("pcg_iteration_count", 0)),
            "sample": (f"oracle (C++/OpenMP restatement of the reference CPU solver): the first {its} LM "
                       f"iteration(s) of the same problem on {threads} thread(s), timed per iteration inside the "
                       f"LM loop ({dt:.1f} s for the whole call with lowering); early iterations need fewer PCG "
                       "iterations than the average of a solve run to convergence, so this rate favours the CPU")}


def cpu_info() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args) -> int:
    """The reference arm: the oracle on this workload's problem, all host threads. Each step is one
    LM iteration of the oracle's loop (per-iteration wall time); the first `warmup` iterations are
    dropped. Iterations come from one solve with a budget of warmup + steps (more solves from the
    start if it converges first)."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from openmvg_ba_cuda import abi
    problem = problem_for(0, args.workload)
    threads = oracle.max_threads()
    oracle.set_threads(threads)
    oracle.set_certificate(False)
    times, calls = [], 0
    try:
        while len(times) < args.warmup + args.steps and calls < 8:
            cfg = solve_config(abi.PRECISION_FP64, max_iterations=args.warmup + args.steps - len(times))
            oracle.solve(problem, cfg)
            times += oracle.iteration_seconds()
            calls += 1
    finally:
        oracle.set_certificate(True)
    timed = times[args.warmup:args.warmup + args.steps]
    total_s = sum(timed)
    value = len(timed) / total_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(timed), "warmup": args.warmup, "ms_per_step": 1e3 * total_s / len(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload]["text"], "max_iterations": args.max_iterations,
                   "parallelism": "host threads", "cpu": cpu_info(), "step": "one LM iteration of the oracle's loop",
                   "oracle_solves": calls},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": (f"oracle (C++/OpenMP restatement of the reference CPU solver) on this problem, "
                                    f"{threads} threads: LM iterations {args.warmup + 1}-{args.warmup + len(timed)} "
                                    "timed one by one inside the LM loop")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---- our arm ---------------------------------------------------------------------------------
def timed_solves(solve, stream, flush, steps: int):
    """Run `steps` solves, each timed by CUDA events on `stream` after an L2 flush."""
    import torch
    reports, ms = [], []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sol = solve()
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        reports.append(sol.report)
    return reports, ms, sol


def kernel_roofline(plan, info: dict, stream, flush, workload: str, launches: int = 20) -> dict:
    """Average duration of the tile kernel k_mv_tiles<float> alone (CUDA events on the plan's
    stream, L2 flushed before every launch) and its algorithmic bytes per launch: the FP32 Jacobian
    entries, one camera index per observation, the FP64 damped point inverse (6 values) per point
    and the camera vector x read once."""
    import torch
    D = int(info["reduced_dimension"])
    x = torch.randn(D, dtype=torch.float64, device="cuda")
    y = torch.empty(D, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    plan.schur_product(x.data_ptr(), y.data_ptr(), 0.1, fp32=True, stage=0)  # linearize once
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(launches):
        with torch.cuda.stream(stream):
            flush.fill_(2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.schur_product(x.data_ptr(), y.data_ptr(), 0.1, fp32=True, stage=1)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    avg_s = total / launches / 1e3
    algorithmic = (4 * int(info["jacobian_entries"]) + 4 * int(info["observation_count"])
                   + 48 * int(info["point_count"]) + 8 * D)
    peak, which = measured_peak()
    achieved = algorithmic / avg_s / 1e9
    traffic = traffic_per_launch(int(info["observation_count"]), workload)
    return {"bound": "hbm", "kernel": "k_mv_tiles<float>", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": which, "traffic": traffic,
            "algorithmic_bytes_per_launch": algorithmic, "avg_launch_us": avg_s * 1e6, "launches_timed": launches}


def stage_timing(plan, info: dict, stream, flush, stage: int, kernel: str, launches: int = 20) -> dict:
    """Average duration of one product stage of the plan by itself (CUDA events on the plan's stream,
    L2 flushed before each launch): stage 2 is k_block_rows, the block-row build of the explicit
    reduced camera system; stage 3 the camera-side assembly sums, k_block_tiles then k_block_records."""
    import torch
    D = int(info["reduced_dimension"])
    x = torch.zeros(D, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(launches):
        with torch.cuda.stream(stream):
            flush.fill_(3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.schur_product(x.data_ptr(), x.data_ptr(), 0.1, fp32=True, stage=stage)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    avg_us = total / launches * 1e3
    out = {"kernel": kernel, "avg_launch_us": avg_us, "launches_timed": launches}
    if stage == 3:  # the FP32 records each observation's sums read, per second
        out["observations_per_s"] = int(info["observation_count"]) / (avg_us * 1e-6)
    return out


def run_batched(args) -> int:
    """windows256: LM iterations/s summed over the windows of one omvgba_solve_batched call, timed
    on the host clock around the synchronous call (its workers run on their own streams), with the
    problems in host memory (so value and e2e are the same measurement)."""
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from openmvg_ba_cuda import RobustLoss, SolveConfig, synthetic
    from openmvg_ba_cuda.adjuster import CudaBundleAdjuster
    problems = [dataclasses_replace_loss(p, RobustLoss.huber(1.0)) for p in synthetic.window_problems(seed=23 + rank)]
    cfg = SolveConfig(max_iterations=args.max_iterations)
    adjuster = CudaBundleAdjuster(local)
    for _ in range(args.warmup):
        adjuster.solve_batched(problems, cfg)
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    total_s, its, launches, conv = 0.0, 0, 0, 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sols = adjuster.solve_batched(problems, cfg)
        torch.cuda.synchronize()
        total_s += time.perf_counter() - t0
        its += sum(s.report["iteration_count"] for s in sols)
        launches += sum(s.report["kernel_launches"] for s in sols)
        conv = sum(1 for s in sols if s.report["status"] == 0)
    clock_summary = clocks.stop()
    barrier()
    s_max, its_all = aggregate(total_s, float(its), device="cuda")
    cpu = None
    if rank == 0 and world == 1 and args.legs == "all":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        oracle.set_threads(oracle.max_threads())
        sample = problems[:CPU_SAMPLE_WINDOWS]
        t0 = time.perf_counter()
        cits = sum(oracle.solve(p, cfg).report["iteration_count"] for p in sample)
        dt = time.perf_counter() - t0
        cpu = {"value": cits / dt, "unit": UNIT, "cores": oracle.max_threads(), "kind": "port", "cpu": cpu_info(),
               "sample": f"oracle on the first {len(sample)} windows, one after another, all host threads"}
    adjuster.close()
    if rank == 0:
        value = its_all / s_max
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * s_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS["windows256"]["text"], "max_iterations": args.max_iterations,
                       "windows": len(problems), "observations": int(sum(p.observation_count for p in problems)),
                       "parallelism": f"replicas x{world}", "timing": "host clock around the batched call"},
            "windows_per_s": len(problems) * args.steps * world / s_max,
            "windows_converged": conv, "clocks": clock_summary,
            "e2e": {"value": value, "unit": UNIT, "note": "the batched call takes host arrays: same as value"},
            "gpu_launches": int(launches), "roofline": None, "cpu_baseline": cpu}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_residual(args) -> int:
    """residual10m: observations/s of one forward and one backward pass (loss = sum of residuals
    times a fixed upstream gradient) through ReprojectionResidual, inputs resident on the device,
    CUDA events on the current stream; L2 flushed before every step."""
    import numpy as np
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    from openmvg_ba_cuda import synthetic
    from openmvg_ba_cuda.autograd import reprojection_residual
    d = synthetic.residual_inputs(seed=5 + rank, dtype=np.float32)
    dev = "cuda"
    cam = torch.as_tensor(d["camera_index"].astype(np.int32), device=dev)
    pt = torch.as_tensor(d["point_index"].astype(np.int32), device=dev)
    px = torch.as_tensor(d["pixel"], device=dev)
    leaves = [torch.as_tensor(d[k], device=dev).requires_grad_(True) for k in ("rotvec", "translation", "intrinsics",
                                                                            "points")]
    n = cam.shape[0]
    g = torch.randn(n, 2, device=dev, generator=torch.Generator(dev).manual_seed(7))
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def step():
        for leaf in leaves:
            leaf.grad = None
        res = reprojection_residual(cam, pt, px, *leaves)
        torch.autograd.backward(res, g)
        return res

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    fwd_ms, tot_ms = 0.0, 0.0
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        for leaf in leaves:
            leaf.grad = None
        e0.record()
        res = reprojection_residual(cam, pt, px, *leaves)
        e1.record()
        torch.autograd.backward(res, g)
        e2.record()
        e2.synchronize()
        fwd_ms += e0.elapsed_time(e1)
        tot_ms += e0.elapsed_time(e2)
    if rank == 0:
        value = n * args.steps / (tot_ms / 1e3)
        fwd_bytes = n * (4 + 4 + 8 + 8) + 12 * leaves[3].shape[0] + 36 * leaves[0].shape[0]
        print(json.dumps({
            "metric": "reprojection residual forward + VJP throughput", "value": value, "unit": "observations/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOADS["residual10m"]["text"], "observations": int(n),
                       "l2": "L2 flushed (512 MB write) before every step; inputs 360 MB"},
            "forward_ms": fwd_ms / args.steps, "backward_ms": (tot_ms - fwd_ms) / args.steps,
            "forward_roofline": {"bound": "hbm", "algorithmic_bytes": fwd_bytes,
                                 "achieved": fwd_bytes / (fwd_ms / args.steps / 1e3) / 1e9, "unit": "GB/s",
                                 "peak": measured_peak()[0]},
        }), flush=True)
    return 0


def dataclasses_replace_loss(problem, loss):
    import dataclasses
    return dataclasses.replace(problem, robust_loss=loss)


def precision_pair(adjuster, problem, stream, flush, steps: int, warmup: int, max_iterations: int) -> dict:
    """Resident mixed-precision and FP64 solves of one problem, `steps` timed solves each (CUDA
    events on the solver's stream, L2 flushed before each), after `warmup` untimed ones."""
    import torch
    from openmvg_ba_cuda import abi
    out = {}
    for name, precision in (("mixed", abi.PRECISION_MIXED), ("fp64", abi.PRECISION_FP64)):
        plan = adjuster.plan(problem, solve_config(precision, max_iterations=max_iterations,
                                                   stream=stream.cuda_stream))
        for _ in range(warmup):
            plan.solve()
        torch.cuda.synchronize()
        barrier()
        reports, ms, _ = timed_solves(plan.solve, stream, flush, steps)
        barrier()
        info = plan.info()
        plan.close()
        seconds, its = aggregate(sum(ms) / 1e3, float(sum(r["iteration_count"] for r in reports)), device="cuda")
        out[name] = {"reports": reports, "seconds": seconds, "iterations": its, "info": info,
                     "local_iterations": sum(r["iteration_count"] for r in reports)}
    return out


def leg_summary(pair: dict, steps: int) -> dict:
    """Time-to-converge, rates, final costs and the target checks of a mixed/FP64 pair."""
    m, f = pair["mixed"], pair["fp64"]
    rm, rf = m["reports"][-1], f["reports"][-1]
    t_m, t_f = m["seconds"] / steps, f["seconds"] / steps
    conv_m, conv_f = rm["status"] == 0, rf["status"] == 0
    gap = abs(rm["final_objective"] - rf["final_objective"]) / abs(rf["final_objective"])
    speedup = t_f / t_m
    return {
        "mixed": {"value": m["iterations"] / m["seconds"], "unit": UNIT, "converged": conv_m,
                  "time_to_converge_s": t_m if conv_m else None, "seconds_per_solve": t_m,
                  "lm_iterations": rm["iteration_count"], "pcg_iterations": rm["pcg_iteration_count"],
                  "final_cost": rm["final_objective"]},
        "fp64": {"value": f["iterations"] / f["seconds"], "unit": UNIT, "converged": conv_f,
                 "time_to_converge_s": t_f if conv_f else None, "seconds_per_solve": t_f,
                 "lm_iterations": rf["iteration_count"], "pcg_iterations": rf["pcg_iteration_count"],
                 "final_cost": rf["final_objective"]},
        "mixed_vs_fp64": {"speedup": speedup, "final_cost_rel_diff": gap},
        "targets": {"both_converged": conv_m and conv_f, "speedup_ge_2x": speedup >= 2.0,
                    "final_cost_rel_diff_le_1e-6": gap <= 1e-6},
    }


def run_ours(args) -> int:
    import torch
    world, rank, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the solver has no CPU path)")
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    from openmvg_ba_cuda import abi
    from openmvg_ba_cuda.adjuster import CudaBundleAdjuster

    problem = problem_for(rank, args.workload)
    stream = torch.cuda.Stream(device=local)  # the solver's stream: events and flushes go here too
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    adjuster = CudaBundleAdjuster(local)
    mixed_cfg = solve_config(abi.PRECISION_MIXED, max_iterations=args.max_iterations, stream=stream.cuda_stream)

    if args.legs == "sfm":  # the SfM-side refresh around the solve, on the workload's landmarks
        adjuster.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "legs": "sfm", "workload": args.workload,
                              "sfm_refresh": sfm_refresh_leg(problem, max(args.steps, 3))}), flush=True)
        return 0
    # value: mixed precision, problem resident in device memory
    plan = adjuster.plan(problem, mixed_cfg)
    info = plan.info()
    if args.legs == "kernel":  # the kernels' timings alone, no solve (for a small ncu capture)
        roofline = kernel_roofline(plan, info, stream, flush, args.workload, launches=max(args.steps, 3))
        rows = stage_timing(plan, info, stream, flush, 2, "k_block_rows", launches=max(args.steps, 3))
        sums = stage_timing(plan, info, stream, flush, 3, "k_block_tiles + k_block_records",
                            launches=max(args.steps, 3))
        plan.close()
        adjuster.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "legs": "kernel", "n_gpus": world, "roofline": roofline,
                              "explicit_rows": rows, "camera_sums": sums, "observations": int(info["observation_count"])}), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0
    for _ in range(args.warmup):
        plan.solve()
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    t_wall = time.perf_counter()
    reports, ms, mixed_sol = timed_solves(plan.solve, stream, flush, args.steps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    clock_summary = clocks.stop()
    barrier()
    local_s = sum(ms) / 1e3
    local_its = sum(r["iteration_count"] for r in reports)
    total_s, total_its = aggregate(local_s, float(local_its), device="cuda")
    value = total_its / total_s
    launches = sum(r["kernel_launches"] for r in reports)
    roofline = kernel_roofline(plan, info, stream, flush, args.workload)
    kernels = {"camera_sums": stage_timing(plan, info, stream, flush, 3, "k_block_tiles + k_block_records"),
               "explicit_rows": stage_timing(plan, info, stream, flush, 2, "k_block_rows")}
    plan.close()

    if args.legs == "value":  # profiling runs: the resident mixed solve and the kernel timing only
        adjuster.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup, "legs": "value", "gpu_launches": int(launches),
                              "roofline": roofline, "clocks": clock_summary}), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0

    # FP64 on the same problem: the comparison at equal final cost
    fp64_cfg = solve_config(abi.PRECISION_FP64, max_iterations=args.max_iterations, stream=stream.cuda_stream)
    plan64 = adjuster.plan(problem, fp64_cfg)
    plan64.solve()
    torch.cuda.synchronize()
    barrier()
    reports64, ms64, sol64 = timed_solves(plan64.solve, stream, flush, args.steps)
    barrier()
    plan64.close()
    s64, its64 = aggregate(sum(ms64) / 1e3, float(sum(r["iteration_count"] for r in reports64)), device="cuda")

    # e2e: omvgba_solve from host arrays every step
    barrier()
    e2e_reports, e2e_ms, _ = timed_solves(lambda: adjuster.solve(problem, mixed_cfg), stream, flush, args.steps)
    barrier()
    e2e_s, e2e_its = aggregate(sum(e2e_ms) / 1e3, float(sum(r["iteration_count"] for r in e2e_reports)),
                               device="cuda")

    # second leg: the 500-camera problem to convergence in both precisions (one timed solve each)
    second = None
    if args.workload != SECOND_LEG and args.second_leg:
        p2 = problem_for(rank, SECOND_LEG)
        pair = precision_pair(adjuster, p2, stream, flush, 1, 1, args.max_iterations)
        second = {"workload": WORKLOADS[SECOND_LEG]["text"],
                  "observations": int(pair["mixed"]["info"]["observation_count"]),
                  "reduced_dimension": int(pair["mixed"]["info"]["reduced_dimension"])} | leg_summary(pair, 1)
    adjuster.close()

    cpu = cpu1 = None
    if rank == 0 and world == 1 and args.legs == "all":
        iterations = CPU_SAMPLE_ITERATIONS.get(args.workload, 1)
        cpu = cpu_sample(problem, iterations)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample", "call_seconds")} | {"cpu": cpu_info()}
        # one host thread on the 500-camera problem's first LM iteration
        c1 = cpu_sample(problem_for(0, SECOND_LEG), 1, threads=1)
        cpu1 = {k: c1[k] for k in ("value", "unit", "cores", "kind")} | {
            "sample": "oracle on the first LM iteration of the 500-camera problem (plane500), one host thread, "
                      "lowering and final certificate included", "cpu": cpu_info()}

    if rank == 0:
        pair = {"mixed": {"reports": reports, "seconds": total_s, "iterations": total_its},
                "fp64": {"reports": reports64, "seconds": s64, "iterations": its64}}
        head = leg_summary(pair, args.steps)
        steps = args.steps
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total_s / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload]["text"], "max_iterations": args.max_iterations,
                       "precision": "mixed", "parallelism": f"replicas x{world}",
                       "observations": int(info["observation_count"]), "points": int(info["point_count"]),
                       "cameras": int(info["camera_count"]), "reduced_dimension": int(info["reduced_dimension"]),
                       "l2": ("inputs larger than L2: %.0f MB of Jacobian records and tile tables per solve vs "
                              "126 MB L2; L2 also flushed (512 MB write) before every step"
                              % ((info["record_bytes_fp32"] + info["record_bytes_fp64"] + info["metadata_bytes_fp32"]
                                  + info["metadata_bytes_fp64"]) / 1e6))},
            "time_to_converge_s": head["mixed"]["time_to_converge_s"],
            "converged": head["mixed"]["converged"],
            "lm_iterations_per_step": local_its / steps,
            "pcg_iterations_per_step": sum(r["pcg_iteration_count"] for r in reports) / steps,
            "final_cost": head["mixed"]["final_cost"],
            "fp64": head["fp64"] | {"pcg_iterations_per_step": sum(r["pcg_iteration_count"] for r in reports64) / steps},
            "mixed_vs_fp64": head["mixed_vs_fp64"],
            "targets": head["targets"],
            "second_leg": second,
            "clocks": clock_summary,
            "e2e": {"value": e2e_its / e2e_s, "unit": UNIT, "time_to_converge_s": e2e_s / steps,
                    "h2d_bytes_per_step": int(sum(r["h2d_bytes"] for r in e2e_reports) / steps),
                    "d2h_bytes_per_step": int(sum(r["d2h_bytes"] for r in e2e_reports) / steps),
                    "host_buffers": "numpy arrays passed to omvgba_solve (lowering on the host inside the step)"},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "kernel_timings": kernels,
            "cpu_baseline": cpu,
            "cpu_baseline_single_thread": cpu1,
            "wall_s_timed_region": wall,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--max-iterations", type=int, default=MAX_ITERATIONS, help="LM iteration budget of every solve")
    ap.add_argument("--legs", choices=["all", "gpu", "value", "kernel", "sfm"], default="all",
                    help="gpu: every leg but the CPU baseline; value: only the resident mixed solve and the kernel "
                         "timing (for profiler runs); kernel: only the product kernel's timing, no solve; sfm: the "
                         "SfM-side reprojection-error refresh over the workload's landmarks")
    ap.add_argument("--no-second-leg", dest="second_leg", action="store_false",
                    help="skip the 500-camera mixed/FP64 leg of the headline line")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "windows256":
        return run_batched(args)
    if args.workload == "residual10m":
        return run_residual(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
