#!/usr/bin/env python
"""Benchmark: LM iterations/s and observations/s of the 4M-observation bundle
adjustment on B200, with the HBM roofline fraction of the dominant kernel.

Workload (default `ring-4m`): 1,200 cameras on a ring with shared pinhole
intrinsics (6000x4000), 500,000 points in a 10 m cube, track lengths geometric
(mean 8, clipped to [2, 60]) -> ~4.06M observations; pixel noise N(0,1),
2% outliers within +-50 px, poses perturbed 0.01 rad / 0.05 m, Huber 1 px,
30 LM iterations, PCG tolerance 1e-6.  Inputs are seeded synthetic data
(no data set is needed or used).

One step = one LM solve (all its iterations) from the same initial state.
`value` times steps on the device with the problem resident in HBM (events
on the solver's stream inside the library); `e2e` times the C-ABI call
`visloc_ba_cuda_optimize` with host buffers (host-side planning, H2D, LM,
D2H).  With --gpus N every rank solves its own problem (replicas, weak
scaling); the reported time is the max over ranks.

--impl reference times the CPU restatement of the reference solver (the FP64
oracle, OpenMP over all host cores): one LM iteration of the same workload
per step.

Workload `windows-512`: 512 uneven local BA windows (5-40 stereo keyframes,
baseline 0.11 m, 752x480 pinhole, 200-5,000 points, 3-12 observations per
point, 10% of the poses fixed), ~9.3M observations, solved as one batch with
the 10-iteration LM loop captured as a CUDA graph; one step = one batched
solve.  `value` counts the LM iterations of all windows.

Workload `served`: a Poisson stream of requests, 70% local windows (10-40
stereo keyframes, 1k-5k points), 25% pose-only refinements (100-2,000
matches, 30% outliers), 5% global BAs (300 cameras, 60k points, ~400k
observations), through the serving loop (visloc_ba_cuda_server_*) at an
offered rate of five times the plain per-problem solve rate; `value` is the
served solves/s (wall clock), with p50/p99 latency, beside the plain rate
(the same requests solved one by one through visloc_ba_cuda_optimize) and the
saturated rate (every request submitted at once).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "visloc-rs_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

FALLBACK_HBM_GBS = 6650.0
PCG_KERNEL = "k_pcg"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ring-4m",
                    choices=["ring-4m", "ring-50", "street-20m", "windows-512", "served",
                             "reduced-5822"])
    ap.add_argument("--requests", type=int, default=300, help="served: stream length")
    ap.add_argument("--reduced-nodes", type=int, default=5822,
                    help="reduced-5822: nodes (smaller for profiling captures)")
    ap.add_argument("--obs-per-frame", type=int, default=2500,
                    help="reduced-5822: observations per frame of the elimination scene")
    ap.add_argument("--reduced-part", default="all", choices=["all", "solve", "eliminate"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="ring-4m: skip the other workloads' sub-objects of the line")
    return ap.parse_args()


# ---------------------------------------------------------------- workloads
def make_workload(name: str, rank: int):
    from visloc_ba import BaConfig, RobustKernel, synth

    if name == "ring-4m":
        problem = synth.large_ring_problem(seed=2000 + rank)
        cfg = BaConfig(max_iterations=30, robust_kernel=RobustKernel.huber(1.0),
                       max_pcg_iterations=200, pcg_relative_tolerance=1e-6, autotune=True)
        desc = {"workload": "ring-4m", "cameras": 1200, "points": 500_000,
                "observations": int(problem.num_observations), "image": "6000x4000",
                "lm_iterations": 30, "pcg_tolerance": 1e-6, "robust": "huber(1px)",
                "track_length": "geometric mean 8, [2,60]"}
    elif name == "street-20m":
        problem = synth.street_loop(seed=3000 + rank)
        cfg = BaConfig(max_iterations=15, robust_kernel=RobustKernel.huber(1.0),
                       max_pcg_iterations=200, pcg_relative_tolerance=1e-6, autotune=True)
        desc = {"workload": "street-20m", "cameras": 5600, "points": int(problem.num_landmarks),
                "observations": int(problem.num_observations), "image": "1920x1080",
                "scene": "closed street loop, facade planes +-0.2 m",
                "lm_iterations": 15, "pcg_tolerance": 1e-6, "robust": "huber(1px)",
                "track_length": "consecutive views, geometric mean 6.7, [2,40]"}
    elif name == "windows-512":
        problem = synth.window_batch(512, seed=4000 + 1000 * rank)
        cfg = BaConfig(max_iterations=10, robust_kernel=RobustKernel.huber(1.0),
                       max_pcg_iterations=200, pcg_relative_tolerance=1e-6, graph=True,
                       autotune=True)
        desc = {"workload": "windows-512", "windows": 512,
                "keyframes": "U{5..40} stereo (baseline 0.11 m)", "image": "752x480",
                "points": int(sum(p.num_landmarks for p in problem)),
                "observations": int(sum(p.num_observations for p in problem)),
                "lm_iterations": 10, "pcg_tolerance": 1e-6, "robust": "huber(1px)",
                "fixed_poses": "10%", "cuda_graph": True, "autotuned_launch_shape": True}
    else:
        problem = synth.ring_problem(50, 5000, seed=1001 + rank)
        cfg = BaConfig(max_iterations=20, robust_kernel=RobustKernel.huber(1.0),
                       max_pcg_iterations=200, pcg_relative_tolerance=1e-6)
        desc = {"workload": "ring-50", "cameras": 50, "points": 5000,
                "observations": int(problem.num_observations), "image": "640x480",
                "lm_iterations": 20, "robust": "huber(1px)"}
    return problem, cfg, desc


# ------------------------------------------------------------- distributed
class Dist:
    """Replicas: one process per GPU, each solving its own problem; the
    process group carries only the barrier and the max/sum of the timings
    (NCCL on GPUs, gloo for the CPU tests)."""

    def __init__(self, backend: str = "nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            if backend == "nccl":
                torch.cuda.set_device(self.local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                        device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def _device(self):
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self._device())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self._device())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def replica_rate(dist: Dist, units: float, seconds: float):
    """Whole-job rate of replicas: the units of all ranks over the slowest
    rank's time (weak scaling).  Returns (rate, max seconds)."""
    t_max = dist.max(seconds)
    return dist.sum(units) / t_max, t_max


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_pcg_iteration(workload: str):
    """DRAM bytes per PCG iteration of k_pcg from the committed ncu summary
    of this workload (profiles/k_pcg_<workload>_traffic.txt); None for a
    workload that has no capture of its own."""
    path = os.path.join(ROOT, "profiles", f"k_pcg_{workload.replace('-', '')}_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_pcg_iteration"):
                    return float(line.split("=")[1])
    except (OSError, ValueError):
        pass
    return None


# -------------------------------------------------------------- CPU side
def cpu_sample(problem, cfg, threads=0):
    """One LM iteration of the FP64 oracle on all host cores, on the whole
    workload: (seconds, fraction of the workload's observations it covered,
    always 1).  The oracle's sparse solve factors the reduced system in band
    storage when it is banded (the street loop) and densely otherwise."""
    from oracle import oracle

    c = problem.copy()
    one = type(cfg)(**{**cfg.__dict__, "max_iterations": 1})
    t0 = time.perf_counter()
    st, _ = oracle.optimize(c, one, solver=oracle.SPARSE_BANDED, threads=threads)
    dt = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError(f"oracle failed: {st}")
    return dt, 1.0


def batch_cpu_sample(problems, cfg, windows=128):
    """The oracle's full solve (all threads) of the first `windows` windows:
    (LM iterations, seconds)."""
    from oracle import oracle

    one = type(cfg)(**{**cfg.__dict__, "graph": False})
    iters, t0 = 0, time.perf_counter()
    for p in problems[:windows]:
        st, res = oracle.optimize(p.copy(), one, solver=oracle.SPARSE)
        if st != 0:
            raise RuntimeError(f"oracle failed: {st}")
        iters += len(res.iterations)
    return iters, time.perf_counter() - t0


def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return
    problem, cfg, desc = make_workload(args.workload, 0)
    from oracle import oracle

    oracle.lib()
    cores = os.cpu_count() or 1
    if args.workload == "windows-512":
        times, iters = [], []
        for k in range(args.warmup + args.steps):
            n, dt = batch_cpu_sample(problem[(128 * k) % 512:], cfg)
            if k >= args.warmup:
                times.append(dt)
                iters.append(n)
        value = sum(iters) / sum(times)
        line = {
            "impl": "reference", "metric": "lm_iterations_per_s", "value": value,
            "unit": "LM iterations/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": desc,
            "cpu_baseline": {"value": value, "unit": "LM iterations/s", "cores": cores,
                             "kind": "port",
                             "sample": "full LM solves of 128 windows of the batch per step "
                                       "(FP64 Schur + Cholesky), all host cores"},
            "e2e": {"value": value, "unit": "LM iterations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    for _ in range(args.warmup):  # a cost pass per warm-up step (page-in, threads)
        oracle.cost(problem, cfg)
    samples = [cpu_sample(problem, cfg) for _ in range(args.steps)]
    frac = samples[0][1]
    total = sum(t for t, _ in samples)
    value = args.steps * frac / total  # LM iterations of the whole workload per second
    line = {
        "impl": "reference", "metric": "lm_iterations_per_s", "value": value,
        "unit": "LM iterations/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": desc,
        "observations_per_s": value * desc["observations"],
        "cpu_baseline": {"value": value, "unit": "LM iterations/s", "cores": cores,
                         "kind": "port",
                         "sample": "1 LM iteration (Schur + Cholesky, FP64) per step of the "
                                   + ("same workload" if frac == 1.0 else
                                      f"sub-problem of 700 consecutive poses ({frac:.3f} of the "
                                      "observations; rate scaled by that share)")
                                   + ", all host cores"},
        "e2e": {"value": value, "unit": "LM iterations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------- GPU side
def run_ours(args, dist: Dist):
    import torch

    from visloc_ba.solver import CudaSolver, plan

    torch.cuda.set_device(dist.local)
    problem, cfg, desc = make_workload(args.workload, dist.rank)
    cfg.profile = True
    st, info = plan(problem, cfg, 1.0)
    if st != 0:
        raise RuntimeError(f"plan failed: {st}")
    solver = CudaSolver(dist.local)
    st = solver.upload(problem, cfg)
    if st != 0:
        raise RuntimeError(f"upload failed: {solver.last_error()}")
    for _ in range(args.warmup):
        st, res = solver.solve_uploaded(cfg)
        if st != 0:
            raise RuntimeError(f"solve failed: {solver.last_error()}")

    clocks = Clocks(dist.local)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    wall0 = time.perf_counter()
    results = []
    for _ in range(args.steps):
        st, res = solver.solve_uploaded(cfg)
        if st != 0:
            raise RuntimeError(f"solve failed: {solver.last_error()}")
        results.append(res)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    dist.barrier()
    clk = clocks.stop()

    # Error of the timed solve's result against the FP64 oracle's solve of the
    # same seeded input (committed fixture), where one exists.
    parity_line = None
    from oracle import parity

    if args.workload in parity.FIXTURES:
        final = problem.copy()
        if solver.download(final) == 0:
            parity_line = parity.workload_parity(args.workload, problem,
                                                 results[-1].final_cost, final.camera_centers())

    dev_ms = sum(r.device_ms for r in results)
    lm_iters = sum(len(r.iterations) for r in results)
    pcg_iters = sum(it.pcg_iterations for r in results for it in r.iterations)
    pcg_ms = sum(it.pcg_ms for r in results for it in r.iterations)
    launches = sum(r.kernel_launches for r in results)
    value, t_max = replica_rate(dist, lm_iters, dev_ms / 1e3)
    nobs = desc["observations"]

    # Roofline of the dominant kernel (k_pcg): algorithmic bytes per PCG
    # iteration x iterations of a launch / launch time, averaged over launches.
    b_pcg = info.bytes_per_pcg_iteration
    peak, peak_kind = hbm_peak()
    achieved = (pcg_iters * b_pcg) / (pcg_ms / 1e3) / 1e9 if pcg_ms > 0 else 0.0
    traffic = traffic_per_pcg_iteration(args.workload)
    n_pcg_launches = sum(1 for r in results for it in r.iterations)
    mean_k = pcg_iters / max(1, n_pcg_launches)
    # Whole LM step: algorithmic bytes of linearisation + trial at the mean k.
    st2, info_k = plan(problem, cfg, mean_k)
    step_bytes = info_k.bytes_per_iteration
    step_gbs = step_bytes * lm_iters / (dev_ms / 1e3) / 1e9

    e2e = None
    if not args.no_e2e:
        e2e_cfg = type(cfg)(**{**cfg.__dict__, "profile": False})
        copies = [problem.copy() for _ in range(args.steps)]
        e2e_iters = 0
        up_ms, solve_ms, up_bytes = [], [], []
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for c in copies:
            st, r = solver.optimize(c, e2e_cfg)
            if st != 0:
                raise RuntimeError(f"optimize failed: {solver.last_error()}")
            e2e_iters += len(r.iterations)
            up_ms.append(r.upload_ms)
            solve_ms.append(r.device_ms)
            up_bytes.append(r.upload_bytes)
        torch.cuda.synchronize()
        t_e2e = dist.max(time.perf_counter() - t0)
        e2e = {"value": dist.sum(e2e_iters) / t_e2e, "unit": "LM iterations/s",
               # The library's own count of each call's host -> device bytes.
               "h2d_bytes_per_step": int(max(up_bytes)),
               "d2h_bytes_per_step": int(problem.num_poses * 56 + problem.num_landmarks * 24
                                         + 64 * 30 + 128),
               "ms_per_step": 1e3 * t_e2e / args.steps,
               # Inside each call: validation, plan build, plan check and upload (host
               # clock) and the solve (device time); the rest is the download.
               "upload_ms_per_step": statistics.median(up_ms),
               "solve_device_ms_per_step": statistics.median(solve_ms)}

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        dt, frac = cpu_sample(problem, cfg)
        what = ("the same workload" if frac == 1.0 else
                f"the sub-problem of 700 consecutive poses ({frac:.3f} of the observations; "
                "rate scaled by that share)")
        cpu = {"value": frac / dt, "unit": "LM iterations/s", "cores": os.cpu_count(),
               "kind": "port",
               "sample": f"1 LM iteration (FP64 Schur + Cholesky, banded when the reduced "
                         f"system is) of {what}, {os.cpu_count()} threads, {dt:.1f} s"}

    if dist.rank == 0:
        line = {
            "metric": "lm_iterations_per_s", "value": value, "unit": "LM iterations/s",
            "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": {**desc, "parallelism": f"replicas x{dist.world}",
                                            "l2": "inputs larger than L2 (problem > 0.8 GB)"},
            "observations_per_s": value * nobs,
            "lm_iterations_per_step": lm_iters / args.steps,
            "pcg_iterations_per_lm_iteration": mean_k,
            "roofline": {"kernel": PCG_KERNEL, "bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind,
                         "traffic": traffic, "traffic_unit": "bytes per PCG iteration",
                         "algorithmic_bytes_per_pcg_iteration": b_pcg},
            "lm_step_roofline": {"achieved": step_gbs, "peak": peak, "unit": "GB/s",
                                 "frac": step_gbs / peak,
                                 "algorithmic_bytes_per_lm_iteration": step_bytes},
            "phase_ms_per_lm_iteration": {
                k: sum(getattr(it, f) for r in results for it in r.iterations) / max(1, lm_iters)
                for k, f in [("linearize", "linearize_ms"), ("assemble", "assemble_ms"),
                             ("pcg", "pcg_ms"), ("update_cost_decide", "update_ms")]},
            "final_cost": results[-1].final_cost,
            "initial_cost": results[-1].initial_cost,
            "parity": parity_line,
            "wall_s": wall,
            "clocks": clk,
            "gpu_launches": int(launches),
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
    solver.close()
    return line if dist.rank == 0 else None


def run_batch(args, dist: Dist):
    """Batched windows: every window of the batch in one launch sequence."""
    import torch

    from visloc_ba.solver import CudaSolver

    torch.cuda.set_device(dist.local)
    problems, cfg, desc = make_workload(args.workload, dist.rank)
    solver = CudaSolver(dist.local)
    solver.batch_upload(problems, cfg)
    for _ in range(args.warmup):
        solver.batch_solve_uploaded()
    clocks = Clocks(dist.local)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    wall0 = time.perf_counter()
    runs = [solver.batch_solve_uploaded() for _ in range(args.steps)]
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    dist.barrier()
    clk = clocks.stop()
    dev_ms = sum(r[0].device_ms for r in runs)
    lm_iters = sum(len(x.iterations) for r in runs for x in r)
    obs_iters = sum(len(x.iterations) * p.num_observations for r in runs
                    for x, p in zip(r, problems))
    launches = sum(r[0].kernel_launches for r in runs)
    t_max = dist.max(dev_ms / 1e3)
    value = dist.sum(lm_iters) / t_max

    # Phase times and the PCG roofline from one profiled (host-driven) solve
    # outside the timed region.
    from visloc_ba.solver import plan

    prof_cfg = type(cfg)(**{**cfg.__dict__, "graph": False, "profile": True})
    solver.batch_upload(problems, prof_cfg)
    prof = solver.batch_solve_uploaded()
    # Iteration records carry the phase times of the batch (same on every window).
    its = max(prof, key=lambda x: len(x.iterations)).iterations
    pcg_ms = sum(i.pcg_ms for i in its)
    pcg_bytes = 0.0
    for p, x in zip(problems, prof):
        st, info = plan(p, cfg, 1.0)
        pcg_bytes += info.bytes_per_pcg_iteration * sum(i.pcg_iterations for i in x.iterations)
    peak, peak_kind = hbm_peak()
    achieved = pcg_bytes / (pcg_ms / 1e3) / 1e9 if pcg_ms > 0 else 0.0

    e2e = None
    if not args.no_e2e:
        copies = [[p.copy() for p in problems] for _ in range(min(args.steps, 2))]
        e2e_cfg = type(cfg)(**{**cfg.__dict__})
        dist.barrier()
        t0 = time.perf_counter()
        e2e_iters = 0
        for batch in copies:
            _, rs = solver.batch_optimize(batch, e2e_cfg)
            e2e_iters += sum(len(x.iterations) for x in rs)
        t_e2e = dist.max(time.perf_counter() - t0)
        h2d = sum(p.num_poses * 57 + p.num_landmarks * 25 + p.num_observations * 20
                  for p in problems)
        e2e = {"value": dist.sum(e2e_iters) / t_e2e, "unit": "LM iterations/s",
               "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(sum(p.num_poses * 56 + p.num_landmarks * 24
                                             for p in problems)),
               "ms_per_step": 1e3 * t_e2e / len(copies)}

    # The plain per-problem GPU solve of the same windows (a sample of 32).
    sample = problems[:32]
    plain_cfg = type(cfg)(**{**cfg.__dict__, "graph": False})
    t0 = time.perf_counter()
    plain_iters = 0
    for p in sample:
        st, r = solver.optimize(p.copy(), plain_cfg)
        plain_iters += len(r.iterations)
    plain = plain_iters / (time.perf_counter() - t0)

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        n, dt = batch_cpu_sample(problems, cfg, windows=512)
        cpu = {"value": n / dt, "unit": "LM iterations/s", "cores": os.cpu_count(),
               "kind": "port",
               "sample": f"full LM solves of all 512 windows, {os.cpu_count()} threads, "
                         f"{dt:.1f} s"}

    if dist.rank == 0:
        line = {
            "metric": "lm_iterations_per_s", "value": value, "unit": "LM iterations/s",
            "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {**desc, "parallelism": f"replicas x{dist.world}",
                       "l2": "inputs larger than L2 (batch > 2 GB)"},
            "observations_per_s": dist.sum(obs_iters) / t_max,
            "windows_per_s": dist.sum(512 * args.steps) / t_max,
            "lm_iterations_per_step": lm_iters / args.steps,
            "plain_per_problem_lm_iterations_per_s": plain,
            "roofline": {"kernel": PCG_KERNEL, "bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": None,
                         "traffic_unit": "bytes per PCG iteration"},
            "phase_ms_per_lm_iteration": {
                k: sum(getattr(i, f) for i in its) / max(1, len(its))
                for k, f in [("linearize", "linearize_ms"), ("assemble", "assemble_ms"),
                             ("pcg", "pcg_ms"), ("update_cost_decide", "update_ms")]},
            "wall_s": wall,
            "clocks": clk,
            "gpu_launches": int(launches),
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
    solver.close()
    return line if dist.rank == 0 else None


def served_requests(n, seed):
    from visloc_ba import synth

    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        u = rng.random()
        if u < 0.70:
            reqs.append(("window", synth.stereo_window(int(rng.integers(10, 41)),
                                                       int(rng.integers(1000, 5001)),
                                                       seed=seed + 1 + i)))
        elif u < 0.95:
            reqs.append(("pose-only", synth.pose_only(int(rng.integers(100, 2001)),
                                                      seed=seed + 1 + i)))
        else:
            reqs.append(("global", synth.ring_problem(
                300, 60000, seed=seed + 1 + i, width=1920, height=1080, focal=(1500.0, 1500.0),
                k1=(0.0, 0.0), per_camera_intrinsics=False, track=("geometric", 6.7, 2, 40))))
    return reqs


def serve_stream(server, reqs, cfg, rate, seed):
    """Submit `reqs` at Poisson arrival times (rate per second; 0 = all at
    once) and wait for all: (wall seconds, latencies ms, kinds)."""
    import threading

    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(reqs)) if rate > 0 else np.zeros(len(reqs))
    copies = [p.copy() for _, p in reqs]
    tickets = [None] * len(reqs)
    lat = [None] * len(reqs)
    ready = threading.Semaphore(0)

    def waiter():
        for i in range(len(reqs)):
            ready.acquire()
            st, _, info = server.wait(tickets[i])
            if st != 0:
                raise RuntimeError(f"request {i} failed: {st} {server.last_error()}")
            lat[i] = info["latency_ms"]

    th = threading.Thread(target=waiter)
    th.start()
    t0 = time.perf_counter()
    due = t0
    for i, c in enumerate(copies):
        due += gaps[i]
        delay = due - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        tickets[i] = server.submit(c, cfg)
        ready.release()
    th.join()
    wall = time.perf_counter() - t0
    return wall, lat, [k for k, _ in reqs]


def run_served(args, dist: Dist):
    """The served mixed stream through the serving loop, against the plain
    per-problem solve of the same requests."""
    import torch

    from visloc_ba import BaConfig, RobustKernel
    from visloc_ba.solver import BaServer, CudaSolver

    torch.cuda.set_device(dist.local)
    reqs = served_requests(args.requests, 5000 + 1000 * dist.rank)
    cfg = BaConfig(max_iterations=10, robust_kernel=RobustKernel.huber(1.0),
                   max_pcg_iterations=100, pcg_relative_tolerance=1e-4)
    solver = CudaSolver(dist.local)
    for _, p in reqs[: args.warmup]:
        solver.optimize(p.copy(), cfg)
    dist.barrier()
    plain = 0.0
    for _ in range(2):  # the faster of two passes (host noise only lowers a pass)
        t0 = time.perf_counter()
        for _, p in reqs:
            st, _ = solver.optimize(p.copy(), cfg)
            if st != 0:
                raise RuntimeError(solver.last_error())
        plain = max(plain, len(reqs) / (time.perf_counter() - t0))
    solver.close()

    server = BaServer(dist.local, slots=3, memory_bytes=12 << 30, max_batch=64)
    serve_stream(server, reqs[: max(8, args.warmup)], cfg, 0.0, 1)  # warm-up
    clocks = Clocks(dist.local)
    dist.barrier()
    clocks.start()
    wall, lat, kinds = serve_stream(server, reqs, cfg, 5.0 * plain, 2)
    clk = clocks.stop()
    sat_wall, sat_lat, _ = serve_stream(server, reqs, cfg, 0.0, 3)
    server.close()
    value = dist.sum(len(reqs) / dist.max(wall))
    lat = np.array(lat)
    by_kind = {}
    for k in sorted(set(kinds)):
        v = np.array([x for x, kk in zip(lat, kinds) if kk == k])
        by_kind[k] = {"count": int(v.size), "p50_ms": float(np.percentile(v, 50)),
                      "p99_ms": float(np.percentile(v, 99))}
    if dist.rank == 0:
        nobs = sum(p.num_observations for _, p in reqs)
        line = {
            "metric": "served_solves_per_s", "value": value, "unit": "solves/s",
            "n_gpus": dist.world, "steps": 1, "warmup": args.warmup,
            "ms_per_step": 1e3 * wall, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "served", "requests": len(reqs),
                       "mix": "70% windows (10-40 kf, 1k-5k pts), 25% pose-only "
                              "(100-2000 matches, 30% outliers), 5% global "
                              "(300 cams, 60k pts, ~400k obs)",
                       "observations": int(nobs), "lm_iterations": 10,
                       "pcg": "tol 1e-4, max 100", "robust": "huber(1px)",
                       "arrivals": "Poisson at 5x the plain solve rate",
                       "server": "3 slots x 4 GiB, batches <= 64",
                       "parallelism": f"replicas x{dist.world}"},
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "latency_by_kind": by_kind,
            "offered_rate": 5.0 * plain,
            "plain_per_problem_solves_per_s": plain,
            "saturated_solves_per_s": len(reqs) / sat_wall,
            "saturated_latency_ms": {"p50": float(np.percentile(sat_lat, 50)),
                                     "p99": float(np.percentile(sat_lat, 99))},
            "clocks": clk,
            "e2e": {"value": value, "unit": "solves/s",
                    "h2d_bytes_per_step": int(sum(p.num_poses * 57 + p.num_landmarks * 25 +
                                                  p.num_observations * 20 for _, p in reqs)),
                    "d2h_bytes_per_step": int(sum(p.num_poses * 56 + p.num_landmarks * 24
                                                  for _, p in reqs))},
            "cpu_baseline": None,
        }
        return line
    return None


# ------------------------------------------------ reduced camera system path
REDUCED_NODES = 5822  # SmallCity's photos


def reduced_tiles(edges, n, tb=8):
    """Tiles of S in the device layout: the tile pairs (I <= J) that hold an
    edge, plus the diagonal tiles."""
    import numpy as np

    ti = edges[:, 0].astype(np.int64) // tb
    tj = edges[:, 1].astype(np.int64) // tb
    rows = -(-n // tb)
    return int(np.unique(np.concatenate([ti * rows + tj, np.arange(rows) * (rows + 1)])).size)


def reduced_cpu_iteration_ms(diag, edges, off, rhs, runs, coarse):
    """The reference's CPU iteration (pcg_core, restated in C++ with OpenMP in
    the oracle) on all host threads with the same preconditioner: ms per PCG
    iteration from a 1e-6 solve less a one-iteration solve (the setup in both
    cancels; each the best of three), and the threads used.  On a system so
    small that the difference is lost in timer and thread-start noise, the
    whole solve per iteration (an upper bound) instead."""
    from oracle import oracle

    def solve(k):
        t0 = time.perf_counter()
        r = oracle.reduced_pcg_threaded(diag, edges, off, rhs, 1e-6, k, clusters=runs,
                                        coarse=coarse)
        return time.perf_counter() - t0, (r[1] if r else 0)

    solve(1)  # page-in
    t1 = min(solve(1)[0] for _ in range(3))
    t2, it = min(solve(2000) for _ in range(3))
    per = (t2 - t1) / max(1, it - 1)
    if not per > 0.0:
        per = t2 / max(1, it)
    return 1e3 * per, os.cpu_count() or 1


def run_reduced(args, dist: Dist):
    """ReducedSolveAccelerator at SmallCity size (5,822 nodes): the
    preconditioned PCG (runs of 32, coarse level of 32-node aggregates) and
    block-Jacobi on a 3.4M-edge covisibility system given with its blocks:
    ms per PCG iteration from the device times of the PCG loop (CUDA events
    on the library's stream) of a 1e-6 solve and of a one-iteration solve, the
    C call's fixed cost beside it; and the point elimination of
    a street capture of 14.5M observations (first call with the structure's
    index, then per trial), followed by the preconditioned solve on the
    resident blocks.  Replicas at N > 1."""
    import numpy as np

    from visloc_ba import reduced, synth
    from visloc_ba.solver import CudaSolver

    if args.impl == "reference" and dist.rank != 0:
        return
    n = args.reduced_nodes
    band, cross = min(450, n // 8), min(150, n // 16)
    diag, edges, off = synth.covisibility_system(n, band, cross)
    rhs = np.random.default_rng(7 + dist.rank).standard_normal((n, 6))
    runs = reduced.cluster_inverses(diag, edges, off, 32)
    coarse = reduced.coarse_correction(diag, edges, off, n, 32)
    desc = {"workload": "reduced-5822" if n == REDUCED_NODES else f"reduced-{n}",
            "nodes": n, "edges": int(len(edges)),
            "system": f"covisibility: +-{band} capture-order neighbours, {cross} cross-pass",
            "runs": 32, "coarse_group": int(coarse[0]), "coarse_aggregates": -(-n // coarse[0]),
            "tiles": reduced_tiles(edges, n)}
    if args.impl == "reference":
        ms, cores = reduced_cpu_iteration_ms(diag, edges, off, rhs, runs, coarse)
        line = {"impl": "reference", "metric": "reduced_pcg_iteration_ms", "value": ms,
                "unit": "ms", "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": ms,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "config": desc,
                "cpu_baseline": {"value": ms, "unit": "ms", "cores": cores, "kind": "port",
                                 "sample": "a 1e-6 solve less a one-iteration solve of the "
                                           "FP64 C++ pcg_core restatement, all host threads"},
                "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch

    torch.cuda.set_device(dist.local)
    solver = CudaSolver(dist.local)
    clocks = Clocks(dist.local)

    def solve(**kw):
        """(iterations, device ms per PCG iteration, C-call ms) of a 1e-6
        solve: the device time of its PCG loop less that of a one-iteration
        solve (the loop's setup, the preconditioner's first application and
        the graph's instantiation), over the iterations past the first."""
        solver.reduced_solve(diag, edges, off, rhs, 1e-6, 1, **kw)
        one = solver.reduced_timing()["pcg_ms"]
        _, it, _ = solver.reduced_solve(diag, edges, off, rhs, 1e-6, 2000, **kw)
        per = (solver.reduced_timing()["pcg_ms"] - one) / max(1, it - 1)
        return it, per, solver.last_call_ms

    do_solve = args.reduced_part in ("all", "solve")
    steps = max(1, args.steps) if do_solve else 0
    for _ in range(args.warmup if do_solve else 0):
        solve(clusters=runs, coarse=coarse)
        solve()
    dist.barrier()
    clocks.start()
    pre = [solve(clusters=runs, coarse=coarse) for _ in range(steps)] or [(0, 0.0, 0.0)]
    bj = [solve() for _ in range(steps)] or [(0, 0.0, 0.0)]
    clk = clocks.stop()
    conv_pre, conv_bj = pre[0][0], bj[0][0]
    it_pre = dist.max(float(np.median([p[1] for p in pre])))
    it_bj = dist.max(float(np.median([b[1] for b in bj])))
    call_pre = float(np.median([p[2] for p in pre]))
    fixed = dist.max(call_pre - conv_pre * it_pre)
    # Algorithmic bytes per preconditioned iteration: S's tiles once, the run
    # inverses and the coarse inverse (FP32), about 40 vector passes.
    m = -(-n // coarse[0])
    b_iter = (desc["tiles"] * 64 * 144 + sum(4 * r.shape[0] ** 2 for _, r in runs)
              + 4 * (6 * m) ** 2 + 40 * 24 * n)
    peak, kind = hbm_peak()
    achieved = b_iter / (it_pre * 1e-3) / 1e9 if it_pre > 0 else 0.0
    el_out = None
    if args.reduced_part != "solve":  # elimination of a street capture
        el = synth.street_elimination(n, args.obs_per_frame, seed=11 + dist.rank)
        el_out = reduced_elimination(solver, el, n, args.steps)
    if dist.rank != 0:
        return
    line = {
        "metric": "reduced_pcg_iteration_ms", "value": it_pre, "unit": "ms",
        "n_gpus": dist.world, "steps": max(1, args.steps), "warmup": args.warmup,
        "ms_per_step": it_pre, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": 3.4 / it_pre if it_pre > 0 else None,
        "dtype": "f32 vectors and S, f64 dots",
        "data": "synthetic", "config": desc, "clocks": clk,
        "block_jacobi_iteration_ms": it_bj, "fixed_cost_ms": fixed,
        "solve_to_1e-6": {"preconditioned": {"iterations": conv_pre, "call_ms": call_pre},
                          "block_jacobi": {"iterations": conv_bj,
                                           "call_ms": float(np.median([b[2] for b in bj]))}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_kind": kind,
                     "algorithmic_bytes_per_iteration": b_iter},
        "elimination": el_out,
        "reference_l4": {"pcg_iteration_ms_3.4M_edges": 3.4, "per_solve_fixed_cost_ms": 590,
                         "elimination_per_trial_ms": 1440},
    }
    if not args.no_cpu_baseline and do_solve:
        cpu, cores = reduced_cpu_iteration_ms(diag, edges, off, rhs, runs, coarse)
        line["cpu_baseline"] = {"value": cpu, "unit": "ms", "cores": cores, "kind": "port",
                                "sample": "a 1e-6 solve less a one-iteration solve of the "
                                          "FP64 C++ pcg_core restatement, all host threads"}
    return line


def reduced_elimination(solver, el, n, steps):
    """The elimination part of the reduced workload: the first call (the
    structure's index and the blocks' upload), per-trial calls with new point
    inverses (device time and C-call time), and a preconditioned solve on the
    resident blocks with runs and a coarse level built from what the
    elimination returned."""
    import numpy as np

    from visloc_ba import reduced

    pl = el["point_off"][1:] - el["point_off"][:-1]
    pairs = int((pl * (pl - 1) // 2).sum())
    e2 = el["edges"]
    in_run = np.flatnonzero(e2[:, 0] // 32 == e2[:, 1] // 32).astype(np.uint32)
    group = reduced.coarse_group_size(n, 32)
    args_el = (n, e2, el["point_off"], el["point_nodes"], el["hcp"])
    solver.reduced_eliminate(1, 1, *args_el, el["point_inverse"], (), in_run, (group, n))
    first_ms = solver.last_call_ms
    trial, trial_dev = [], []
    for k in range(max(2, steps)):
        rb, sums = solver.reduced_eliminate(1, 1, *args_el, el["point_inverse"] * (1.0 - 0.01 * k),
                                            (), in_run, (group, n))
        trial.append(solver.last_call_ms)
        trial_dev.append(solver.reduced_timing()["eliminate_ms"])
    el_runs = reduced.cluster_inverses(el["diag"], e2[in_run], rb, 32)
    el_coarse = reduced.coarse_from_sums(el["diag"], sums, n, group)
    _, el_iters, el_rr = solver.reduced_solve(el["diag"], e2, None, el["rhs"], 1e-6, 500,
                                              clusters=el_runs, coarse=el_coarse)
    return {"observations": int(len(el["point_nodes"])), "points": int(len(pl)),
            "edges": int(len(e2)), "pairs": pairs, "first_call_ms": first_ms,
            "per_trial_ms": float(np.median(trial)),
            "per_trial_device_ms": float(np.median(trial_dev)),
            "solve_on_resident_blocks": {"iterations": el_iters, "relative_residual": el_rr,
                                         "call_ms": solver.last_call_ms,
                                         "pcg_device_ms": solver.reduced_timing()["pcg_ms"]}}


def compact(line, keys):
    """The named keys of a workload's line (for the default line's
    other_workloads object)."""
    if line is None:
        return None
    return {k: line.get(k) for k in keys if k in line}


def other_workloads(args, dist: Dist):
    """The other benchmarked workloads, each run and timed on its own after
    the headline solve (short step counts; each with its own clock record),
    so that one default bench run records them all.  Outside the headline
    `value`."""
    out = {}
    common = ["metric", "value", "unit", "ms_per_step", "config", "clocks"]
    sub = argparse.Namespace(**{**vars(args), "steps": min(args.steps, 3),
                                "warmup": min(args.warmup, 2), "no_e2e": False,
                                "no_cpu_baseline": False, "workload": "windows-512"})
    t0 = time.perf_counter()
    out["windows-512"] = compact(run_batch(sub, dist), common + [
        "observations_per_s", "windows_per_s", "plain_per_problem_lm_iterations_per_s",
        "roofline", "phase_ms_per_lm_iteration", "e2e", "cpu_baseline"])
    sub = argparse.Namespace(**{**vars(sub), "workload": "served", "no_cpu_baseline": True})
    out["served"] = compact(run_served(sub, dist), common + [
        "latency_ms", "latency_by_kind", "offered_rate", "plain_per_problem_solves_per_s",
        "saturated_solves_per_s", "saturated_latency_ms"])
    if out["served"]:
        s = out["served"]
        s["speedup_over_plain"] = s["value"] / s["plain_per_problem_solves_per_s"]
    sub = argparse.Namespace(**{**vars(sub), "workload": "reduced-5822", "no_cpu_baseline": False,
                                "reduced_nodes": REDUCED_NODES, "reduced_part": "all"})
    out["reduced-5822"] = compact(run_reduced(sub, dist), common + [
        "block_jacobi_iteration_ms", "fixed_cost_ms", "solve_to_1e-6", "roofline",
        "elimination", "reference_l4", "cpu_baseline", "vs_baseline"])
    out["wall_s"] = time.perf_counter() - t0
    return out


def main():
    args = parse_args()
    dist = Dist()
    try:
        line = None
        if args.workload == "reduced-5822":
            line = run_reduced(args, dist)
        elif args.impl == "reference":
            run_reference(args, dist)
        elif args.workload == "windows-512":
            line = run_batch(args, dist)
        elif args.workload == "served":
            line = run_served(args, dist)
        else:
            line = run_ours(args, dist)
            # One process per GPU of the default run also measures the other
            # workloads (N = 1 only: the scaling runs time the headline alone).
            if dist.world == 1 and args.workload == "ring-4m" and not args.no_extras:
                extra = other_workloads(args, dist)
                if line is not None:
                    line["other_workloads"] = extra
        if line is not None and dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
