"""Diagnostics: one damped linear step of a named synthetic workload on the
GPU (linearisation, reduced-system assembly, a fixed number of PCG
iterations, back-substitution), for profiling single kernels in isolation.

    python visloc-rs_b200/visloc_ba/diag.py --workload ring-4m --pcg-iterations 40

Workloads: ring-4m (1,200 cameras, 500k points, ~4.06M observations, shared
pinhole intrinsics, Huber 1 px), street-20m (5,600 cameras along a closed
street loop, ~20M observations) and ring-50 (50 SIMPLE_RADIAL cameras, 5k
points).  The PCG tolerance is set below reach, so exactly
--pcg-iterations iterations run.
"""

from __future__ import annotations

import argparse
import os
import sys

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from visloc_ba import BaConfig, RobustKernel, synth  # noqa: E402
from visloc_ba.solver import CudaSolver  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="ring-4m", choices=["ring-4m", "street-20m", "ring-50"])
    ap.add_argument("--pcg-iterations", type=int, default=40)
    ap.add_argument("--lam", type=float, default=1e-4)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if a.workload == "ring-4m":
        p = synth.large_ring_problem()
    elif a.workload == "street-20m":
        p = synth.street_loop(seed=3000)
    else:
        p = synth.ring_problem(50, 5000, seed=1001)
    cfg = BaConfig(robust_kernel=RobustKernel.huber(1.0), max_pcg_iterations=a.pcg_iterations,
                   pcg_relative_tolerance=1e-14)
    with CudaSolver(a.device) as s:
        _, _, iters, rr = s.linear_step(p, cfg, a.lam)
    print(f"workload={a.workload} observations={p.num_observations} pcg_iterations={iters} "
          f"relative_residual={rr:.3e}")


if __name__ == "__main__":
    main()
