"""Replay a dumped bundle-adjustment problem (the reference's
VISLOC_SFM_BA_DUMP text format, see problem_io) on the GPU solver: time,
LM iterations, robust cost, RMS reprojection error before and after.  The
counterpart of the reference's crates/ba-gpu/examples/ba_gpu_replay.rs
(whose CPU-solver comparison has its place in this repository's tests).

    python visloc-rs_b200/visloc_ba/replay.py problem.txt [--iterations 20]
        [--local N] [--robust huber:1.0] [--pcg-tol 1e-4] [--pcg-max 100]
        [--repeat 3] [--weights]

--local N keeps only the last N poses variable (fixing the rest), only the
landmarks they observe and every pose observing those: the shape of the
SfM's local BA window.  Per-observation weights in the file are used only with
--weights (the semantics of optimize_with_observation_weights; the reference
offers only unweighted problems to its accelerator, pipelines/slam/src/
ba_accel.rs:1-7); the replay reports whether they were present.  Prints one
JSON object.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402

from visloc_ba import BaConfig, RobustKernel  # noqa: E402
from visloc_ba.problem import PackedProblem  # noqa: E402
from visloc_ba.problem_io import read_packed_problem  # noqa: E402
from visloc_ba.solver import CudaSolver  # noqa: E402


def local_window(packed: PackedProblem, n: int) -> PackedProblem:
    """The last n poses variable, the landmarks they observe, the poses that
    observe those (the others fixed); ba_gpu_replay.rs:45-66."""
    variable = np.zeros(packed.num_poses, bool)
    variable[max(0, packed.num_poses - n):] = True
    keep_lm = np.zeros(packed.num_landmarks, bool)
    keep_lm[packed.obs_landmark[variable[packed.obs_pose]]] = True
    sel = keep_lm[packed.obs_landmark]
    used = np.zeros(packed.num_poses, bool)
    used[packed.obs_pose[sel]] = True
    pose_map = np.cumsum(used) - 1
    lm_map = np.cumsum(keep_lm) - 1
    fixed = (~variable[used]).astype(np.uint8)
    return PackedProblem(packed.pose_q[used], packed.pose_t[used], packed.landmarks[keep_lm],
                         pose_map[packed.obs_pose[sel]], lm_map[packed.obs_landmark[sel]],
                         packed.obs_xy[sel], packed.cameras, fixed,
                         np.zeros(int(keep_lm.sum()), np.uint8), None,
                         None if packed.obs_weight is None else packed.obs_weight[sel])


def robust(spec: str) -> RobustKernel:
    if spec == "none":
        return RobustKernel.none()
    kind, _, value = spec.partition(":")
    if kind == "huber":
        return RobustKernel.huber(float(value or 1.0))
    if kind == "cauchy":
        return RobustKernel.cauchy(float(value or 1.0))
    raise ValueError(f"robust kernel {spec!r}: none, huber:<delta> or cauchy:<c>")


def rms_reprojection(solver: CudaSolver, packed: PackedProblem) -> float:
    """sqrt(mean squared reprojection error), from the device cost with no
    robust kernel and no weights (ba_gpu_replay.rs:18-28)."""
    plain = packed.copy()
    plain.obs_weight = None
    cost, _ = solver.cost(plain, BaConfig(robust_kernel=RobustKernel.none()))
    return math.sqrt(cost / max(1, packed.num_observations))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("problem")
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--local", type=int, default=0)
    ap.add_argument("--robust", default="none")
    ap.add_argument("--pcg-tol", type=float, default=1e-4)
    ap.add_argument("--pcg-max", type=int, default=100)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--weights", action="store_true",
                    help="solve with the file's per-observation weights")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    packed, pose_ids, lm_ids, weights = read_packed_problem(a.problem)
    if a.weights and weights is not None:
        packed.obs_weight = np.ascontiguousarray(weights, dtype=np.float64)
    if a.local:
        packed = local_window(packed, a.local)
    load_s = time.perf_counter() - t0
    cfg = BaConfig(max_iterations=a.iterations, robust_kernel=robust(a.robust),
                   max_pcg_iterations=a.pcg_max, pcg_relative_tolerance=a.pcg_tol)
    out = {"problem": a.problem, "poses": packed.num_poses,
           "fixed_poses": int(packed.pose_fixed.sum()), "landmarks": packed.num_landmarks,
           "observations": packed.num_observations, "weights_in_file": weights is not None,
           "weights_used": packed.obs_weight is not None,
           "local_window": a.local or None, "load_s": load_s}
    runs = []
    with CudaSolver(a.device) as solver:
        out["rms_px_before"] = rms_reprojection(solver, packed)
        for _ in range(max(1, a.repeat)):
            q = packed.copy()
            t = time.perf_counter()
            st, res = solver.optimize(q, cfg)
            wall = time.perf_counter() - t
            if st != 0:
                out["gpu_error"] = solver.last_error() or str(st)
                break
            runs.append({"wall_s": wall, "upload_ms": res.upload_ms, "device_ms": res.device_ms,
                         "iterations": len(res.iterations),
                         "accepted": sum(i.step_accepted for i in res.iterations),
                         "initial_cost": res.initial_cost, "final_cost": res.final_cost,
                         "converged": res.converged})
            out["rms_px_after"] = rms_reprojection(solver, q)
    out["gpu"] = runs
    print(json.dumps(out))
    return 0 if runs else 1


if __name__ == "__main__":
    sys.exit(main())
