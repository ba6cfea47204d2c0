"""Writes the fixtures of tests/golden: problems in the reference's dump
format (ba_problem_io.rs) and the FP64 oracle's solve of each, so the CPU
tests pin the oracle's results, the dump reader/writer round trip and the
replay of a file against committed data.  The expected values come from the
oracle (this repository's FP64 restatement), not from the Rust reference,
which cannot run here.

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "visloc-rs_b200"), os.path.dirname(HERE)]

import numpy as np  # noqa: E402

from oracle import oracle  # noqa: E402
from visloc_ba import BaConfig, RobustKernel, synth  # noqa: E402
from visloc_ba.problem_io import read_packed_problem, write_packed_problem  # noqa: E402

CASES = {
    # 12 cameras on a ring, shared 4-parameter pinhole (the dump format's camera).
    "ring12": dict(make=lambda: synth.ring_problem(12, 300, seed=1212, width=1280, height=960,
                                                   focal=(900.0, 900.0), k1=(0.0, 0.0),
                                                   per_camera_intrinsics=False),
                   config=dict(max_iterations=15, robust_kernel=("huber", 1.0))),
    # A short street loop: forward cameras, facade points.
    "street160": dict(make=lambda: synth.street_loop(160, 1200, seed=1616, fixed=(0, 1, 80),
                                                    track=(10.0, 3, 20), outlier_fraction=0.0),
                     config=dict(max_iterations=20, robust_kernel=("none", 0.0))),
}


def config_of(spec) -> BaConfig:
    kind, value = spec["robust_kernel"]
    rk = {"none": RobustKernel.none(), "huber": RobustKernel.huber(value),
          "cauchy": RobustKernel.cauchy(value)}[kind]
    return BaConfig(max_iterations=spec["max_iterations"], robust_kernel=rk)


def main():
    for name, case in CASES.items():
        p = case["make"]()
        pose_ids = [10 * i + 3 for i in range(p.num_poses)]  # sparse ascending ids
        lm_ids = [7 * i + 1 for i in range(p.num_landmarks)]
        path = os.path.join(HERE, f"{name}_problem.txt")
        write_packed_problem(p, pose_ids, lm_ids, None, path)
        q, _, _, _ = read_packed_problem(path)
        cfg = config_of(case["config"])
        st, res = oracle.optimize(q, cfg)
        assert st == 0
        expected = {
            "config": case["config"],
            "initial_cost": res.initial_cost,
            "final_cost": res.final_cost,
            "converged": res.converged,
            "step_accepted": [bool(i.step_accepted) for i in res.iterations],
            "lambda": [i.lambda_ for i in res.iterations],
            "camera_centers": q.camera_centers().tolist(),
            "landmark_sum": np.asarray(q.landmarks).sum(0).tolist(),
            "scene_extent": synth.scene_extent(q),
        }
        with open(os.path.join(HERE, f"{name}_expected.json"), "w") as f:
            json.dump(expected, f, indent=1)
        print(name, p.num_poses, p.num_landmarks, p.num_observations, res.final_cost)


if __name__ == "__main__":
    main()
