"""Full-size parity against the FP64 oracle's committed solves (test
infrastructure: used by tests/, bench.py's parity figure and the fixture
script tests/golden/make_parity_fixtures.py; never by the product).

The oracle (ba_oracle.cpp, the FP64 restatement of the reference solver,
bundle/lm.rs:162-1017) needs minutes of CPU for the benchmarked workloads,
so its answers are computed once and committed as fixtures under
tests/golden/.  Each fixture carries a digest of the generated input; a
comparison first checks that the seeded generator still produces the same
problem, then states the device solve's error:

  final_cost_rel   |cost - cost_oracle| / cost_oracle
  centre_err       max over cameras of |c - c_oracle| (each coordinate) /
                   scene extent

against the north-star tolerance of 1e-5 for both.
"""

from __future__ import annotations

import hashlib
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
TOLERANCE = 1e-5

# Windows of the windows-512 batch (seed 4000) that the fixture solves.
WINDOW_SAMPLE = list(range(0, 512, 16))


def input_digest(p) -> str:
    """sha256 over the arrays that define a PackedProblem (state,
    observations, fixed flags, weights, stereo data, camera parameters)."""
    h = hashlib.sha256()
    for a in (p.pose_q, p.pose_t, p.landmarks, p.obs_pose, p.obs_landmark, p.obs_xy,
              p.pose_fixed, p.landmark_fixed, p.obs_camera, p.obs_weight, p.obs_kind,
              p.obs_stereo, p.obs_right_camera):
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    for cam, ext in p.cameras:
        h.update(np.asarray(cam.params, dtype=np.float64).tobytes())
        h.update(np.asarray(tuple(ext.rotation) + tuple(ext.translation), np.float64).tobytes())
    return h.hexdigest()


def ring4m_config():
    """The benchmarked ring-4m solve: Huber 1 px, 30 LM iterations, PCG
    tolerance 1e-6 with at most 200 iterations on the device."""
    from visloc_ba import BaConfig, RobustKernel

    return BaConfig(max_iterations=30, robust_kernel=RobustKernel.huber(1.0),
                    max_pcg_iterations=200, pcg_relative_tolerance=1e-6)


def street20m_config():
    """The benchmarked street-20m solve: Huber 1 px, 15 LM iterations, PCG
    tolerance 1e-6 with at most 200 iterations on the device."""
    from visloc_ba import BaConfig, RobustKernel

    return BaConfig(max_iterations=15, robust_kernel=RobustKernel.huber(1.0),
                    max_pcg_iterations=200, pcg_relative_tolerance=1e-6)


def windows_config():
    """The benchmarked windows-512 solve: Huber 1 px, 10 LM iterations, PCG
    tolerance 1e-6 with at most 200 iterations on the device."""
    from visloc_ba import BaConfig, RobustKernel

    return BaConfig(max_iterations=10, robust_kernel=RobustKernel.huber(1.0),
                    max_pcg_iterations=200, pcg_relative_tolerance=1e-6)


def fixture_path(name: str) -> str:
    return os.path.join(GOLDEN, f"{name}_oracle.npz")


def load(name: str):
    """The committed fixture `name` (ring4m, windows512_sample), or None."""
    path = fixture_path(name)
    if not os.path.exists(path):
        return None
    with np.load(path, allow_pickle=False) as f:
        return {k: f[k] for k in f.files}


def compare_state(final_cost: float, centers: np.ndarray, oracle_cost: float,
                  oracle_centers: np.ndarray, extent: float) -> dict:
    rel = abs(final_cost - oracle_cost) / max(abs(oracle_cost), 1e-300)
    dc = float(np.abs(np.asarray(centers) - oracle_centers).max()) / extent
    return {"final_cost_rel": rel, "centre_err_of_extent": dc}


FIXTURES = {
    "ring-4m": ("ring4m", "FP64 sparse Schur + block Cholesky LM, 30 iterations "
                          "(tests/golden/ring4m_oracle.npz)"),
    "street-20m": ("street20m", "FP64 sparse Schur + banded block Cholesky LM, 15 iterations "
                                "(tests/golden/street20m_oracle.npz)"),
}


def workload_parity(workload: str, problem, final_cost: float, centers: np.ndarray):
    """Error of a benchmarked solve (its final cost and camera centres)
    against the oracle fixture of `workload`; None when the fixture is absent
    or was made from a different input."""
    if workload not in FIXTURES:
        return None
    name, what = FIXTURES[workload]
    fx = load(name)
    if fx is None or str(fx["digest"]) != input_digest(problem):
        return None
    out = compare_state(final_cost, centers, float(fx["final_cost"]), fx["centers"],
                        float(fx["extent"]))
    out.update({"oracle": what, "oracle_final_cost": float(fx["final_cost"]),
                "tolerance": TOLERANCE,
                "within_tolerance": bool(out["final_cost_rel"] <= TOLERANCE
                                         and out["centre_err_of_extent"] <= TOLERANCE)})
    return out


def ring4m_parity(problem, final_cost: float, centers: np.ndarray):
    return workload_parity("ring-4m", problem, final_cost, centers)
