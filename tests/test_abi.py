"""The C ABI without a GPU: the library loads, exports every entry point the
header declares, and its host-side validation and planning behave."""

from __future__ import annotations

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from _scenes import drifted_bundle, pinhole
from visloc_ba import BaConfig, Camera, CameraModel, PackedProblem, RobustKernel, synth
from visloc_ba import _abi
from visloc_ba.solver import check, plan

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(visloc_ba_cuda_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _abi.load_solver_library()
    declared = header_functions()
    assert len(declared) >= 10
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) <= set(_abi.SOLVER_EXPORTS), set(declared) - set(_abi.SOLVER_EXPORTS)
    assert lib.visloc_ba_cuda_abi_version() == _abi.ABI_VERSION


def test_struct_sizes_match_the_header_layout():
    assert C.sizeof(_abi.Camera) == 8 + 8 * 8 + 4 * 8 + 3 * 8
    # ... cameras, obs_weight, then obs_kind, obs_stereo, obs_right_camera, stereo_baseline
    assert C.sizeof(_abi.Problem) == 3 * 8 + 9 * 8 + 8 + 8 + 8 + 4 * 8
    assert C.sizeof(_abi.Iteration) == 8 + 5 * 8 + 8 + 8 + 4 * 8
    assert C.sizeof(_abi.ReducedSystem) == 8 + 8 + 4 * 8 + 8 + 8
    assert C.sizeof(_abi.ReducedPreconditioner) == 8 + 3 * 8 + 8 + 8
    assert C.sizeof(_abi.ReducedTiming) == 4 * 8
    assert C.sizeof(_abi.PointElimination) == 8 + 8 + 8 + 8 + 6 * 8 + 8 + 2 * 8 + 8 + 8 + 8


def test_default_config_is_the_reference_default():
    """BaConfig::default (bundle/mod.rs:729-752) and GpuBaSettings
    (crates/ba-gpu/src/solver.rs:36-50)."""
    lib = _abi.load_solver_library()
    c = _abi.Config()
    lib.visloc_ba_cuda_default_config(C.byref(c))
    assert c.max_iterations == 20
    assert c.has_initial_lambda == 1 and c.initial_lambda == 1e-4
    assert (c.lambda_increase_factor, c.lambda_decrease_factor) == (10.0, 0.1)
    assert (c.max_lambda, c.min_lambda) == (1e12, 1e-9)
    assert (c.step_tolerance, c.cost_tolerance) == (1e-7, 1e-9)
    assert c.has_relative_cost_tolerance == 0
    assert c.robust_kernel == _abi.KERNEL_NONE
    assert c.max_pcg_iterations == 100 and c.pcg_relative_tolerance == 1e-4
    py = BaConfig().to_abi()
    for name, _ in _abi.Config._fields_:
        if name != "reserved":
            assert getattr(py, name) == getattr(c, name), name


def test_validation_statuses():
    cam = pinhole()
    assert check(PackedProblem(np.zeros((0, 4)), np.zeros((0, 3)), np.zeros((0, 3)), [], [],
                               np.zeros((0, 2)), [cam]))[0] == _abi.ERR_NO_POSES
    assert check(PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], [[0, 0, 5]], [], [],
                               np.zeros((0, 2)), [cam]))[0] == _abi.ERR_NO_OBSERVATIONS
    assert check(PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], np.zeros((0, 3)), [0], [0],
                               [[1, 2]], [cam]))[0] == _abi.ERR_NO_LANDMARKS
    assert check(PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], [[0, 0, 5]], [4], [0], [[1, 2]],
                               [cam])) == (_abi.ERR_MISSING_POSE, 4)
    assert check(PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], [[0, 0, 5]], [0], [7], [[1, 2]],
                               [cam])) == (_abi.ERR_MISSING_LANDMARK, 7)
    assert check(PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], [[0, 0, 5]], [0], [0], [[1, 2]],
                               [cam], pose_fixed=[1], landmark_fixed=[1]))[0] == \
        _abi.ERR_ALL_POSES_FIXED
    fisheye = Camera(CameraModel.OTHER, 640, 480, [300.0, 300.0, 320.0, 240.0])
    assert check(PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], [[0, 0, 5]], [0], [0], [[1, 2]],
                               [fisheye]))[0] == _abi.DECLINED
    tangential = Camera(CameraModel.OPENCV, 640, 480, [500, 500, 320, 240, 0.1, 0.0, 0.01, 0])
    assert check(PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], [[0, 0, 5]], [0], [0], [[1, 2]],
                               [tangential]))[0] == _abi.DECLINED
    bad_params = Camera(CameraModel.PINHOLE, 640, 480, [500.0, 500.0])
    assert check(PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], [[0, 0, 5]], [0], [0], [[1, 2]],
                               [bad_params]))[0] == _abi.ERR_UNSUPPORTED_CAMERA_MODEL
    ba = drifted_bundle()
    packed, _, _, _ = ba.pack()
    assert check(packed)[0] == _abi.OK


def test_validation_of_a_large_problem_reports_the_first_bad_observation():
    """Past a few hundred thousand observations validation scans them on the
    host's threads; the error reported is still the serial scan's: the
    lowest bad observation, its pose checked before its landmark."""
    n, poses, points = 1_500_000, 50, 200_000
    rng = np.random.default_rng(5)
    q = np.tile([1.0, 0.0, 0.0, 0.0], (poses, 1))
    t = np.zeros((poses, 3))
    x = rng.normal(size=(points, 3)) + [0.0, 0.0, 10.0]
    obs_pose = rng.integers(0, poses, n).astype(np.uint32)
    obs_landmark = rng.integers(0, points, n).astype(np.uint32)
    xy = rng.normal(size=(n, 2))

    def run(pose, landmark, weight=None):
        return check(PackedProblem(q, t, x, pose, landmark, xy, [pinhole()], obs_weight=weight))

    assert run(obs_pose, obs_landmark)[0] == _abi.OK
    op, ol = obs_pose.copy(), obs_landmark.copy()
    op[1_400_000] = poses + 3
    ol[900_000] = points + 9
    assert run(op, ol) == (_abi.ERR_MISSING_LANDMARK, points + 9)
    op[700_000] = poses + 1
    assert run(op, ol) == (_abi.ERR_MISSING_POSE, poses + 1)
    ol[700_000] = points + 2  # same observation: the pose is checked first
    assert run(op, ol) == (_abi.ERR_MISSING_POSE, poses + 1)
    w = np.ones(n)
    w[1_200_000] = -1.0
    w[300_001] = np.nan
    assert run(obs_pose, obs_landmark, w) == (_abi.ERR_INVALID_OBSERVATION_WEIGHT, 300_001)


@pytest.mark.parametrize("maker", [
    lambda: synth.ring_problem(12, 400, seed=7),
    lambda: synth.ring_problem(50, 5000, seed=1001),
    lambda: synth.stereo_window(25, 1200, seed=4),
    lambda: synth.pose_only(300, seed=2),
    lambda: drifted_bundle().pack()[0],
])
def test_plan_is_consistent(maker):
    """The device layout passes its bounds check (every index inside the array
    it addresses) and its counts agree with a direct count."""
    p = maker()
    st, info = plan(p, BaConfig())
    assert st == _abi.OK
    var_cams = int(p.num_poses - (p.pose_fixed.sum() if p.pose_fixed is not None else 0))
    assert info.variable_cameras == var_cams
    assert info.tile_rows * info.tile_size >= var_cams
    assert info.device_bytes > 0 and info.upload_bytes > 0
    # Camera pairs: distinct (i, j) of variable cameras sharing a variable point.
    pose_fixed = p.pose_fixed if p.pose_fixed is not None else np.zeros(p.num_poses, np.uint8)
    lm_fixed = p.landmark_fixed if p.landmark_fixed is not None else np.zeros(p.num_landmarks,
                                                                              np.uint8)
    pairs = set()
    terms = 0
    by_point = {}
    for k in range(p.num_observations):
        if pose_fixed[p.obs_pose[k]] or lm_fixed[p.obs_landmark[k]]:
            continue
        by_point.setdefault(int(p.obs_landmark[k]), []).append(int(p.obs_pose[k]))
    for cams in by_point.values():
        for a in cams:
            for b in cams:
                if a > b:
                    pairs.add((a, b))
                    terms += 1
    assert info.camera_pairs == len(pairs)
    assert info.schur_terms == terms


def test_plan_handles_duplicate_observations():
    """A camera observing the same point twice contributes same-camera Schur
    terms; the plan stays consistent."""
    p = synth.ring_problem(6, 50, seed=3)
    dup = PackedProblem(p.pose_q, p.pose_t, p.landmarks,
                        np.concatenate([p.obs_pose, p.obs_pose[:5]]),
                        np.concatenate([p.obs_landmark, p.obs_landmark[:5]]),
                        np.concatenate([p.obs_xy, p.obs_xy[:5] + 0.5]), p.cameras, p.pose_fixed,
                        p.landmark_fixed,
                        None if p.obs_camera is None else
                        np.concatenate([p.obs_camera, p.obs_camera[:5]]))
    st, info = plan(dup, BaConfig(robust_kernel=RobustKernel.huber(1.0)))
    assert st == _abi.OK


REFINEMENT_FLAGS = ["refine_intrinsics", "refine_distortion", "refine_tangential_distortion",
                    "shared_focal"]


@pytest.mark.parametrize("flag", REFINEMENT_FLAGS)
def test_intrinsics_refinement_is_declined(flag):
    """GpuBundleAdjuster::check declines refine_intrinsics || refine_distortion
    before looking at the problem (crates/ba-gpu/src/solver.rs:214-216); this
    library keeps the intrinsics fixed, so it declines every self-calibration
    switch of BaConfig (bundle/mod.rs:669-700), first of all checks."""
    cfg = BaConfig(**{flag: True})
    assert getattr(cfg.to_abi(), flag) == 1
    packed, _, _, _ = drifted_bundle().pack()
    assert check(packed, BaConfig())[0] == _abi.OK
    assert check(packed, cfg)[0] == _abi.DECLINED
    assert plan(packed, cfg)[0] == _abi.DECLINED
    # Declined before validation: a problem with a missing pose is not an error here.
    bad = PackedProblem([[1, 0, 0, 0]], [[0, 0, 0]], [[0, 0, 5]], [4], [0], [[1, 2]], [pinhole()])
    assert check(bad, cfg)[0] == _abi.DECLINED


@pytest.mark.parametrize("term,value", [
    ("gravity_prior", object()),
    ("per_pose_gravity_prior", object()),
    ("position_prior", object()),
    ("pairwise_pose_factors", [object()]),
    ("velocities", {1: (0.0, 0.0, 0.0)}),
    ("imu_factors", [object()]),
    ("biases", {1: object()}),
    ("bias_random_walk_factors", [object()]),
    ("navigation_state_prior", object()),
    ("fixed_pose_rotations", {1}),
])
def test_unmodelled_terms_are_declined_by_the_accelerator(term, value):
    """Priors, the inertial state and rotation-fixed poses make
    GpuBundleAdjuster::check return Unsupported (solver.rs:230-246), so the
    plug-in returns None and the CPU solver runs.  The accelerator here is
    built without a device: a solve attempt would fail on its missing solver,
    so None proves that the decline came first and left `ba` untouched."""
    from visloc_ba.solver import GpuBaSettings, GpuBundleAdjuster

    ba = drifted_bundle()
    before = {k: (tuple(p.world_to_camera.rotation), tuple(p.world_to_camera.translation))
              for k, p in ba.poses.items()}
    acc = object.__new__(GpuBundleAdjuster)
    acc.solver = None
    acc.settings = GpuBaSettings()
    assert ba.unsupported_terms() is None
    setattr(ba, term, value)
    assert ba.unsupported_terms() is not None
    assert acc.optimize(ba, BaConfig()) is None
    after = {k: (tuple(p.world_to_camera.rotation), tuple(p.world_to_camera.translation))
             for k, p in ba.poses.items()}
    assert after == before
