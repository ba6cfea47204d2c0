"""Stereo observations: rectified (BaStereoObservation, normal_equations.rs:
496-570) and calibrated general stereo (BaGeneralStereoObservation,
sqrt_qr.rs:465-518).

The scenes are the reference's stereo tests restated (pipelines/slam/tests/
bundle_adjustment.rs:1516-1760): a rectified rig over the six-point grid, a
general stereo pair with a rotated right camera and unequal intrinsics.  The
CPU tests pin the oracle by those tests' assertions; the GPU tests run the
same scenes through the device and hold a synthetic stereo window to the
oracle."""

from __future__ import annotations

import math

import numpy as np
import pytest

from _scenes import (general_stereo_window_packed, pinhole, pose_at, pose_with_yaw, project,
                     stereo_window_packed, world_grid)
from oracle import oracle
from visloc_ba import (
    SE3,
    BaConfig,
    BaError,
    BaGeneralStereoObservation,
    BaStereoObservation,
    BundleAdjustment,
    Camera,
    CameraModel,
    PackedProblem,
    Pose,
    synth,
)
from visloc_ba import _abi
from visloc_ba.problem import quat_to_matrix
from visloc_ba.solver import GpuBaSettings, GpuBundleAdjuster, check


def quat_from_euler(roll, pitch, yaw):
    """Rz(yaw) Ry(pitch) Rx(roll) as a unit quaternion (w, i, j, k)."""
    cr, sr = math.cos(roll / 2), math.sin(roll / 2)
    cp, sp = math.cos(pitch / 2), math.sin(pitch / 2)
    cy, sy = math.cos(yaw / 2), math.sin(yaw / 2)
    return (cr * cp * cy + sr * sp * sy, sr * cp * cy - cr * sp * sy,
            cr * sp * cy + sr * cp * sy, cr * cp * sy - sr * sp * cy)


def apply(se3: SE3, p):
    r = quat_to_matrix(se3.rotation)
    return tuple(r @ np.asarray(p, dtype=float) + np.asarray(se3.translation, dtype=float))


def pinhole_pixel(camera: Camera, xc):
    fx, fy, cx, cy = camera.params[0], camera.params[1], camera.params[2], camera.params[3]
    return (fx * xc[0] / xc[2] + cx, fy * xc[1] / xc[2] + cy)


def truth_stereo_bundle(baseline: float) -> BundleAdjustment:
    """truth_stereo_bundle (:1516-1551): three poses along x, every grid point
    seen by each left camera and its rectified right camera."""
    camera = pinhole()
    ba = BundleAdjustment(camera)
    ba.set_stereo_baseline(baseline)
    poses = [(10, pose_at((0.0, 0.0, 0.0))), (20, pose_at((0.5, 0.0, 0.0))),
             (30, pose_at((1.0, 0.0, 0.0)))]
    for pid, p in poses:
        ba.add_pose(pid, p)
    for lid, x in world_grid():
        ba.add_landmark(lid, x)
    fx = camera.params[0]
    for pid, p in poses:
        for lid, x in world_grid():
            xc = p.transform_world_point(x)
            uv = project(camera, xc)
            ba.add_stereo_observation(BaStereoObservation(pid, lid, uv, uv[0] - fx * baseline / xc[2]))
    return ba


RIGHT = Camera.pinhole(640, 480, 510.0, 495.0, 318.0, 242.0)
LEFT_TO_RIGHT = SE3(quat_from_euler(0.01, -0.02, 0.015), (-0.11, 0.002, 0.001))


def general_observation(pid, lid, pose: Pose, x, left: Camera):
    pl = pose.transform_world_point(x)
    pr = apply(LEFT_TO_RIGHT, pl)
    return BaGeneralStereoObservation(pid, lid, pinhole_pixel(left, pl), pinhole_pixel(RIGHT, pr),
                                      RIGHT, LEFT_TO_RIGHT)


def truth_general_stereo_bundle():
    """truth_general_stereo_bundle (:1636-1667): one fixed pose, one point."""
    left = pinhole()
    pose = Pose()
    truth = (0.2, -0.1, 4.0)
    ba = BundleAdjustment(left)
    ba.add_pose(10, pose)
    ba.fix_pose(10)
    ba.add_landmark(5, truth)
    ba.add_general_stereo_observation(general_observation(10, 5, pose, truth, left))
    return ba, truth


def general_stereo_pose_bundle():
    """bundle_general_stereo_recovers_pose_with_rotated_right_camera
    (:1702-1755): fixed grid, one drifted pose."""
    left = pinhole()
    truth_pose = pose_with_yaw((0.25, -0.03, 0.04), 0.035)
    ba = BundleAdjustment(left)
    ba.add_pose(10, Pose.from_world_to_camera(quat_from_euler(0.025, 0.07, -0.018),
                                              (-0.39, 0.12, -0.08)))
    for lid, x in world_grid():
        ba.add_landmark(lid, x)
        ba.fix_landmark(lid)
        ba.add_general_stereo_observation(general_observation(10, lid, truth_pose, x, left))
    return ba, truth_pose


def oracle_solve(ba: BundleAdjustment, cfg: BaConfig | None = None):
    packed, pose_ids, lm_ids, missing = ba.pack()
    st, res = oracle.optimize(packed, cfg or BaConfig())
    assert st == 0, _abi.STATUS_NAMES.get(st, st)
    ba.unpack(packed, pose_ids, lm_ids)
    return res


def center(ba, pid):
    return np.asarray(ba.poses[pid].camera_center_world())


# ------------------------------------------------------------------ CPU side
def test_stereo_costs_vanish_at_truth():
    packed = truth_stereo_bundle(0.5).pack()[0]
    assert oracle.cost(packed)[0] < 1e-20
    ba, _ = truth_general_stereo_bundle()
    assert oracle.cost(ba.pack()[0])[0] < 1e-20


def test_missing_or_invalid_baseline_is_rejected():
    """bundle_stereo_optimize_rejects_missing_baseline (:1564-1581)."""
    for b in (None, 0.0, float("nan")):
        ba = truth_stereo_bundle(0.5)
        ba.stereo_baseline = b
        packed = ba.pack()[0]
        assert check(packed)[0] == _abi.ERR_MISSING_STEREO_BASELINE
        assert oracle.check(packed)[0] == _abi.ERR_MISSING_STEREO_BASELINE


def test_stereo_needs_a_pinhole_camera():
    """non_pinhole_lens_with_stereo_or_unknown_model_is_rejected (:825-848)."""
    ba = truth_stereo_bundle(0.12)
    ba.camera = Camera(CameraModel.SIMPLE_RADIAL, 640, 480, [500.0, 320.0, 240.0, -0.1])
    ba.fix_pose(10)
    packed = ba.pack()[0]
    assert check(packed)[0] == _abi.ERR_UNSUPPORTED_CAMERA_MODEL
    assert oracle.check(packed)[0] == _abi.ERR_UNSUPPORTED_CAMERA_MODEL


def test_oracle_stereo_recovers_metric_pose_with_one_anchor():
    """bundle_stereo_recovers_metric_pose_with_single_anchor (:1584-1616)."""
    ba = truth_stereo_bundle(0.5)
    ba.fix_pose(10)
    ba.add_pose(30, pose_at((1.07, 0.04, 0.05)))
    res = oracle_solve(ba)
    assert res.final_cost < 1e-12
    assert np.linalg.norm(center(ba, 30) - (1.0, 0.0, 0.0)) < 1e-7
    assert np.linalg.norm(center(ba, 20) - (0.5, 0.0, 0.0)) < 1e-7


def test_oracle_stereo_recovers_drifted_landmark():
    """bundle_stereo_recovers_drifted_landmark (:1619-1633)."""
    ba = truth_stereo_bundle(0.5)
    for pid in (10, 20, 30):
        ba.fix_pose(pid)
    ba.add_landmark(5, (0.20, 0.10, 6.30))
    res = oracle_solve(ba)
    assert res.final_cost < 1e-14
    assert np.linalg.norm(np.asarray(ba.landmarks[5]) - (0.0, 0.0, 6.0)) < 1e-8


def test_oracle_general_stereo_recovers_landmark_and_pose():
    """bundle_general_stereo_recovers_landmark_with_rotated_right_camera
    (:1680-1699) and ..._recovers_pose_with_rotated_right_camera (:1702-1755)."""
    ba, truth = truth_general_stereo_bundle()
    ba.add_landmark(5, (0.45, 0.08, 4.8))
    assert oracle.cost(ba.pack()[0])[0] > 1.0
    res = oracle_solve(ba)
    assert res.final_cost < 1e-14
    assert np.linalg.norm(np.asarray(ba.landmarks[5]) - truth) < 1e-8
    ba, truth_pose = general_stereo_pose_bundle()
    res = oracle_solve(ba)
    assert res.final_cost < 1e-12
    assert np.linalg.norm(center(ba, 10) - truth_pose.camera_center_world()) < 1e-7


def test_weights_follow_the_flattened_observation_order():
    """Monocular, rectified, general stereo: a zero weight on the general
    stereo observation removes exactly its residual."""
    ba, _ = truth_general_stereo_bundle()
    ba.add_landmark(5, (0.45, 0.08, 4.8))
    packed = ba.pack()[0]
    assert packed.obs_kind.tolist() == [_abi.OBS_GENERAL_STEREO]
    packed.obs_weight = np.array([0.0])
    assert oracle.cost(packed)[0] == 0.0


# ------------------------------------------------------------------ GPU side
@pytest.mark.gpu
def test_device_stereo_scenes_recover_truth(solver):
    acc = GpuBundleAdjuster(0, GpuBaSettings(100, 1e-8, True))
    ba = truth_stereo_bundle(0.5)
    ba.fix_pose(10)
    ba.add_pose(30, pose_at((1.07, 0.04, 0.05)))
    res = acc.solve(ba, BaConfig())
    assert res.final_cost < 1e-10 and res.converged
    assert np.linalg.norm(center(ba, 30) - (1.0, 0.0, 0.0)) < 1e-6
    assert np.linalg.norm(center(ba, 20) - (0.5, 0.0, 0.0)) < 1e-6
    ba, truth = truth_general_stereo_bundle()
    ba.add_landmark(5, (0.45, 0.08, 4.8))
    res = acc.solve(ba, BaConfig())
    assert res.final_cost < 1e-10
    assert np.linalg.norm(np.asarray(ba.landmarks[5]) - truth) < 1e-6
    ba, truth_pose = general_stereo_pose_bundle()
    res = acc.solve(ba, BaConfig())
    assert res.final_cost < 1e-10
    assert np.linalg.norm(center(ba, 10) - truth_pose.camera_center_world()) < 1e-6
    ba = truth_stereo_bundle(0.5)
    ba.stereo_baseline = None
    with pytest.raises(BaError) as e:
        acc.solve(ba, BaConfig())
    assert e.value.kind == "MissingStereoBaseline"


@pytest.mark.gpu
@pytest.mark.parametrize("general", [False, True])
def test_stereo_window_matches_the_oracle(solver, general):
    p = general_stereo_window_packed() if general else stereo_window_packed()
    from visloc_ba import RobustKernel

    cfg = BaConfig(max_iterations=20, robust_kernel=RobustKernel.huber(1.0),
                   max_pcg_iterations=300, pcg_relative_tolerance=1e-8)
    gpu, ref = p.copy(), p.copy()
    c, bad = solver.cost(gpu, cfg)
    c_ref, bad_ref = oracle.cost(ref, cfg)
    assert bad == bad_ref and c == pytest.approx(c_ref, rel=1e-12)
    st, res = solver.optimize(gpu, cfg)
    assert st == _abi.OK, solver.last_error()
    st, rr = oracle.optimize(ref, cfg)
    assert st == 0
    assert abs(res.final_cost - rr.final_cost) <= 1e-5 * rr.final_cost
    extent = synth.scene_extent(ref)
    assert np.abs(gpu.camera_centers() - ref.camera_centers()).max() <= 1e-5 * extent


@pytest.mark.gpu
def test_stereo_and_monocular_problems_in_one_batch(solver):
    probs = [stereo_window_packed(seed=4), synth.ring_problem(12, 500, seed=9),
             stereo_window_packed(seed=5, cams=8, points=400)]
    cfg = BaConfig(max_iterations=8)
    alone = []
    for p in probs:
        q = p.copy()
        st, r = solver.optimize(q, cfg)
        assert st == _abi.OK, solver.last_error()
        alone.append((q, r))
    batch = [p.copy() for p in probs]
    statuses, results = solver.batch_optimize(batch, cfg)
    assert statuses == [_abi.OK] * 3
    for (q, ra), b, rb in zip(alone, batch, results):
        assert rb.final_cost == ra.final_cost
        assert np.array_equal(q.pose_q, b.pose_q) and np.array_equal(q.landmarks, b.landmarks)
