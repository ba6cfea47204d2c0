"""The reference's own BA test scenes, restated (pipelines/slam/tests/
bundle_adjustment.rs): the 640x480 f=500 pinhole (:17-19), cameras translated
along x with identity rotation (:21-25), the six-point grid (:33-44) and the
exact truth bundle (:47-77)."""

from __future__ import annotations

import math

import numpy as np

from visloc_ba import (
    SE3,
    BaObservation,
    BundleAdjustment,
    Camera,
    CameraModel,
    PackedProblem,
    Pose,
    quat_from_axis_angle,
    synth,
)
from visloc_ba import _abi


def pinhole() -> Camera:
    return Camera.pinhole(640, 480, 500.0, 500.0, 320.0, 240.0)


def pose_at(center) -> Pose:
    return Pose.from_world_to_camera((1.0, 0.0, 0.0, 0.0),
                                     (-center[0], -center[1], -center[2]))


def pose_with_yaw(center, yaw) -> Pose:
    q = quat_from_axis_angle((0.0, 1.0, 0.0), yaw)
    p = Pose.from_world_to_camera(q, (0.0, 0.0, 0.0))
    t = p.world_to_camera.transform_point(center)
    return Pose.from_world_to_camera(q, (-t[0], -t[1], -t[2]))


def world_grid():
    return [
        (1, (-1.0, -0.5, 5.0)),
        (2, (1.0, -0.5, 5.0)),
        (3, (-1.0, 0.5, 5.0)),
        (4, (1.0, 0.5, 5.0)),
        (5, (0.0, 0.0, 6.0)),
        (6, (0.5, 0.25, 7.0)),
    ]


def intrinsics(camera: Camera):
    """(fx, fy, cx, cy, k1, k2) of the radial pinhole family (camera.rs:213-260)."""
    p = list(camera.params)
    if camera.model in (CameraModel.PINHOLE, CameraModel.OPENCV):
        return p[0], p[1], p[2], p[3], (p[4] if len(p) > 4 else 0.0), (p[5] if len(p) > 5 else 0.0)
    if camera.model == CameraModel.SIMPLE_PINHOLE:
        return p[0], p[0], p[1], p[2], 0.0, 0.0
    if camera.model == CameraModel.SIMPLE_RADIAL:
        return p[0], p[0], p[1], p[2], (p[3] if len(p) > 3 else 0.0), 0.0
    return p[0], p[0], p[1], p[2], (p[3] if len(p) > 3 else 0.0), (p[4] if len(p) > 4 else 0.0)


def project(camera: Camera, xc):
    """Camera::project for the radial pinhole family (camera.rs:412-430)."""
    fx, fy, cx, cy, k1, k2 = intrinsics(camera)
    x = xc[0] / xc[2]
    y = xc[1] / xc[2]
    if k1 != 0.0 or k2 != 0.0:
        r2 = x * x + y * y
        d = 1.0 + k1 * r2 + k2 * r2 * r2
        x *= d
        y *= d
    return (fx * x + cx, fy * y + cy)


TRUTH_POSES = [(10, (0.0, 0.0, 0.0)), (20, (0.5, 0.0, 0.0)), (30, (1.0, 0.0, 0.0))]


def truth_bundle(camera: Camera | None = None) -> BundleAdjustment:
    camera = camera or pinhole()
    ba = BundleAdjustment(camera)
    poses = [(i, pose_at(c)) for i, c in TRUTH_POSES]
    for i, p in poses:
        ba.add_pose(i, p)
    for lid, x in world_grid():
        ba.add_landmark(lid, x)
    for kid, p in poses:
        for lid, x in world_grid():
            ba.add_observation(BaObservation(kid, lid, project(camera, p.transform_world_point(x))))
    return ba


def drifted_bundle(camera: Camera | None = None) -> BundleAdjustment:
    """bundle_optimize_pulls_drifted_pose_back_to_truth (:367-402) and
    drifted_bundle_through (:406-437): KF 10 and 20 fixed, KF 30 drifted
    (and, with `camera` given, landmark 5 drifted too)."""
    ba = truth_bundle(camera)
    ba.fix_pose(10)
    ba.fix_pose(20)
    ba.add_pose(30, pose_at((1.05, 0.02, 0.03)))
    if camera is not None:
        ba.add_landmark(5, (0.03, -0.02, 6.1))
    return ba


def center_error(ba: BundleAdjustment, pid: int, truth) -> float:
    c = ba.poses[pid].camera_center_world()
    return math.sqrt(sum((a - b) ** 2 for a, b in zip(c, truth)))


# ------------------------------------------------ synthetic stereo windows
def _left_and_rectified(seed, cams, points):
    """The synthetic rig window, its left-camera observation rows, and for
    each left observation with a right partner (same pose and point) its row
    and the right column u_r."""
    p = synth.stereo_window(cams, points, seed=seed)
    left = np.nonzero(p.obs_camera == 0)[0]
    keys = {}
    for k in np.nonzero(p.obs_camera != 0)[0]:
        keys[(int(p.obs_pose[k]), int(p.obs_landmark[k]))] = k
    rows, ur = [], []
    for k in left:
        r = keys.get((int(p.obs_pose[k]), int(p.obs_landmark[k])))
        if r is not None:
            rows.append(k)
            ur.append(p.obs_xy[r, 0])
    return p, left, np.array(rows), np.array(ur)


def stereo_window_packed(seed=3, cams=12, points=700):
    """A synthetic rectified-stereo window: every rig observation pair of the
    synthetic stereo window becomes one rectified observation (the right
    camera of that window is translated by the baseline along x)."""
    p, _, rows, ur = _left_and_rectified(seed, cams, points)
    cam_left, ext_right = p.cameras[0][0], p.cameras[1][1]
    baseline = -ext_right.translation[0]
    stereo = np.zeros((rows.size, 2))
    stereo[:, 0] = ur
    return PackedProblem(p.pose_q, p.pose_t, p.landmarks, p.obs_pose[rows], p.obs_landmark[rows],
                         p.obs_xy[rows], [cam_left], p.pose_fixed, p.landmark_fixed, None, None,
                         np.full(rows.size, _abi.OBS_STEREO, np.uint8), stereo, None, baseline)


def general_stereo_window_packed(seed=3, cams=12, points=700):
    """The same window as calibrated stereo: right pixel (u_r, v), right
    camera = the left one shifted by the baseline."""
    p = stereo_window_packed(seed, cams, points)
    st = p.obs_stereo.copy()
    st[:, 1] = p.obs_xy[:, 1]
    right = (p.cameras[0][0], SE3((1.0, 0.0, 0.0, 0.0), (-p.stereo_baseline, 0.0, 0.0)))
    return PackedProblem(p.pose_q, p.pose_t, p.landmarks, p.obs_pose, p.obs_landmark, p.obs_xy,
                         [p.cameras[0], right], p.pose_fixed, p.landmark_fixed, None, None,
                         np.full(p.num_observations, _abi.OBS_GENERAL_STEREO, np.uint8), st,
                         np.ones(p.num_observations, np.uint32), 0.0)


def mixed_stereo_window_packed(seed=3, cams=12, points=700, camera=None):
    """Monocular and rectified stereo observations in one problem, in the
    reference's flattened order (monocular first): every left-camera
    observation of the window as a monocular one, then the rectified ones.
    Returns the problem and its monocular part alone.  `camera` replaces
    BundleAdjustment::camera (cameras[0])."""
    p, left, rows, ur = _left_and_rectified(seed, cams, points)
    cam_left, ext_right = p.cameras[0][0], p.cameras[1][1]
    cam = camera or cam_left
    baseline = -ext_right.translation[0]
    idx = np.concatenate([left, rows])
    kind = np.concatenate([np.zeros(left.size, np.uint8),
                           np.full(rows.size, _abi.OBS_STEREO, np.uint8)])
    stereo = np.zeros((idx.size, 2))
    stereo[left.size:, 0] = ur
    mixed = PackedProblem(p.pose_q, p.pose_t, p.landmarks, p.obs_pose[idx], p.obs_landmark[idx],
                          p.obs_xy[idx], [cam], p.pose_fixed, p.landmark_fixed, None, None, kind,
                          stereo, None, baseline)
    mono = PackedProblem(p.pose_q, p.pose_t, p.landmarks, p.obs_pose[left], p.obs_landmark[left],
                         p.obs_xy[left], [cam], p.pose_fixed, p.landmark_fixed)
    return mixed, mono
