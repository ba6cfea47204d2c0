"""Plain-text dump and load of a monocular pinhole bundle adjustment, in the
format of the reference's ba_problem_io (pipelines/slam/src/ba_problem_io.rs
:20-149), so the problems its incremental SfM dumps (VISLOC_SFM_BA_DUMP) can
be replayed here:

    camera <width> <height> <fx> <fy> <cx> <cy>
    poses <N>
    <id> <qw> <qi> <qj> <qk> <tx> <ty> <tz> <fixed 0|1>      (ascending id)
    landmarks <M>
    <id> <x> <y> <z>                                         (ascending id)
    observations <K> <weighted 0|1>
    <pose id> <landmark id> <u> <v> [<weight>]

Floats are written with Python's shortest round-trip repr, so a reload is
exact (the reference writes Rust's shortest round-trip form; both parse to
the same doubles).  Quaternions are normalised on load, as
UnitQuaternion::from_quaternion does (ba_problem_io.rs:111-116).
"""

from __future__ import annotations

import math

import numpy as np

from .problem import (
    SE3,
    BaObservation,
    BundleAdjustment,
    Camera,
    CameraModel,
    PackedProblem,
    Pose,
)


def _normalise(q):
    """nalgebra Unit::new_normalize of Quaternion(w, i, j, k): divide by the
    norm of its coordinate vector, summed in storage order (i, j, k, w)."""
    w, i, j, k = (float(v) for v in q)
    n = math.sqrt(i * i + j * j + k * k + w * w)
    return (w / n, i / n, j / n, k / n)


def write_ba_problem(ba: BundleAdjustment, weights, path) -> None:
    """write_ba_problem (ba_problem_io.rs:20-64): the pinhole monocular part."""
    c = ba.camera
    if c.model != CameraModel.PINHOLE or len(c.params) < 4:
        raise ValueError("the dump format holds a 4-parameter pinhole camera")
    fx, fy, cx, cy = (float(v) for v in c.params[:4])
    out = [f"camera {int(c.width)} {int(c.height)} {fx!r} {fy!r} {cx!r} {cy!r}",
           f"poses {len(ba.poses)}"]
    for pid in sorted(ba.poses):
        s = ba.poses[pid].world_to_camera
        q, t = s.rotation, s.translation
        out.append(f"{pid} {float(q[0])!r} {float(q[1])!r} {float(q[2])!r} {float(q[3])!r} "
                   f"{float(t[0])!r} {float(t[1])!r} {float(t[2])!r} "
                   f"{1 if pid in ba.fixed_poses else 0}")
    out.append(f"landmarks {len(ba.landmarks)}")
    for lid in sorted(ba.landmarks):
        x = ba.landmarks[lid]
        out.append(f"{lid} {float(x[0])!r} {float(x[1])!r} {float(x[2])!r}")
    out.append(f"observations {len(ba.observations)} {1 if weights is not None else 0}")
    for n, o in enumerate(ba.observations):
        line = f"{o.keyframe_id} {o.landmark_id} {float(o.xy[0])!r} {float(o.xy[1])!r}"
        if weights is not None:
            line += f" {float(weights[n])!r}"
        out.append(line)
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def _sections(path):
    with open(path) as f:
        lines = f.read().split("\n")
    pos = 0

    def take(tag: str):
        nonlocal pos
        if pos >= len(lines):
            raise ValueError(f"missing {tag}")
        head = lines[pos].split()
        pos += 1
        if not head or head[0] != tag:
            raise ValueError(f"expected a {tag} line")
        return head

    def rows(n: int, tag: str):
        nonlocal pos
        if pos + n > len(lines):
            raise ValueError(f"truncated {tag}")
        block = lines[pos:pos + n]
        pos += n
        return block

    cam = take("camera")
    if len(cam) != 7:
        raise ValueError("camera line")
    camera = Camera.pinhole(int(cam[1]), int(cam[2]), float(cam[3]), float(cam[4]),
                            float(cam[5]), float(cam[6]))
    np_ = int(take("poses")[1])
    poses = rows(np_, "poses")
    nl = int(take("landmarks")[1])
    lms = rows(nl, "landmarks")
    head = take("observations")
    no = int(head[1])
    weighted = len(head) > 2 and head[2] == "1"
    obs = rows(no, "observations")
    return camera, poses, lms, obs, weighted


def read_ba_problem(path):
    """read_ba_problem (ba_problem_io.rs:70-149): (BundleAdjustment, weights
    or None), ids as in the file."""
    camera, poses, lms, obs, weighted = _sections(path)
    ba = BundleAdjustment(camera)
    for line in poses:
        v = line.split()
        pid = int(v[0])
        q = _normalise(v[1:5])
        ba.add_pose(pid, Pose(SE3(q, (float(v[5]), float(v[6]), float(v[7])))))
        if v[8] == "1":
            ba.fix_pose(pid)
    for line in lms:
        v = line.split()
        ba.add_landmark(int(v[0]), (float(v[1]), float(v[2]), float(v[3])))
    weights = [] if weighted else None
    for line in obs:
        v = line.split()
        ba.add_observation(BaObservation(int(v[0]), int(v[1]), (float(v[2]), float(v[3]))))
        if weighted:
            weights.append(float(v[4]))
    return ba, weights


def read_packed_problem(path):
    """The same file straight into the dense arrays of the C ABI (fast for
    large dumps): (PackedProblem, pose ids, landmark ids, weights or None).
    Observations whose ids do not resolve keep the index 0xFFFFFFFF, which
    validation reports as MissingPose / MissingLandmark."""
    camera, poses, lms, obs, weighted = _sections(path)
    P = np.array([line.split() for line in poses], dtype=object).reshape(-1, 9)
    pose_ids = P[:, 0].astype(np.uint64)
    q = P[:, 1:5].astype(np.float64)
    q = np.array([_normalise(r) for r in q]).reshape(-1, 4)
    t = P[:, 5:8].astype(np.float64)
    fixed = (P[:, 8] == "1").astype(np.uint8)
    L = np.array([line.split() for line in lms], dtype=object).reshape(-1, 4)
    lm_ids = L[:, 0].astype(np.uint64)
    X = L[:, 1:4].astype(np.float64)
    width = 5 if weighted else 4
    O = np.array([line.split()[:width] for line in obs], dtype=object).reshape(-1, width)
    o_pose = O[:, 0].astype(np.uint64)
    o_lm = O[:, 1].astype(np.uint64)
    xy = O[:, 2:4].astype(np.float64)
    weights = O[:, 4].astype(np.float64) if weighted else None

    def dense(ids_sorted, refs):
        if not np.all(ids_sorted[1:] > ids_sorted[:-1]):
            raise ValueError("ids must be ascending and unique")
        at = np.searchsorted(ids_sorted, refs)
        ok = (at < ids_sorted.size)
        ok[ok] = ids_sorted[at[ok]] == refs[ok]
        return np.where(ok, at, 0xFFFFFFFF).astype(np.uint32)

    packed = PackedProblem(q, t, X, dense(pose_ids, o_pose), dense(lm_ids, o_lm), xy, [camera],
                           fixed, np.zeros(X.shape[0], np.uint8), None)
    return packed, [int(v) for v in pose_ids], [int(v) for v in lm_ids], weights


def write_packed_problem(packed: PackedProblem, pose_ids, lm_ids, weights, path) -> None:
    """Dense arrays to the dump format (monocular, cameras[0] a pinhole)."""
    cam = packed.cameras[0][0]
    if cam.model != CameraModel.PINHOLE or packed.obs_camera is not None:
        raise ValueError("the dump format holds monocular observations of a pinhole camera")
    pf = packed.pose_fixed if packed.pose_fixed is not None else np.zeros(packed.num_poses)
    fx, fy, cx, cy = (float(v) for v in cam.params[:4])
    out = [f"camera {int(cam.width)} {int(cam.height)} {fx!r} {fy!r} {cx!r} {cy!r}",
           f"poses {packed.num_poses}"]
    for i in range(packed.num_poses):
        q, t = packed.pose_q[i], packed.pose_t[i]
        out.append(f"{pose_ids[i]} {float(q[0])!r} {float(q[1])!r} {float(q[2])!r} "
                   f"{float(q[3])!r} {float(t[0])!r} {float(t[1])!r} {float(t[2])!r} "
                   f"{int(pf[i])}")
    out.append(f"landmarks {packed.num_landmarks}")
    for i in range(packed.num_landmarks):
        x = packed.landmarks[i]
        out.append(f"{lm_ids[i]} {float(x[0])!r} {float(x[1])!r} {float(x[2])!r}")
    out.append(f"observations {packed.num_observations} {1 if weights is not None else 0}")
    for n in range(packed.num_observations):
        line = (f"{pose_ids[packed.obs_pose[n]]} {lm_ids[packed.obs_landmark[n]]} "
                f"{float(packed.obs_xy[n, 0])!r} {float(packed.obs_xy[n, 1])!r}")
        if weights is not None:
            line += f" {float(weights[n])!r}"
        out.append(line)
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
