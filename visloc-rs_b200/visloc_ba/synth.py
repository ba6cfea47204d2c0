"""Seeded synthetic bundle-adjustment problems (no public data set exists for
this path; the shapes follow the benchmark configurations of the solver):

  ring_problem     cameras on a ring looking at points in a cube: the 50-camera
                   SIMPLE_RADIAL problem (per-camera intrinsics, 640x480) and
                   the 1,200-camera / 500k-point / ~4M-observation problem
                   (shared pinhole, 6000x4000), at any size in between;
  street_problem   forward-facing cameras along a closed street loop, points
                   on facade planes;
  stereo_window    a local window of stereo-rig keyframes (752x480 pinhole,
                   baseline 0.11 m, right camera as a rig extrinsic);
  pose_only        one free camera against fixed 2D-3D matches with outliers.

Every generator is deterministic in its seed.  Noise model: pixel noise
N(0, sigma), a fraction of outliers displaced uniformly within +-50 px,
poses perturbed by rotation_noise rad / translation_noise m, points by
point_noise m.
"""

from __future__ import annotations

import math

import numpy as np

from .problem import SE3, Camera, CameraModel, PackedProblem

# ------------------------------------------------------------ vector algebra


def quat_to_matrix_v(q):
    """(N,4) (w,i,j,k) -> (N,3,3)."""
    w, i, j, k = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    return np.stack(
        [
            np.stack([w * w + i * i - j * j - k * k, 2 * (i * j - w * k), 2 * (w * j + i * k)], -1),
            np.stack([2 * (w * k + i * j), w * w - i * i + j * j - k * k, 2 * (j * k - w * i)], -1),
            np.stack([2 * (i * k - w * j), 2 * (w * i + j * k), w * w - i * i - j * j + k * k], -1),
        ],
        1,
    )


def matrix_to_quat_v(r):
    """(N,3,3) rotation -> (N,4) unit quaternion (w,i,j,k), w >= 0."""
    n = r.shape[0]
    q = np.empty((n, 4))
    tr = r[:, 0, 0] + r[:, 1, 1] + r[:, 2, 2]
    for idx in range(n):
        m = r[idx]
        t = tr[idx]
        if t > 0:
            s = math.sqrt(t + 1.0) * 2
            q[idx] = [0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s,
                      (m[1, 0] - m[0, 1]) / s]
        elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
            s = math.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2
            q[idx] = [(m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s,
                      (m[0, 2] + m[2, 0]) / s]
        elif m[1, 1] > m[2, 2]:
            s = math.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2
            q[idx] = [(m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s,
                      (m[1, 2] + m[2, 1]) / s]
        else:
            s = math.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2
            q[idx] = [(m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s,
                      (m[1, 2] + m[2, 1]) / s, 0.25 * s]
    q *= np.where(q[:, :1] < 0, -1.0, 1.0)
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def axis_angle_quat_v(v):
    """(N,3) rotation vectors -> (N,4) quaternions."""
    th = np.linalg.norm(v, axis=1, keepdims=True)
    s = np.where(th > 1e-12, np.sin(th / 2) / np.maximum(th, 1e-300), 0.5)
    return np.concatenate([np.cos(th / 2), v * s], 1)


def quat_mul_v(a, b):
    aw, ai, aj, ak = a.T
    bw, bi, bj, bk = b.T
    return np.stack(
        [aw * bw - ai * bi - aj * bj - ak * bk, aw * bi + ai * bw + aj * bk - ak * bj,
         aw * bj - ai * bk + aj * bw + ak * bi, aw * bk + ai * bj - aj * bi + ak * bw], 1)


def look_at(centers, targets, up=(0.0, 1.0, 0.0)):
    """World->camera rotations (N,3,3) of cameras at `centers` looking at
    `targets` (+z forward, +y down in the image)."""
    f = targets - centers
    f /= np.linalg.norm(f, axis=1, keepdims=True)
    up = np.broadcast_to(np.asarray(up, dtype=np.float64), f.shape)
    x = np.cross(-up, f)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(f, x)
    return np.stack([x, y, f], 1)  # rows: camera axes in world coordinates


def project_v(r, t, X, cam):
    """Project world points X (N,3) through poses (R (N,3,3), t (N,3)) with
    intrinsics cam = (fx, fy, cx, cy, k1, k2): Camera::project."""
    xc = np.einsum("nij,nj->ni", r, X) + t
    z = xc[:, 2]
    x = xc[:, 0] / z
    y = xc[:, 1] / z
    fx, fy, cx, cy, k1, k2 = [np.broadcast_to(np.asarray(c, dtype=np.float64), z.shape)
                              for c in cam]
    r2 = x * x + y * y
    d = 1.0 + k1 * r2 + k2 * r2 * r2
    return np.stack([fx * (x * d) + cx, fy * (y * d) + cy], 1), z


def _perturb(rng, q, t, rot_noise, trans_noise):
    """Pose noise about each camera's own centre: a rotation of N(0,
    rot_noise) per axis and a centre offset of N(0, trans_noise) per axis
    (perturbing t directly would swing far-off cameras about the origin)."""
    n = q.shape[0]
    dq = axis_angle_quat_v(rng.normal(0.0, rot_noise, (n, 3)))
    q1 = quat_mul_v(q, dq)
    c = -np.einsum("nji,nj->ni", quat_to_matrix_v(q), t)
    c1 = c + rng.normal(0.0, trans_noise, (n, 3))
    return q1, -np.einsum("nij,nj->ni", quat_to_matrix_v(q1), c1)


def _measure(rng, uv, sigma, outlier_fraction):
    uv = uv + rng.normal(0.0, sigma, uv.shape)
    out = rng.random(uv.shape[0]) < outlier_fraction
    uv[out] += rng.uniform(-50.0, 50.0, (int(out.sum()), 2))
    return uv


# ------------------------------------------------------------------ problems


def ring_problem(num_cameras=50, num_points=5000, seed=0, *, radius=15.0, cube=10.0,
                 width=640, height=480, focal=(500.0, 800.0), k1=(-0.05, 0.05),
                 per_camera_intrinsics=True, track=("uniform", 2, 8), sigma=1.0,
                 outlier_fraction=0.02, rotation_noise=0.01, translation_noise=0.05,
                 point_noise=0.05, fixed=(0, 1), height_jitter=1.0):
    """Cameras on a ring of `radius` around points uniform in a cube.

    track: ("uniform", lo, hi) draws each point's view count from U{lo..hi};
           ("geometric", mean, lo, hi) from a geometric law clipped to [lo, hi].
    Each point is observed by that many distinct cameras drawn uniformly among
    the cameras in which it is visible (in front and inside the image)."""
    rng = np.random.default_rng(seed)
    ang = 2.0 * np.pi * np.arange(num_cameras) / num_cameras
    centers = np.stack([radius * np.cos(ang), rng.uniform(-height_jitter, height_jitter,
                                                          num_cameras), radius * np.sin(ang)], 1)
    r_true = look_at(centers, np.zeros_like(centers) + rng.normal(0, 0.3, centers.shape))
    t_true = -np.einsum("nij,nj->ni", r_true, centers)
    q_true = matrix_to_quat_v(r_true)
    if per_camera_intrinsics:
        f = rng.uniform(focal[0], focal[1], num_cameras)
        kk = rng.uniform(k1[0], k1[1], num_cameras)
    else:
        f = np.full(num_cameras, float(np.mean(focal)))
        kk = np.full(num_cameras, float(np.mean(k1)))
    cx, cy = width / 2.0, height / 2.0
    X = rng.uniform(-cube / 2, cube / 2, (num_points, 3))

    # Track lengths.
    if track[0] == "uniform":
        T = rng.integers(track[1], track[2] + 1, num_points)
    else:
        mean, lo, hi = track[1], track[2], track[3]
        T = np.clip(rng.geometric(1.0 / mean, num_points), lo, hi)
    T = np.minimum(T, num_cameras)

    # Candidate cameras: sample with replacement, keep visible distinct ones.
    obs_cam_list = []
    obs_pt_list = []
    chunk = 65536
    for p0 in range(0, num_points, chunk):
        p1 = min(num_points, p0 + chunk)
        npts = p1 - p0
        tmax = int(T[p0:p1].max())
        k = min(num_cameras, 2 * tmax + 4)
        cand = rng.integers(0, num_cameras, (npts, k))
        cand = np.sort(cand, axis=1)
        dup = np.zeros_like(cand, dtype=bool)
        dup[:, 1:] = cand[:, 1:] == cand[:, :-1]
        # Visibility of each candidate.
        pts = np.repeat(X[p0:p1], k, axis=0)
        cc = cand.reshape(-1)
        cam_p = (f[cc], f[cc], np.full(cc.shape, cx), np.full(cc.shape, cy), kk[cc],
                 np.zeros(cc.shape))
        uv, z = project_v(r_true[cc], t_true[cc], pts, cam_p)
        vis = (z > 0.1) & (uv[:, 0] >= 0) & (uv[:, 0] < width) & (uv[:, 1] >= 0) & (uv[:, 1] < height)
        ok = vis.reshape(npts, k) & ~dup
        # Random order among the visible candidates, take the first T.
        key = rng.random((npts, k)) + np.where(ok, 0.0, 2.0)
        order = np.argsort(key, axis=1)
        taken = np.take_along_axis(ok, order, 1) & (np.arange(k)[None, :] < T[p0:p1, None])
        cams = np.take_along_axis(cand, order, 1)
        rows, cols = np.nonzero(taken)
        obs_pt_list.append(rows + p0)
        obs_cam_list.append(cams[rows, cols])
    obs_pt = np.concatenate(obs_pt_list).astype(np.uint32)
    obs_pose = np.concatenate(obs_cam_list).astype(np.uint32)
    cam_p = (f[obs_pose], f[obs_pose], np.full(obs_pose.shape, cx), np.full(obs_pose.shape, cy),
             kk[obs_pose], np.zeros(obs_pose.shape))
    uv, _ = project_v(r_true[obs_pose], t_true[obs_pose], X[obs_pt], cam_p)
    uv = _measure(rng, uv, sigma, outlier_fraction)

    q0, t0 = _perturb(rng, q_true, t_true, rotation_noise, translation_noise)
    pose_fixed = np.zeros(num_cameras, np.uint8)
    for i in fixed:
        if i < num_cameras:
            pose_fixed[i] = 1
            q0[i], t0[i] = q_true[i], t_true[i]
    X0 = X + rng.normal(0.0, point_noise, X.shape)
    if per_camera_intrinsics:
        cameras = [Camera(CameraModel.SIMPLE_RADIAL, width, height, [f[i], cx, cy, kk[i]])
                   for i in range(num_cameras)]
        obs_camera = obs_pose.copy()
    else:
        cameras = [Camera(CameraModel.SIMPLE_RADIAL, width, height, [f[0], cx, cy, kk[0]])
                   if kk[0] != 0.0 else Camera.pinhole(width, height, f[0], f[0], cx, cy)]
        obs_camera = None
    packed = PackedProblem(q0, t0, X0, obs_pose, obs_pt, uv, cameras, pose_fixed,
                           np.zeros(num_points, np.uint8), obs_camera)
    packed.truth = dict(pose_q=q_true, pose_t=t_true, points=X, centers=centers)
    return packed


def large_ring_problem(num_cameras=1200, num_points=500_000, seed=2000):
    """The 1,200-camera / 500k-point / ~4M-observation ring: shared pinhole
    intrinsics on 6000x4000 images, track length geometric with mean 8 clipped
    to [2, 60], cameras 0 and 1 fixed."""
    return ring_problem(num_cameras, num_points, seed, radius=20.0, cube=10.0, width=6000,
                        height=4000, focal=(4500.0, 4500.0), k1=(0.0, 0.0),
                        per_camera_intrinsics=False, track=("geometric", 8.0, 2, 60))


def stereo_window(num_keyframes=20, num_points=2000, seed=0, *, baseline=0.11,
                  width=752, height=480, f=458.0, obs_per_point=(3, 12), fixed_fraction=0.1,
                  sigma=1.0, outlier_fraction=0.02, rotation_noise=0.01,
                  translation_noise=0.05, point_noise=0.05):
    """A local BA window of stereo keyframes moving forward along +z.  Each
    keyframe pose is the left camera (T_left<-world); the right camera is a rig
    observation with sensor_from_rig = (I, (-baseline, 0, 0))."""
    rng = np.random.default_rng(seed)
    n = num_keyframes
    cx, cy = width / 2.0, height / 2.0
    s = np.arange(n) * 0.35
    centers = np.stack([0.3 * np.sin(s / 3.0), rng.normal(0, 0.02, n), s], 1)
    yaw = 0.05 * np.sin(s / 2.0)
    rv = np.stack([np.zeros(n), yaw, np.zeros(n)], 1)
    q_true = axis_angle_quat_v(rv)
    q_true[:, 1:] *= -1  # world->camera is the inverse rotation of the camera's
    r_true = quat_to_matrix_v(q_true)
    t_true = -np.einsum("nij,nj->ni", r_true, centers)
    # Points in front of the trajectory.
    X = np.stack([rng.uniform(-6, 6, num_points), rng.uniform(-3, 3, num_points),
                  rng.uniform(3, 25, num_points) + s.max() * rng.random(num_points)], 1)
    ext_t = np.array([-baseline, 0.0, 0.0])
    # Candidate sensors: 2n (kf, side); each point takes U{lo..hi} of the
    # sensors that see it, in random order (points seen by fewer than two
    # sensors stay unobserved).
    kf = np.repeat(np.arange(n), 2)
    side = np.tile([0, 1], n)
    lo, hi = obs_per_point
    want = rng.integers(lo, hi + 1, num_points)
    ts = t_true[kf] + np.where(side[:, None] == 1, ext_t, 0.0)
    xc = np.einsum("sij,mj->msi", r_true[kf], X) + ts[None]
    z = xc[..., 2]
    u = f * xc[..., 0] / np.maximum(z, 1e-9) + cx
    v = f * xc[..., 1] / np.maximum(z, 1e-9) + cy
    vis = (z > 0.5) & (u >= 0) & (u < width) & (v >= 0) & (v < height)
    nvis = vis.sum(1)
    take = np.where(nvis >= 2, np.minimum(want, nvis), 0)
    order = np.argsort(rng.random(vis.shape) + np.where(vis, 0.0, 2.0), axis=1)
    rows, cols = np.nonzero(np.arange(2 * n)[None, :] < take[:, None])
    sensor = order[rows, cols]
    obs_pose = kf[sensor].astype(np.uint32)
    obs_side = side[sensor].astype(np.uint32)
    obs_pt = rows.astype(np.uint32)
    xc = np.einsum("nij,nj->ni", r_true[obs_pose], X[obs_pt]) + t_true[obs_pose]
    xc = xc + np.where(obs_side[:, None] == 1, ext_t, 0.0)
    uv = np.stack([f * xc[:, 0] / xc[:, 2] + cx, f * xc[:, 1] / xc[:, 2] + cy], 1)
    uv = _measure(rng, uv, sigma, outlier_fraction)
    q0, t0 = _perturb(rng, q_true, t_true, rotation_noise, translation_noise)
    pose_fixed = np.zeros(n, np.uint8)
    nfix = max(1, int(round(fixed_fraction * n)))
    pose_fixed[:nfix] = 1
    q0[:nfix], t0[:nfix] = q_true[:nfix], t_true[:nfix]
    X0 = X + rng.normal(0.0, point_noise, X.shape)
    cam = Camera.pinhole(width, height, f, f, cx, cy)
    cameras = [(cam, SE3()), (cam, SE3((1.0, 0.0, 0.0, 0.0), tuple(ext_t)))]
    packed = PackedProblem(q0, t0, X0, obs_pose, obs_pt, uv, cameras, pose_fixed,
                           np.zeros(num_points, np.uint8), obs_side)
    packed.truth = dict(pose_q=q_true, pose_t=t_true, points=X, centers=centers)
    return packed


def street_loop(num_cameras=5600, num_points=3_000_000, seed=3000, *, spacing=1.0,
                width=1920, height=1080, f=1000.0, street_half_width=8.0, facade_jitter=0.2,
                facade_height=(0.5, 12.0), track=(6.7, 2, 40), sigma=1.0, outlier_fraction=0.02,
                rotation_noise=0.01, translation_noise=0.05, point_noise=0.05, fixed=(0, 1)):
    """Forward-facing cameras along a closed circular street loop, points on
    the facade planes on both sides (normal jitter +-facade_jitter).  Each
    point is seen by a run of consecutive cameras (track length geometric,
    mean track[0], clipped to [track[1], track[2]]) drawn among the cameras
    that have it in view ahead of them."""
    rng = np.random.default_rng(seed)
    n = num_cameras
    perim = n * spacing
    radius = perim / (2.0 * np.pi)
    ang = 2.0 * np.pi * np.arange(n) / n
    centers = np.stack([radius * np.cos(ang), np.full(n, 1.6), radius * np.sin(ang)], 1)
    fwd = np.stack([-np.sin(ang), np.zeros(n), np.cos(ang)], 1)  # tangent (direction of travel)
    r_true = look_at(centers, centers + fwd)
    t_true = -np.einsum("nij,nj->ni", r_true, centers)
    q_true = matrix_to_quat_v(r_true)
    cx, cy = width / 2.0, height / 2.0
    # Points: arc position, side, height; radial offset = facade +- jitter.
    s_arc = rng.uniform(0.0, perim, num_points)
    side = np.where(rng.random(num_points) < 0.5, -1.0, 1.0)
    h = rng.uniform(facade_height[0], facade_height[1], num_points)
    rad = radius + side * (street_half_width + rng.normal(0.0, facade_jitter, num_points))
    pa = s_arc / radius
    X = np.stack([rad * np.cos(pa), h, rad * np.sin(pa)], 1)
    # Cameras with the point in view lie behind it along the loop, from about
    # d_min (facade at the image edge) to d_max metres.
    half_fov = np.arctan(cx / f)
    d_min = (street_half_width + 1.0) / np.tan(half_fov)
    d_max = 45.0
    lo_cam = np.floor((s_arc - d_max) / spacing).astype(np.int64)
    hi_cam = np.floor((s_arc - d_min) / spacing).astype(np.int64)
    avail = hi_cam - lo_cam + 1
    mean, tlo, thi = track
    T = np.clip(rng.geometric(1.0 / mean, num_points), tlo, thi)
    T = np.minimum(T, avail)
    start = lo_cam + (rng.random(num_points) * (avail - T + 1)).astype(np.int64)
    obs_pt = np.repeat(np.arange(num_points, dtype=np.int64), T)
    first = np.repeat(np.cumsum(T) - T, T)
    obs_cam = (np.repeat(start, T) + (np.arange(obs_pt.size) - first)) % n
    # Keep the observations that project inside the image in front.
    keep = np.zeros(obs_pt.size, bool)
    uv = np.zeros((obs_pt.size, 2))
    chunk = 1 << 22
    for a in range(0, obs_pt.size, chunk):
        b = min(obs_pt.size, a + chunk)
        ci, pi = obs_cam[a:b], obs_pt[a:b]
        xc = np.einsum("nij,nj->ni", r_true[ci], X[pi]) + t_true[ci]
        z = xc[:, 2]
        u = f * xc[:, 0] / np.maximum(z, 1e-9) + cx
        v = f * xc[:, 1] / np.maximum(z, 1e-9) + cy
        keep[a:b] = (z > 0.5) & (u >= 0) & (u < width) & (v >= 0) & (v < height)
        uv[a:b, 0], uv[a:b, 1] = u, v
    # Points left with fewer than two observations drop out of the problem.
    cnt = np.bincount(obs_pt[keep], minlength=num_points)
    keep &= cnt[obs_pt] >= 2
    obs_pt, obs_cam, uv = obs_pt[keep], obs_cam[keep], uv[keep]
    used = np.zeros(num_points, bool)
    used[obs_pt] = True
    remap = np.cumsum(used) - 1
    X = X[used]
    obs_pt = remap[obs_pt]
    uv = _measure(rng, uv, sigma, outlier_fraction)
    q0, t0 = _perturb(rng, q_true, t_true, rotation_noise, translation_noise)
    pose_fixed = np.zeros(n, np.uint8)
    for i in fixed:
        pose_fixed[i] = 1
        q0[i], t0[i] = q_true[i], t_true[i]
    X0 = X + rng.normal(0.0, point_noise, X.shape)
    cam = Camera.pinhole(width, height, f, f, cx, cy)
    packed = PackedProblem(q0, t0, X0, obs_cam.astype(np.uint32), obs_pt.astype(np.uint32), uv,
                           [cam], pose_fixed, np.zeros(X.shape[0], np.uint8), None)
    packed.truth = dict(pose_q=q_true, pose_t=t_true, points=X, centers=centers)
    return packed


def sub_problem(packed: PackedProblem, cameras) -> PackedProblem:
    """The part of a problem seen by a set of poses: those poses, their
    observations, and the landmarks they observe at least twice (the first
    selected pose fixed, as in the whole problem's gauge)."""
    cams = np.asarray(sorted(set(int(c) for c in cameras)), dtype=np.int64)
    pose_map = np.full(packed.num_poses, -1, np.int64)
    pose_map[cams] = np.arange(cams.size)
    sel = pose_map[packed.obs_pose] >= 0
    cnt = np.bincount(packed.obs_landmark[sel], minlength=packed.num_landmarks)
    sel &= cnt[packed.obs_landmark] >= 2
    used = np.zeros(packed.num_landmarks, bool)
    used[packed.obs_landmark[sel]] = True
    lm_map = np.cumsum(used) - 1
    fixed = np.zeros(cams.size, np.uint8)
    fixed[0] = 1
    lf = None if packed.landmark_fixed is None else packed.landmark_fixed[used]
    oc = None if packed.obs_camera is None else packed.obs_camera[sel]
    return PackedProblem(packed.pose_q[cams], packed.pose_t[cams], packed.landmarks[used],
                         pose_map[packed.obs_pose[sel]], lm_map[packed.obs_landmark[sel]],
                         packed.obs_xy[sel], packed.cameras, fixed, lf, oc)


def window_batch(num_windows=512, seed=4000, *, keyframes=(5, 40), points=(200, 5000)):
    """Uneven local BA windows: each a stereo window of U{5..40} keyframes
    and U{200..5000} points (3-12 observations per point, 10% of the poses
    fixed as anchors), seeded per window."""
    rng = np.random.default_rng(seed)
    nk = rng.integers(keyframes[0], keyframes[1] + 1, num_windows)
    npt = rng.integers(points[0], points[1] + 1, num_windows)
    return [stereo_window(int(nk[w]), int(npt[w]), seed=seed + 1 + w) for w in range(num_windows)]


def pose_only(num_matches=500, seed=0, *, width=752, height=480, f=458.0,
              outlier_fraction=0.3, sigma=1.0, rotation_noise=0.02, translation_noise=0.1):
    """One free camera refined against fixed landmarks (2D-3D matches)."""
    rng = np.random.default_rng(seed)
    cx, cy = width / 2.0, height / 2.0
    # Points visible from the identity camera.
    z = rng.uniform(2.0, 20.0, num_matches)
    u = rng.uniform(0, width, num_matches)
    v = rng.uniform(0, height, num_matches)
    X = np.stack([(u - cx) / f * z, (v - cy) / f * z, z], 1)
    q_true = np.array([[1.0, 0.0, 0.0, 0.0]])
    t_true = np.zeros((1, 3))
    uv = np.stack([u, v], 1)
    uv = uv + rng.normal(0.0, sigma, uv.shape)
    out = rng.random(num_matches) < outlier_fraction
    uv[out] = np.stack([rng.uniform(0, width, int(out.sum())),
                        rng.uniform(0, height, int(out.sum()))], 1)
    q0, t0 = _perturb(rng, q_true, t_true, rotation_noise, translation_noise)
    cam = Camera.pinhole(width, height, f, f, cx, cy)
    packed = PackedProblem(q0, t0, X, np.zeros(num_matches, np.uint32),
                           np.arange(num_matches, dtype=np.uint32), uv, [cam],
                           np.zeros(1, np.uint8), np.ones(num_matches, np.uint8))
    packed.truth = dict(pose_q=q_true, pose_t=t_true, points=X, centers=np.zeros((1, 3)))
    return packed


def scene_extent(packed: PackedProblem) -> float:
    """Diagonal of the bounding box of the camera centres and points."""
    pts = np.concatenate([packed.camera_centers(), packed.landmarks], 0)
    return float(np.linalg.norm(pts.max(0) - pts.min(0)))


# ------------------------------------------------------ reduced camera systems
def covisibility_system(n=5822, band=450, cross=150, laplacian=False):
    """A reduced camera system shaped like a city block revisited in four
    passes (the shape of the reference's dense_covisibility_system test
    fixture, rig_ba_solver.rs:5158-5196, widened to a SmallCity-sized
    system): every node couples to its `band` capture-order neighbours on
    each side (weight 1) and to `cross` nodes of the other passes at the same
    place (weight 0.5); block entries ((7 r + 3 c + lo + hi) mod 11) 1e-3 w.
    The diagonal is 10 + (i mod 5) plus node i's off-diagonal absolute row
    sums times the identity, so the system is diagonally dominant SPD.
    With laplacian=True the same graph carries the reference's chain_system
    values instead (rig_ba_solver.rs:5244-5272): blocks -w I, w = 1 +
    ((7 a + 3 b) mod 5) / 10, and the diagonal the weights' sum plus damping
    1e-4 (1 + (i + r) mod 3), an ill-conditioned system whose solves run
    hundreds of iterations.
    Returns (diag (n,6,6), edges (e,2) sorted, offdiag (e,6,6) float32);
    n=5822, band 450, cross 150 gives about 3.4M edges."""
    q = n // 4
    i = np.arange(n, dtype=np.int64)
    a = np.repeat(i, band)
    b = a + np.tile(np.arange(1, band + 1, dtype=np.int64), n)
    keep = b < n
    band_keys = a[keep] * n + b[keep]
    ii = np.repeat(i, cross)
    kk = np.tile(np.arange(cross, dtype=np.int64), n)
    other = ((ii // q + 1 + kk % 3) % 4) * q + (ii % q + kk // 3) % q
    lo, hi = np.minimum(ii, other), np.maximum(ii, other)
    cross_keys = np.unique((lo * n + hi)[lo != hi])
    keys = np.union1d(band_keys, cross_keys)
    w = np.where(np.isin(keys, cross_keys, assume_unique=True), 0.5, 1.0).astype(np.float32)
    lo, hi = keys // n, keys % n
    if laplacian:
        wl = 1.0 + ((lo * 7 + hi * 3) % 5) * 0.1
        off = np.zeros((len(keys), 6, 6), np.float32)
        for rr in range(6):
            off[:, rr, rr] = -wl
        wsum = np.bincount(lo, wl, minlength=n) + np.bincount(hi, wl, minlength=n)
        damp = 1e-4 * (1 + (i[:, None] + np.arange(6)[None, :]) % 3)
        diag = np.zeros((n, 6, 6))
        diag[:, np.arange(6), np.arange(6)] = wsum[:, None] + damp
        return diag, np.stack([lo, hi], 1).astype(np.uint32), off
    r = np.arange(6)[:, None]
    c = np.arange(6)[None, :]
    off = np.empty((len(keys), 6, 6), np.float32)
    s = (lo + hi).astype(np.int64)
    for rr in range(6):
        for cc in range(6):
            off[:, rr, cc] = ((rr * 7 + cc * 3 + s) % 11) * 1e-3 * w
    rowsum = np.abs(off).sum(axis=2).max(axis=1).astype(np.float64)
    dom = np.bincount(lo, rowsum, minlength=n) + np.bincount(hi, rowsum, minlength=n)
    diag = (10.0 + (i % 5) + dom)[:, None, None] * np.eye(6)
    del r, c
    return diag, np.stack([lo, hi], 1).astype(np.uint32), off


def street_elimination(n=5822, obs_per_frame=2500, seed=0, chunk=1 << 20):
    """A point elimination shaped like a long street capture (the reference's
    street_scene benchmark, rig_ba_solver.rs:5322-5340): n frames along a
    line, each point seen by consecutive frames with heavy-tailed track
    lengths (95% 3-15 frames, 5% 40-120), about `obs_per_frame` observations
    per frame.  Each observation has a random Jacobian [A (3x6) | B (3x3)];
    hcp = A^T B, V_p = I + sum B^T B over its observations, and the damped
    diagonal of the reduced system U - sum hcp V^-1 hcp^T, U = I + sum A^T A
    (a Schur complement of an SPD matrix, so SPD).  Returns a dict with
    edges, point_off, point_nodes, hcp (K,6,3), point_inverse (P,3,3), diag
    (n,6,6) and rhs (n,6)."""
    rng = np.random.default_rng(seed)
    mean_len = 0.95 * 9.0 + 0.05 * 80.0
    npts = int(n * obs_per_frame / mean_len)
    long = rng.random(npts) < 0.05
    length = np.where(long, rng.integers(40, 121, npts), rng.integers(3, 16, npts))
    length = np.minimum(length, n)
    start = rng.integers(0, n - length + 1)
    point_off = np.zeros(npts + 1, np.uint64)
    np.cumsum(length, out=point_off[1:])
    nobs = int(point_off[-1])
    pidx = np.repeat(np.arange(npts), length)
    point_nodes = (start[pidx] + np.arange(nobs) - point_off[:-1][pidx].astype(np.int64)
                   ).astype(np.uint32)
    hcp = np.empty((nobs, 6, 3))
    btb = np.empty((nobs, 3, 3))
    ata = np.zeros((n, 6, 6))
    for o0 in range(0, nobs, chunk):
        o1 = min(nobs, o0 + chunk)
        A = rng.standard_normal((o1 - o0, 3, 6))
        B = rng.standard_normal((o1 - o0, 3, 3))
        hcp[o0:o1] = np.einsum("oji,ojk->oik", A, B)
        btb[o0:o1] = np.einsum("oji,ojk->oik", B, B)
        g = np.einsum("oji,ojk->oik", A, A).reshape(-1, 36)
        nodes = point_nodes[o0:o1]
        for q in range(36):
            ata.reshape(n, 36)[:, q] += np.bincount(nodes, g[:, q], minlength=n)
    V = np.add.reduceat(btb, point_off[:-1].astype(np.int64), axis=0) + np.eye(3)
    del btb
    vinv = np.linalg.inv(V)
    wvw = np.zeros((n, 36))
    for o0 in range(0, nobs, chunk):
        o1 = min(nobs, o0 + chunk)
        h = hcp[o0:o1]
        t = np.einsum("oij,ojk,olk->oil", h, vinv[pidx[o0:o1]], h).reshape(-1, 36)
        nodes = point_nodes[o0:o1]
        for q in range(36):
            wvw[:, q] += np.bincount(nodes, t[:, q], minlength=n)
    diag = ata + np.eye(6) - wvw.reshape(n, 6, 6)
    ends = start + length - 1
    reach = np.full(n, -1, np.int64)
    np.maximum.at(reach, start, ends)
    reach = np.maximum.accumulate(reach)
    cnt = np.maximum(reach - np.arange(n), 0)
    s = np.repeat(np.arange(n), cnt)
    t = s + 1 + (np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt))
    edges = np.stack([s, t], 1).astype(np.uint32)
    rhs = rng.standard_normal((n, 6))
    return {"edges": edges, "point_off": point_off, "point_nodes": point_nodes, "hcp": hcp,
            "point_inverse": vinv, "diag": diag, "rhs": rhs}
