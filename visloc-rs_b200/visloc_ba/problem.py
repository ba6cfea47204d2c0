"""Host-side mirror of the reference's bundle-adjustment API.

These are the types the reference's BA entry point takes and returns
(pipelines/slam/src/bundle/mod.rs):

  BundleAdjustment   mod.rs:530-622 (add_*/fix_* at problem.rs:186-233)
  BaObservation      mod.rs:194-199
  BaRigObservation   mod.rs:245-251
  BaConfig           mod.rs:626-752 (defaults :729-752)
  BaIterationStats   mod.rs:755-763
  BaResult           mod.rs:765-771
  BaError            mod.rs:1022-1056
  RobustKernel       pipelines/slam/src/pose_graph.rs:87-138
  Camera             crates/core/src/types/camera.rs:99-105
  Pose / SE3         crates/core/src/geometry/pose.rs:4-46, se3.rs:4-121

Ids are u64 keys kept in dicts; packing maps them to dense indices in
ascending id order (the BTreeMap order the reference iterates in), exactly as
GpuBundleAdjuster::upload does (crates/ba-gpu/src/solver.rs:256-314).
"""

from __future__ import annotations

import ctypes as C
import enum
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _abi


# ----------------------------------------------------------------- geometry
def quat_mul(a, b):
    """Hamilton product of (w, i, j, k) quaternions."""
    aw, ai, aj, ak = a
    bw, bi, bj, bk = b
    return (
        aw * bw - ai * bi - aj * bj - ak * bk,
        aw * bi + ai * bw + aj * bk - ak * bj,
        aw * bj - ai * bk + aj * bw + ak * bi,
        aw * bk + ai * bj - aj * bi + ak * bw,
    )


def quat_rotate(q, p):
    """nalgebra's UnitQuaternion * Vector3: t = 2 (v x p); p + w t + v x t."""
    w, vx, vy, vz = q
    px, py, pz = p
    tx = 2.0 * (vy * pz - vz * py)
    ty = 2.0 * (vz * px - vx * pz)
    tz = 2.0 * (vx * py - vy * px)
    cx = vy * tz - vz * ty
    cy = vz * tx - vx * tz
    cz = vx * ty - vy * tx
    return (tx * w + cx + px, ty * w + cy + py, tz * w + cz + pz)


def quat_from_axis_angle(axis, angle):
    n = math.sqrt(sum(a * a for a in axis))
    s = math.sin(angle / 2.0) / n
    return (math.cos(angle / 2.0), axis[0] * s, axis[1] * s, axis[2] * s)


def quat_to_matrix(q):
    w, i, j, k = q
    ww, ii, jj, kk = w * w, i * i, j * j, k * k
    ij, wk, wj = i * j * 2.0, w * k * 2.0, w * j * 2.0
    ik, jk, wi = i * k * 2.0, j * k * 2.0, w * i * 2.0
    return np.array(
        [
            [ww + ii - jj - kk, ij - wk, wj + ik],
            [wk + ij, ww - ii + jj - kk, jk - wi],
            [ik - wj, wi + jk, ww - ii - jj + kk],
        ]
    )


@dataclass
class SE3:
    """Rigid transform: unit quaternion (w, i, j, k) and translation."""

    rotation: tuple = (1.0, 0.0, 0.0, 0.0)
    translation: tuple = (0.0, 0.0, 0.0)

    def transform_point(self, p):
        r = quat_rotate(self.rotation, p)
        return (r[0] + self.translation[0], r[1] + self.translation[1], r[2] + self.translation[2])

    def inverse(self) -> "SE3":
        w, i, j, k = self.rotation
        qi = (w, -i, -j, -k)
        t = quat_rotate(qi, self.translation)
        return SE3(qi, (-t[0], -t[1], -t[2]))

    def compose(self, other: "SE3") -> "SE3":
        r = quat_rotate(self.rotation, other.translation)
        return SE3(
            quat_mul(self.rotation, other.rotation),
            (r[0] + self.translation[0], r[1] + self.translation[1], r[2] + self.translation[2]),
        )


@dataclass
class Pose:
    """Pose::world_to_camera (core/geometry/pose.rs:4-7)."""

    world_to_camera: SE3 = field(default_factory=SE3)

    @staticmethod
    def from_world_to_camera(rotation, translation) -> "Pose":
        return Pose(SE3(tuple(rotation), tuple(translation)))

    def transform_world_point(self, p):
        return self.world_to_camera.transform_point(p)

    def camera_center_world(self):
        return self.world_to_camera.inverse().translation


# ------------------------------------------------------------------ cameras
class CameraModel(enum.IntEnum):
    PINHOLE = _abi.CAMERA_PINHOLE
    SIMPLE_PINHOLE = _abi.CAMERA_SIMPLE_PINHOLE
    SIMPLE_RADIAL = _abi.CAMERA_SIMPLE_RADIAL
    RADIAL = _abi.CAMERA_RADIAL
    OPENCV = _abi.CAMERA_OPENCV
    OTHER = _abi.CAMERA_OTHER


@dataclass
class Camera:
    """Camera { model, width, height, params } (camera.rs:99-105)."""

    model: CameraModel
    width: int
    height: int
    params: list

    @staticmethod
    def pinhole(width, height, fx, fy, cx, cy) -> "Camera":
        return Camera(CameraModel.PINHOLE, width, height, [fx, fy, cx, cy])

    @staticmethod
    def pinhole_radial(width, height, fx, fy, cx, cy, k1, k2) -> "Camera":
        return Camera(CameraModel.PINHOLE, width, height, [fx, fy, cx, cy, k1, k2])

    @staticmethod
    def simple_radial(width, height, f, cx, cy, k1) -> "Camera":
        return Camera(CameraModel.SIMPLE_RADIAL, width, height, [f, cx, cy, k1])

    def to_abi(self, sensor_from_rig: Optional[SE3] = None) -> _abi.Camera:
        c = _abi.Camera()
        c.model = int(self.model)
        if len(self.params) > 8:
            raise ValueError("at most 8 camera parameters")
        c.num_params = len(self.params)
        for i, v in enumerate(self.params):
            c.params[i] = float(v)
        t = sensor_from_rig or SE3()
        for i in range(4):
            c.sensor_from_rig_q[i] = float(t.rotation[i])
        for i in range(3):
            c.sensor_from_rig_t[i] = float(t.translation[i])
        return c


# -------------------------------------------------------- observations etc.
@dataclass
class BaObservation:
    keyframe_id: int
    landmark_id: int
    xy: tuple


@dataclass
class BaRigObservation:
    keyframe_id: int
    landmark_id: int
    xy: tuple
    camera: Camera
    sensor_from_rig: SE3 = field(default_factory=SE3)


@dataclass
class BaStereoObservation:
    """BaStereoObservation (mod.rs:213-221): rectified stereo, the right
    row taken equal to the left one."""

    keyframe_id: int
    landmark_id: int
    xy: tuple
    u_right: float


@dataclass
class BaGeneralStereoObservation:
    """BaGeneralStereoObservation (mod.rs:223-237): calibrated stereo with
    T_right<-left = left_to_right."""

    keyframe_id: int
    landmark_id: int
    xy_left: tuple
    xy_right: tuple
    right_camera: Camera
    left_to_right: SE3 = field(default_factory=SE3)


@dataclass(frozen=True)
class RobustKernel:
    """RobustKernel::{None, Huber{delta}, Cauchy{c}} (pose_graph.rs:87-101)."""

    kind: int = _abi.KERNEL_NONE
    parameter: float = 0.0

    @staticmethod
    def none() -> "RobustKernel":
        return RobustKernel(_abi.KERNEL_NONE, 0.0)

    @staticmethod
    def huber(delta: float) -> "RobustKernel":
        return RobustKernel(_abi.KERNEL_HUBER, float(delta))

    @staticmethod
    def cauchy(c: float) -> "RobustKernel":
        return RobustKernel(_abi.KERNEL_CAUCHY, float(c))

    def cost(self, s: float) -> float:
        if self.kind == _abi.KERNEL_HUBER:
            d = self.parameter
            return s if s <= d * d else 2.0 * d * math.sqrt(s) - d * d
        if self.kind == _abi.KERNEL_CAUCHY:
            c2 = self.parameter * self.parameter
            return c2 * math.log(1.0 + s / c2)
        return s

    def weight(self, s: float) -> float:
        if self.kind == _abi.KERNEL_HUBER:
            d = self.parameter
            return 1.0 if s <= d * d else d / math.sqrt(s)
        if self.kind == _abi.KERNEL_CAUCHY:
            c2 = self.parameter * self.parameter
            return 1.0 / (1.0 + s / c2)
        return 1.0


@dataclass
class BaConfig:
    """BaConfig with the reference defaults (mod.rs:729-752) plus the PCG
    controls of GpuBaSettings (crates/ba-gpu/src/solver.rs:36-50)."""

    max_iterations: int = 20
    initial_lambda: Optional[float] = 1e-4
    lambda_increase_factor: float = 10.0
    lambda_decrease_factor: float = 0.1
    max_lambda: float = 1e12
    min_lambda: float = 1e-9
    step_tolerance: float = 1e-7
    cost_tolerance: float = 1e-9
    relative_cost_tolerance: Optional[float] = None
    robust_kernel: RobustKernel = field(default_factory=RobustKernel.none)
    max_pcg_iterations: int = 100
    pcg_relative_tolerance: float = 1e-4
    profile: bool = False
    # Run the LM loop as one captured CUDA graph (VLBA_FLAG_GRAPH).
    graph: bool = False
    # Choose the launch shape before the first solve of an upload.
    autotune: bool = False
    # Joint self-calibration (mod.rs:669-700).  The device solver holds the
    # intrinsics fixed, so any of these makes it decline (the caller's CPU
    # solver runs instead), as GpuBundleAdjuster::check does for
    # refine_intrinsics / refine_distortion (crates/ba-gpu/src/solver.rs:214-216).
    refine_intrinsics: bool = False
    refine_distortion: bool = False
    refine_tangential_distortion: bool = False
    shared_focal: bool = False

    def to_abi(self) -> _abi.Config:
        c = _abi.Config()
        c.max_iterations = int(self.max_iterations)
        c.has_initial_lambda = 0 if self.initial_lambda is None else 1
        c.initial_lambda = 0.0 if self.initial_lambda is None else float(self.initial_lambda)
        c.lambda_increase_factor = self.lambda_increase_factor
        c.lambda_decrease_factor = self.lambda_decrease_factor
        c.max_lambda = self.max_lambda
        c.min_lambda = self.min_lambda
        c.step_tolerance = self.step_tolerance
        c.cost_tolerance = self.cost_tolerance
        c.has_relative_cost_tolerance = 0 if self.relative_cost_tolerance is None else 1
        c.relative_cost_tolerance = (
            0.0 if self.relative_cost_tolerance is None else float(self.relative_cost_tolerance)
        )
        c.robust_kernel = int(self.robust_kernel.kind)
        c.robust_parameter = float(self.robust_kernel.parameter)
        c.max_pcg_iterations = int(self.max_pcg_iterations)
        c.pcg_relative_tolerance = float(self.pcg_relative_tolerance)
        c.flags = ((_abi.FLAG_PROFILE if self.profile else 0) | (_abi.FLAG_GRAPH if self.graph else 0)
                   | (_abi.FLAG_AUTOTUNE if self.autotune else 0))
        c.refine_intrinsics = int(bool(self.refine_intrinsics))
        c.refine_distortion = int(bool(self.refine_distortion))
        c.refine_tangential_distortion = int(bool(self.refine_tangential_distortion))
        c.shared_focal = int(bool(self.shared_focal))
        return c


@dataclass
class GncConfig:
    """GncConfig (pipelines/slam/src/gnc.rs:50-110) with its defaults."""

    kernel: int = _abi.GNC_GEMAN_MCCLURE
    c: float = 1.0
    anneal_factor: float = 1.4
    max_outer: int = 100
    inner_iterations: int = 5
    auto_scale: Optional[float] = None
    auto_scale_readapt: bool = False

    def to_abi(self) -> _abi.GncConfig:
        g = _abi.GncConfig()
        g.kernel = int(self.kernel)
        g.max_outer = int(self.max_outer)
        g.inner_iterations = int(self.inner_iterations)
        g.has_auto_scale = 0 if self.auto_scale is None else 1
        g.c = float(self.c)
        g.anneal_factor = float(self.anneal_factor)
        g.auto_scale = 0.0 if self.auto_scale is None else float(self.auto_scale)
        g.auto_scale_readapt = 1 if self.auto_scale_readapt else 0
        return g


# GncConfig::auto_scale's recommended k (gnc.rs:92-96).
AUTO_SCALE_K = 3.5


@dataclass
class BaGncResult:
    """BaGncResult (bundle/mod.rs:975-1000)."""

    initial_cost: float
    final_cost: float
    inlier_cost: float
    inlier_scale: float
    observation_count: int
    outer_iterations: int
    converged: bool
    observation_weights: "np.ndarray"
    lm_iterations: int = 0
    device_ms: float = 0.0


@dataclass
class BaIterationStats:
    iteration: int
    cost_before: float
    cost_after: float
    max_pose_step: float
    max_landmark_step: float
    lambda_: float
    step_accepted: bool
    pcg_iterations: int = 0
    pcg_relative_residual: float = 0.0
    linearize_ms: float = 0.0
    assemble_ms: float = 0.0
    pcg_ms: float = 0.0
    update_ms: float = 0.0


@dataclass
class BaResult:
    initial_cost: float
    final_cost: float
    iterations: list
    converged: bool
    initial_nonprojectable: int = 0
    final_nonprojectable: int = 0
    total_pcg_iterations: int = 0
    device_ms: float = 0.0
    upload_ms: float = 0.0
    kernel_launches: int = 0
    upload_bytes: int = 0


class BaError(Exception):
    """BaError (mod.rs:1022-1056); `kind` is the variant name, `id` the
    offending pose/landmark id for MissingPose / MissingLandmark."""

    def __init__(self, kind: str, id: Optional[int] = None, message: str = ""):
        self.kind = kind
        self.id = id
        super().__init__(f"{kind}{'' if id is None else f'({id})'} {message}".strip())

    def __eq__(self, other):
        return isinstance(other, BaError) and (self.kind, self.id) == (other.kind, other.id)

    def __hash__(self):
        return hash((self.kind, self.id))


class BaScope(enum.Enum):
    GLOBAL = "global"
    LOCAL = "local"


def result_from_abi(res: _abi.Result, iters, count: int) -> BaResult:
    out = []
    for k in range(min(count, len(iters) if iters is not None else 0)):
        it = iters[k]
        out.append(
            BaIterationStats(
                int(it.iteration),
                it.cost_before,
                it.cost_after,
                it.max_pose_step,
                it.max_landmark_step,
                it.lambda_,
                bool(it.step_accepted),
                int(it.pcg_iterations),
                it.pcg_relative_residual,
                it.linearize_ms,
                it.assemble_ms,
                it.pcg_ms,
                it.update_ms,
            )
        )
    return BaResult(
        res.initial_cost,
        res.final_cost,
        out,
        bool(res.converged),
        int(res.initial_nonprojectable),
        int(res.final_nonprojectable),
        int(res.total_pcg_iterations),
        res.device_ms,
        res.upload_ms,
        int(res.kernel_launches),
        int(res.upload_bytes),
    )


# ------------------------------------------------------------ packed form
def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return C.POINTER(ctype)()
    return a.ctypes.data_as(C.POINTER(ctype))


class PackedProblem:
    """A problem as dense numpy arrays, the layout the C ABI takes.

    pose_q (N,4) f64 (w,i,j,k), pose_t (N,3), pose_fixed (N,) u8,
    landmarks (M,3), landmark_fixed (M,) u8, obs_pose / obs_landmark (K,) u32,
    obs_xy (K,2) f64, obs_camera (K,) u32 or None, cameras: list of
    (Camera, SE3 sensor_from_rig), obs_weight (K,) f64 external weights or
    None (all 1; optimize_with_observation_weights, optimize.rs:43-53);
    stereo observations: obs_kind (K,) u8 (0 monocular/rig, 1 rectified,
    2 general stereo) or None, obs_stereo (K,2) f64 (u_r; the right pixel),
    obs_right_camera (K,) u32 into `cameras`, stereo_baseline."""

    def __init__(self, pose_q, pose_t, landmarks, obs_pose, obs_landmark, obs_xy, cameras,
                 pose_fixed=None, landmark_fixed=None, obs_camera=None, obs_weight=None,
                 obs_kind=None, obs_stereo=None, obs_right_camera=None, stereo_baseline=0.0):
        self.pose_q = np.ascontiguousarray(pose_q, dtype=np.float64).reshape(-1, 4)
        self.pose_t = np.ascontiguousarray(pose_t, dtype=np.float64).reshape(-1, 3)
        self.landmarks = np.ascontiguousarray(landmarks, dtype=np.float64).reshape(-1, 3)
        self.obs_pose = np.ascontiguousarray(obs_pose, dtype=np.uint32).reshape(-1)
        self.obs_landmark = np.ascontiguousarray(obs_landmark, dtype=np.uint32).reshape(-1)
        self.obs_xy = np.ascontiguousarray(obs_xy, dtype=np.float64).reshape(-1, 2)
        self.pose_fixed = (
            None if pose_fixed is None else np.ascontiguousarray(pose_fixed, dtype=np.uint8)
        )
        self.landmark_fixed = (
            None
            if landmark_fixed is None
            else np.ascontiguousarray(landmark_fixed, dtype=np.uint8)
        )
        self.obs_camera = (
            None if obs_camera is None else np.ascontiguousarray(obs_camera, dtype=np.uint32)
        )
        self.cameras = [c if isinstance(c, tuple) else (c, SE3()) for c in cameras]
        self.obs_weight = (
            None if obs_weight is None else np.ascontiguousarray(obs_weight, dtype=np.float64)
        )
        self.obs_kind = None if obs_kind is None else np.ascontiguousarray(obs_kind, dtype=np.uint8)
        self.obs_stereo = (
            None if obs_stereo is None
            else np.ascontiguousarray(obs_stereo, dtype=np.float64).reshape(-1, 2)
        )
        self.obs_right_camera = (
            None if obs_right_camera is None
            else np.ascontiguousarray(obs_right_camera, dtype=np.uint32)
        )
        self.stereo_baseline = float(stereo_baseline)
        self._abi = None

    @property
    def num_poses(self):
        return self.pose_q.shape[0]

    @property
    def num_landmarks(self):
        return self.landmarks.shape[0]

    @property
    def num_observations(self):
        return self.obs_pose.shape[0]

    def copy(self) -> "PackedProblem":
        return PackedProblem(
            self.pose_q.copy(), self.pose_t.copy(), self.landmarks.copy(), self.obs_pose,
            self.obs_landmark, self.obs_xy, list(self.cameras), self.pose_fixed,
            self.landmark_fixed, self.obs_camera, self.obs_weight, self.obs_kind, self.obs_stereo,
            self.obs_right_camera, self.stereo_baseline,
        )

    def abi(self) -> _abi.Problem:
        """ctypes view of the arrays (the arrays stay owned by this object)."""
        p = _abi.Problem()
        p.num_poses = self.num_poses
        p.num_landmarks = self.num_landmarks
        p.num_observations = self.num_observations
        p.pose_q = _ptr(self.pose_q, C.c_double)
        p.pose_t = _ptr(self.pose_t, C.c_double)
        p.pose_fixed = _ptr(self.pose_fixed, C.c_uint8)
        p.landmarks = _ptr(self.landmarks, C.c_double)
        p.landmark_fixed = _ptr(self.landmark_fixed, C.c_uint8)
        p.obs_pose = _ptr(self.obs_pose, C.c_uint32)
        p.obs_landmark = _ptr(self.obs_landmark, C.c_uint32)
        p.obs_xy = _ptr(self.obs_xy, C.c_double)
        p.obs_camera = _ptr(self.obs_camera, C.c_uint32)
        p.obs_weight = _ptr(self.obs_weight, C.c_double)
        p.obs_kind = _ptr(self.obs_kind, C.c_uint8)
        p.obs_stereo = _ptr(self.obs_stereo, C.c_double)
        p.obs_right_camera = _ptr(self.obs_right_camera, C.c_uint32)
        p.stereo_baseline = self.stereo_baseline
        cams = (_abi.Camera * len(self.cameras))(
            *[cam.to_abi(ext) for cam, ext in self.cameras]
        )
        p.num_cameras = len(self.cameras)
        p.cameras = C.cast(cams, C.POINTER(_abi.Camera))
        self._abi = (p, cams)  # keep the camera array alive
        return p

    def camera_centers(self) -> np.ndarray:
        """World camera centres -R^T t of every pose (N,3)."""
        out = np.empty((self.num_poses, 3))
        for i in range(self.num_poses):
            r = quat_to_matrix(self.pose_q[i])
            out[i] = -r.T @ self.pose_t[i]
        return out


# ------------------------------------------------------- BundleAdjustment
class BundleAdjustment:
    """The reference's BundleAdjustment (mod.rs:530-622) for monocular and
    rig observations."""

    def __init__(self, camera: Camera):
        self.poses: dict[int, Pose] = {}
        self.landmarks: dict[int, tuple] = {}
        self.observations: list[BaObservation] = []
        self.stereo_observations: list[BaStereoObservation] = []
        self.general_stereo_observations: list[BaGeneralStereoObservation] = []
        self.rig_observations: list[BaRigObservation] = []
        self.stereo_baseline: Optional[float] = None
        self.camera = camera
        self.fixed_poses: set[int] = set()
        self.fixed_landmarks: set[int] = set()
        # Terms of the reference problem that this solver does not model
        # (mod.rs:530-622): rotation-fixed poses, priors and the inertial
        # state.  They are carried so that the accelerator can decline a
        # problem that holds any of them, as GpuBundleAdjuster::check does
        # (crates/ba-gpu/src/solver.rs:230-246); the device never sees them.
        self.fixed_pose_rotations: set[int] = set()
        self.gravity_prior = None
        self.per_pose_gravity_prior = None
        self.position_prior = None
        self.pairwise_pose_factors: list = []
        self.velocities: dict = {}
        self.imu_factors: list = []
        self.biases: dict = {}
        self.bias_random_walk_factors: list = []
        self.navigation_state_prior = None

    def unsupported_terms(self) -> Optional[str]:
        """The first term of the problem this solver does not model, in the
        order GpuBundleAdjuster::check tests them (solver.rs:230-246), or
        None."""
        if (self.gravity_prior is not None or self.per_pose_gravity_prior is not None
                or self.position_prior is not None or self.pairwise_pose_factors
                or self.velocities or self.imu_factors or self.biases
                or self.bias_random_walk_factors or self.navigation_state_prior is not None):
            return "prior/inertial terms"
        if self.fixed_pose_rotations:
            return "rotation-fixed poses"
        return None

    # problem.rs:186-233
    def add_pose(self, id: int, pose: Pose):
        self.poses[id] = pose

    def fix_pose(self, id: int):
        self.fixed_poses.add(id)

    def add_landmark(self, id: int, xyz):
        self.landmarks[id] = tuple(float(v) for v in xyz)

    def fix_landmark(self, id: int):
        self.fixed_landmarks.add(id)

    def add_observation(self, obs: BaObservation):
        self.observations.append(obs)

    def add_rig_observation(self, obs: BaRigObservation):
        self.rig_observations.append(obs)

    def add_stereo_observation(self, obs: BaStereoObservation):
        self.stereo_observations.append(obs)

    def add_general_stereo_observation(self, obs: BaGeneralStereoObservation):
        self.general_stereo_observations.append(obs)

    def set_stereo_baseline(self, baseline: float):
        self.stereo_baseline = float(baseline)

    def pack(self):
        """Dense arrays in ascending id order, plus the id lists and a
        validation error (BaError) for ids that do not resolve.  The
        observations are flattened in the reference's order -- monocular,
        rectified stereo, general stereo, rig (optimize.rs:30-35) -- which is
        also the order of external weights."""
        pose_ids = sorted(self.poses)
        lm_ids = sorted(self.landmarks)
        pose_at = {pid: i for i, pid in enumerate(pose_ids)}
        lm_at = {lid: i for i, lid in enumerate(lm_ids)}
        mono, rect, gen, rig = (self.observations, self.stereo_observations,
                                self.general_stereo_observations, self.rig_observations)
        k = len(mono) + len(rect) + len(gen) + len(rig)
        obs_pose = np.empty(k, np.uint32)
        obs_lm = np.empty(k, np.uint32)
        obs_xy = np.empty((k, 2))
        kinds = np.zeros(k, np.uint8)
        stereo = np.zeros((k, 2))
        right = np.zeros(k, np.uint32)
        obs_camera = np.zeros(k, np.uint32)
        # cameras[0] is BundleAdjustment::camera; rig sensors and right
        # cameras follow, each (camera, extrinsic) once.
        cams: list = [(self.camera, SE3())]
        keys: dict = {}

        def camera_index(camera, ext):
            key = (int(camera.model), tuple(camera.params), ext.rotation, ext.translation)
            if key not in keys:
                keys[key] = len(cams)
                cams.append((camera, ext))
            return keys[key]

        missing = None
        n = 0
        for group, kind in ((mono, _abi.OBS_MONO), (rect, _abi.OBS_STEREO),
                            (gen, _abi.OBS_GENERAL_STEREO), (rig, _abi.OBS_MONO)):
            for o in group:
                if o.keyframe_id not in pose_at:
                    missing = missing or BaError("MissingPose", o.keyframe_id)
                    obs_pose[n] = 0xFFFFFFFF
                else:
                    obs_pose[n] = pose_at[o.keyframe_id]
                if o.landmark_id not in lm_at:
                    if missing is None and o.keyframe_id in pose_at:
                        missing = BaError("MissingLandmark", o.landmark_id)
                    obs_lm[n] = 0xFFFFFFFF
                else:
                    obs_lm[n] = lm_at[o.landmark_id]
                kinds[n] = kind
                if group is gen:
                    obs_xy[n] = o.xy_left
                    stereo[n] = o.xy_right
                    right[n] = camera_index(o.right_camera, o.left_to_right)
                else:
                    obs_xy[n] = o.xy
                if group is rect:
                    stereo[n, 0] = o.u_right
                if group is rig:
                    obs_camera[n] = camera_index(o.camera, o.sensor_from_rig)
                n += 1
        pose_q = np.array([self.poses[i].world_to_camera.rotation for i in pose_ids],
                          dtype=np.float64).reshape(-1, 4)
        pose_t = np.array([self.poses[i].world_to_camera.translation for i in pose_ids],
                          dtype=np.float64).reshape(-1, 3)
        lms = np.array([self.landmarks[i] for i in lm_ids], dtype=np.float64).reshape(-1, 3)
        pf = np.array([1 if i in self.fixed_poses else 0 for i in pose_ids], np.uint8)
        lf = np.array([1 if i in self.fixed_landmarks else 0 for i in lm_ids], np.uint8)
        has_stereo = bool(rect) or bool(gen)
        packed = PackedProblem(
            pose_q, pose_t, lms, obs_pose, obs_lm, obs_xy, cams, pf, lf,
            obs_camera if rig else None, None,
            kinds if has_stereo else None, stereo if has_stereo else None,
            right if gen else None,
            self.stereo_baseline if self.stereo_baseline is not None else float("nan"),
        )
        return packed, pose_ids, lm_ids, missing

    def unpack(self, packed: PackedProblem, pose_ids, lm_ids):
        for i, pid in enumerate(pose_ids):
            self.poses[pid] = Pose(SE3(tuple(packed.pose_q[i]), tuple(packed.pose_t[i])))
        for i, lid in enumerate(lm_ids):
            self.landmarks[lid] = tuple(packed.landmarks[i])
