"""ctypes mirror of include/visloc_ba_cuda.h (the solver's C ABI).

The structures below are laid out field for field as in the header; the
loaders bind every exported entry point with its prototype, so a missing
symbol fails at load time rather than at the first call.
"""

from __future__ import annotations

import ctypes as C
import os

ABI_VERSION = 4

# enum vlba_status
OK = 0
DECLINED = 1
ERR_NO_POSES = 2
ERR_NO_LANDMARKS = 3
ERR_NO_OBSERVATIONS = 4
ERR_ALL_POSES_FIXED = 5
ERR_MISSING_POSE = 6
ERR_MISSING_LANDMARK = 7
ERR_UNSUPPORTED_CAMERA_MODEL = 8
ERR_SINGULAR_SYSTEM = 9
ERR_INVALID_ARGUMENT = 10
ERR_CUDA = 11
ERR_OUT_OF_MEMORY = 12
ERR_TIMEOUT = 13
ERR_BUSY = 14
ERR_INVALID_OBSERVATION_WEIGHT = 15
ERR_MISSING_STEREO_BASELINE = 16

STATUS_NAMES = {
    OK: "OK",
    DECLINED: "DECLINED",
    ERR_NO_POSES: "NoPoses",
    ERR_NO_LANDMARKS: "NoLandmarks",
    ERR_NO_OBSERVATIONS: "NoObservations",
    ERR_ALL_POSES_FIXED: "AllPosesFixed",
    ERR_MISSING_POSE: "MissingPose",
    ERR_MISSING_LANDMARK: "MissingLandmark",
    ERR_UNSUPPORTED_CAMERA_MODEL: "UnsupportedCameraModel",
    ERR_SINGULAR_SYSTEM: "SingularSystem",
    ERR_INVALID_ARGUMENT: "InvalidArgument",
    ERR_CUDA: "CudaError",
    ERR_OUT_OF_MEMORY: "OutOfMemory",
    ERR_TIMEOUT: "Timeout",
    ERR_BUSY: "Busy",
    ERR_INVALID_OBSERVATION_WEIGHT: "InvalidObservationWeight",
    ERR_MISSING_STEREO_BASELINE: "MissingStereoBaseline",
}

# vlba_problem.obs_kind
OBS_MONO = 0
OBS_STEREO = 1
OBS_GENERAL_STEREO = 2

# enum vlba_camera_model
CAMERA_PINHOLE = 0
CAMERA_SIMPLE_PINHOLE = 1
CAMERA_SIMPLE_RADIAL = 2
CAMERA_RADIAL = 3
CAMERA_OPENCV = 4
CAMERA_OTHER = 255

# enum vlba_robust_kernel
KERNEL_NONE = 0
KERNEL_HUBER = 1
KERNEL_CAUCHY = 2

FLAG_PROFILE = 1
FLAG_GRAPH = 2
FLAG_AUTOTUNE = 4

# enum vlba_gnc_kernel
GNC_GEMAN_MCCLURE = 0
GNC_TRUNCATED_LEAST_SQUARES = 1


class Camera(C.Structure):
    _fields_ = [
        ("model", C.c_uint32),
        ("num_params", C.c_uint32),
        ("params", C.c_double * 8),
        ("sensor_from_rig_q", C.c_double * 4),
        ("sensor_from_rig_t", C.c_double * 3),
    ]


class Problem(C.Structure):
    _fields_ = [
        ("num_poses", C.c_uint64),
        ("num_landmarks", C.c_uint64),
        ("num_observations", C.c_uint64),
        ("pose_q", C.POINTER(C.c_double)),
        ("pose_t", C.POINTER(C.c_double)),
        ("pose_fixed", C.POINTER(C.c_uint8)),
        ("landmarks", C.POINTER(C.c_double)),
        ("landmark_fixed", C.POINTER(C.c_uint8)),
        ("obs_pose", C.POINTER(C.c_uint32)),
        ("obs_landmark", C.POINTER(C.c_uint32)),
        ("obs_xy", C.POINTER(C.c_double)),
        ("obs_camera", C.POINTER(C.c_uint32)),
        ("num_cameras", C.c_uint32),
        ("cameras", C.POINTER(Camera)),
        ("obs_weight", C.POINTER(C.c_double)),
        ("obs_kind", C.POINTER(C.c_uint8)),
        ("obs_stereo", C.POINTER(C.c_double)),
        ("obs_right_camera", C.POINTER(C.c_uint32)),
        ("stereo_baseline", C.c_double),
    ]


class Config(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_uint32),
        ("has_initial_lambda", C.c_uint32),
        ("initial_lambda", C.c_double),
        ("lambda_increase_factor", C.c_double),
        ("lambda_decrease_factor", C.c_double),
        ("max_lambda", C.c_double),
        ("min_lambda", C.c_double),
        ("step_tolerance", C.c_double),
        ("cost_tolerance", C.c_double),
        ("has_relative_cost_tolerance", C.c_uint32),
        ("robust_kernel", C.c_uint32),
        ("relative_cost_tolerance", C.c_double),
        ("robust_parameter", C.c_double),
        ("max_pcg_iterations", C.c_uint32),
        ("flags", C.c_uint32),
        ("pcg_relative_tolerance", C.c_double),
        ("refine_intrinsics", C.c_uint32),
        ("refine_distortion", C.c_uint32),
        ("refine_tangential_distortion", C.c_uint32),
        ("shared_focal", C.c_uint32),
        ("reserved", C.c_uint32 * 4),
    ]


class Iteration(C.Structure):
    _fields_ = [
        ("iteration", C.c_uint64),
        ("cost_before", C.c_double),
        ("cost_after", C.c_double),
        ("max_pose_step", C.c_double),
        ("max_landmark_step", C.c_double),
        ("lambda_", C.c_double),
        ("step_accepted", C.c_uint32),
        ("pcg_iterations", C.c_uint32),
        ("pcg_relative_residual", C.c_double),
        ("linearize_ms", C.c_double),
        ("assemble_ms", C.c_double),
        ("pcg_ms", C.c_double),
        ("update_ms", C.c_double),
    ]


class Result(C.Structure):
    _fields_ = [
        ("initial_cost", C.c_double),
        ("final_cost", C.c_double),
        ("converged", C.c_uint32),
        ("num_iterations", C.c_uint32),
        ("initial_nonprojectable", C.c_uint64),
        ("final_nonprojectable", C.c_uint64),
        ("total_pcg_iterations", C.c_uint64),
        ("error_index", C.c_uint64),
        ("device_ms", C.c_double),
        ("upload_ms", C.c_double),
        ("kernel_launches", C.c_uint64),
        ("upload_bytes", C.c_uint64),
    ]


class PlanInfo(C.Structure):
    _fields_ = [
        ("variable_cameras", C.c_uint64),
        ("variable_landmarks", C.c_uint64),
        ("variable_observations", C.c_uint64),
        ("camera_pairs", C.c_uint64),
        ("schur_terms", C.c_uint64),
        ("tile_size", C.c_uint32),
        ("tile_rows", C.c_uint32),
        ("tiles", C.c_uint32),
        ("assembly_lanes", C.c_uint32),
        ("device_bytes", C.c_uint64),
        ("upload_bytes", C.c_uint64),
        ("bytes_per_iteration", C.c_double),
        ("bytes_per_pcg_iteration", C.c_double),
    ]


P = C.POINTER
# name -> (restype, argtypes): every symbol include/visloc_ba_cuda.h declares.
class ReducedSystem(C.Structure):
    _fields_ = [
        ("num_nodes", C.c_uint32),
        ("reserved", C.c_uint32),
        ("num_edges", C.c_uint64),
        ("diag", C.POINTER(C.c_double)),
        ("edges", C.POINTER(C.c_uint32)),
        ("offdiag", C.POINTER(C.c_float)),
        ("rhs", C.POINTER(C.c_double)),
        ("tol", C.c_double),
        ("max_iterations", C.c_uint32),
        ("reserved2", C.c_uint32),
    ]


class PointElimination(C.Structure):
    _fields_ = [
        ("structure_id", C.c_uint64),
        ("linearization_id", C.c_uint64),
        ("num_nodes", C.c_uint32),
        ("num_points", C.c_uint32),
        ("num_edges", C.c_uint64),
        ("edges", C.POINTER(C.c_uint32)),
        ("point_off", C.POINTER(C.c_uint64)),
        ("point_nodes", C.POINTER(C.c_uint32)),
        ("hcp", C.POINTER(C.c_double)),
        ("point_inverse", C.POINTER(C.c_double)),
        ("point_used", C.POINTER(C.c_uint8)),
        ("num_extra", C.c_uint64),
        ("extra_edge", C.POINTER(C.c_uint32)),
        ("extra_block", C.POINTER(C.c_double)),
        ("num_run_edges", C.c_uint64),
        ("run_edges", C.POINTER(C.c_uint32)),
        ("coarse_group", C.c_uint32),
        ("coarse_nodes", C.c_uint32),
    ]


class ReducedTiming(C.Structure):
    _fields_ = [
        ("fill_ms", C.c_double),
        ("pcg_ms", C.c_double),
        ("eliminate_ms", C.c_double),
        ("reserved", C.c_double),
    ]


class ReducedPreconditioner(C.Structure):
    _fields_ = [
        ("num_clusters", C.c_uint32),
        ("reserved", C.c_uint32),
        ("cluster_first", C.POINTER(C.c_uint32)),
        ("cluster_size", C.POINTER(C.c_uint32)),
        ("cluster_inverse", C.POINTER(C.c_double)),
        ("coarse_group", C.c_uint32),
        ("coarse_nodes", C.c_uint32),
        ("coarse_inverse", C.POINTER(C.c_double)),
    ]


class LaunchShape(C.Structure):
    _fields_ = [
        ("pcg_blocks", C.c_int32),
        ("reserved", C.c_int32),
        ("l2_resident_fraction", C.c_double),
        ("pcg_iteration_us", C.c_double),
    ]


class TicketInfo(C.Structure):
    _fields_ = [
        ("latency_ms", C.c_double),
        ("queue_ms", C.c_double),
        ("solve_ms", C.c_double),
        ("batch_size", C.c_uint32),
        ("slot", C.c_uint32),
    ]


class GncConfig(C.Structure):
    _fields_ = [
        ("kernel", C.c_uint32),
        ("max_outer", C.c_uint32),
        ("inner_iterations", C.c_uint32),
        ("has_auto_scale", C.c_uint32),
        ("c", C.c_double),
        ("anneal_factor", C.c_double),
        ("auto_scale", C.c_double),
        ("auto_scale_readapt", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class GncResult(C.Structure):
    _fields_ = [
        ("initial_cost", C.c_double),
        ("final_cost", C.c_double),
        ("inlier_cost", C.c_double),
        ("inlier_scale", C.c_double),
        ("observation_count", C.c_uint64),
        ("outer_iterations", C.c_uint32),
        ("converged", C.c_uint32),
        ("lm_iterations", C.c_uint64),
        ("device_ms", C.c_double),
    ]


SOLVER_EXPORTS = {
    "visloc_ba_cuda_abi_version": (C.c_uint32, []),
    "visloc_ba_cuda_default_config": (None, [P(Config)]),
    "visloc_ba_cuda_create": (C.c_void_p, [C.c_int]),
    "visloc_ba_cuda_destroy": (None, [C.c_void_p]),
    "visloc_ba_cuda_last_error": (C.c_char_p, [C.c_void_p]),
    "visloc_ba_cuda_check": (C.c_int, [P(Problem), P(Config), P(C.c_uint64)]),
    "visloc_ba_cuda_optimize": (
        C.c_int,
        [C.c_void_p, P(Problem), P(Config), P(Result), P(Iteration), C.c_uint32],
    ),
    "visloc_ba_cuda_upload": (C.c_int, [C.c_void_p, P(Problem), P(Config)]),
    "visloc_ba_cuda_solve_uploaded": (
        C.c_int,
        [C.c_void_p, P(Config), P(Result), P(Iteration), C.c_uint32],
    ),
    "visloc_ba_cuda_download": (C.c_int, [C.c_void_p, P(Problem)]),
    "visloc_ba_cuda_plan": (C.c_int, [P(Problem), P(Config), C.c_double, P(PlanInfo)]),
    "visloc_ba_cuda_linear_step": (
        C.c_int,
        [C.c_void_p, P(Problem), P(Config), C.c_double, P(C.c_double), P(C.c_double),
         P(C.c_uint32), P(C.c_double)],
    ),
    "visloc_ba_cuda_reduced_system": (
        C.c_int,
        [C.c_void_p, P(Problem), P(Config), C.c_double, P(C.c_double), P(C.c_double)],
    ),
    "visloc_ba_cuda_cost": (
        C.c_int,
        [C.c_void_p, P(Problem), P(Config), P(C.c_double), P(C.c_uint64)],
    ),
    "visloc_ba_cuda_batch_optimize": (
        C.c_int,
        [C.c_void_p, C.c_uint32, P(P(Problem)), P(P(Config)), P(C.c_int), P(Result),
         P(Iteration), C.c_uint32],
    ),
    "visloc_ba_cuda_batch_upload": (
        C.c_int, [C.c_void_p, C.c_uint32, P(P(Problem)), P(P(Config)), P(C.c_int)],
    ),
    "visloc_ba_cuda_batch_solve_uploaded": (
        C.c_int, [C.c_void_p, P(Result), P(Iteration), C.c_uint32],
    ),
    "visloc_ba_cuda_batch_download": (C.c_int, [C.c_void_p, C.c_uint32, P(P(Problem))]),
    "visloc_ba_cuda_reduced_solve": (
        C.c_int, [C.c_void_p, P(ReducedSystem), P(C.c_double), P(C.c_uint32), P(C.c_double)],
    ),
    "visloc_ba_cuda_reduced_timing": (C.c_int, [C.c_void_p, P(ReducedTiming)]),
    "visloc_ba_cuda_reduced_eliminate": (
        C.c_int, [C.c_void_p, P(PointElimination), P(C.c_double), P(C.c_double)],
    ),
    "visloc_ba_cuda_reduced_solve_preconditioned": (
        C.c_int, [C.c_void_p, P(ReducedSystem), P(ReducedPreconditioner), P(C.c_double),
                  P(C.c_uint32), P(C.c_double)],
    ),
    "visloc_ba_cuda_autotune": (C.c_int, [C.c_void_p, P(LaunchShape)]),
    "visloc_ba_cuda_wait_probe": (C.c_int, [C.c_void_p, C.c_double, P(C.c_double)]),
    "visloc_ba_cuda_set_launch_shape": (C.c_int, [C.c_void_p, P(LaunchShape)]),
    "visloc_ba_cuda_server_create": (C.c_void_p, [C.c_int, C.c_uint32, C.c_uint64, C.c_uint32]),
    "visloc_ba_cuda_server_destroy": (None, [C.c_void_p]),
    "visloc_ba_cuda_server_submit": (
        C.c_int, [C.c_void_p, P(Problem), P(Config), P(C.c_uint64)],
    ),
    "visloc_ba_cuda_server_wait": (
        C.c_int,
        [C.c_void_p, C.c_uint64, C.c_double, P(Result), P(Iteration), C.c_uint32,
         P(TicketInfo)],
    ),
    "visloc_ba_cuda_server_last_error": (C.c_char_p, [C.c_void_p]),
    # Device pointers for the problem arrays and both outputs; see the header.
    "visloc_ba_cuda_cost_noalloc": (
        C.c_int,
        [P(Problem), P(Config), C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t],
    ),
    "visloc_ba_cuda_default_gnc_config": (None, [P(GncConfig)]),
    "visloc_ba_cuda_optimize_gnc": (
        C.c_int,
        [C.c_void_p, P(Problem), P(Config), P(GncConfig), P(GncResult), P(C.c_double)],
    ),
}

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBRARY_NAME = "libvisloc_ba_cuda.so"


def library_path() -> str:
    """In-tree location of the built CUDA library (next to this package)."""
    return os.path.join(PACKAGE_DIR, LIBRARY_NAME)


def bind(lib: C.CDLL, exports: dict) -> C.CDLL:
    for name, (restype, argtypes) in exports.items():
        fn = getattr(lib, name)  # AttributeError if the symbol is missing
        fn.restype = restype
        fn.argtypes = argtypes
    return lib


_LIB = None


def load_solver_library(path: str | None = None) -> C.CDLL:
    """Load libvisloc_ba_cuda.so (raises OSError if it was not built)."""
    global _LIB
    if path is None and _LIB is not None:
        return _LIB
    p = path or library_path()
    if not os.path.exists(p):
        raise OSError(
            f"{p} is missing: build the CUDA library first "
            "(python __graft_entry__.py build, or make -C visloc-rs_b200)"
        )
    lib = bind(C.CDLL(p), SOLVER_EXPORTS)
    if lib.visloc_ba_cuda_abi_version() != ABI_VERSION:
        raise OSError(f"{p}: ABI version mismatch")
    if path is None:
        _LIB = lib
    return lib
