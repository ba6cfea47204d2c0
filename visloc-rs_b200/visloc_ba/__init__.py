"""visloc_ba: B200 bundle-adjustment solver (host side).

The solver itself is the CUDA library libvisloc_ba_cuda.so built from
../csrc; this package mirrors the reference's BA API (problem.py) and binds
the library's C ABI (_abi.py, solver.py).
"""

from .problem import (  # noqa: F401
    AUTO_SCALE_K,
    SE3,
    BaConfig,
    BaError,
    BaGncResult,
    BaIterationStats,
    BaObservation,
    BaResult,
    BaGeneralStereoObservation,
    BaRigObservation,
    BaStereoObservation,
    BaScope,
    BundleAdjustment,
    Camera,
    CameraModel,
    GncConfig,
    PackedProblem,
    Pose,
    RobustKernel,
    quat_from_axis_angle,
)
