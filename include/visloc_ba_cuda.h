/*
 * visloc_ba_cuda.h -- C ABI of the B200 bundle-adjustment solver.
 *
 * This is the drop-in boundary for the reference's bundle-adjustment
 * accelerator plug-in:
 *
 *   trait BaAccelerator { fn optimize(&self, ba: &mut BundleAdjustment,
 *                                     config: &BaConfig, scope: BaScope)
 *                         -> Option<Result<BaResult, BaError>>; }
 *   (pipelines/slam/src/ba_accel.rs:23-32, registered with
 *    set_ba_accelerator, ba_accel.rs:38-40)
 *
 * The reference's own GPU implementation of that trait is GpuBundleAdjuster
 * (crates/ba-gpu/src/solver.rs:80-85, impl at :729-742).  The entry points
 * below follow the repository's native-library convention
 * (native/descriptor_gemm/descriptor_gemm.cu:101-193: versioned ABI, opaque
 * context, error string, int status with 0 = ok).
 *
 * Memory: the caller owns every array.  All calls are synchronous.  A context
 * is not thread-safe; use one context per thread (or serialise calls).
 *
 * Identifiers: the reference keys poses and landmarks by u64 ids in BTreeMaps.
 * This ABI takes dense indices; the host shim maps ids to indices in ascending
 * id order, as GpuBundleAdjuster::upload does (solver.rs:256-314).
 */
#ifndef VISLOC_BA_CUDA_H
#define VISLOC_BA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VLBA_ABI_VERSION 4u

/* ------------------------------------------------------------------ status */
/* Return codes.  The Rust shim maps VLBA_DECLINED to `None` (the caller then
 * runs the CPU solver) and the VLBA_ERR_* values that mirror BaError
 * (pipelines/slam/src/bundle/mod.rs:1022-1056) to `Some(Err(..))`. */
enum vlba_status {
  VLBA_OK = 0,
  VLBA_DECLINED = 1,                   /* outside what this solver implements */
  VLBA_ERR_NO_POSES = 2,               /* BaError::NoPoses */
  VLBA_ERR_NO_LANDMARKS = 3,           /* BaError::NoLandmarks */
  VLBA_ERR_NO_OBSERVATIONS = 4,        /* BaError::NoObservations */
  VLBA_ERR_ALL_POSES_FIXED = 5,        /* BaError::AllPosesFixed */
  VLBA_ERR_MISSING_POSE = 6,           /* BaError::MissingPose(id) */
  VLBA_ERR_MISSING_LANDMARK = 7,       /* BaError::MissingLandmark(id) */
  VLBA_ERR_UNSUPPORTED_CAMERA_MODEL = 8, /* BaError::UnsupportedCameraModel */
  VLBA_ERR_SINGULAR_SYSTEM = 9,        /* BaError::SingularSystem */
  VLBA_ERR_INVALID_ARGUMENT = 10,      /* null pointer, bad size or config */
  VLBA_ERR_CUDA = 11,                  /* a CUDA call failed */
  VLBA_ERR_OUT_OF_MEMORY = 12,         /* device memory exhausted */
  VLBA_ERR_TIMEOUT = 13,               /* a bounded device wait gave up */
  VLBA_ERR_BUSY = 14,                  /* server queue full / ticket pending */
  VLBA_ERR_INVALID_OBSERVATION_WEIGHT = 15, /* BaError::InvalidObservationWeight(index) */
  VLBA_ERR_MISSING_STEREO_BASELINE = 16  /* BaError::MissingStereoBaseline */
};

/* ------------------------------------------------------------------ camera */
/* The pinhole family whose Camera::project is the pinhole followed by radial
 * 1 + k1 r^2 + k2 r^4 (core/types/camera.rs:15-41, project at :351-432,
 * intrinsics at :243-260, radial_distortion at :213-227).  Parameter layouts
 * are the reference's (COLMAP) layouts:
 *   PINHOLE        [fx, fy, cx, cy (, k1 (, k2))]
 *   SIMPLE_PINHOLE [f, cx, cy]
 *   SIMPLE_RADIAL  [f, cx, cy, k1]
 *   RADIAL         [f, cx, cy, k1 (, k2)]
 *   OPENCV         [fx, fy, cx, cy, k1, k2, p1, p2] with p1 = p2 = 0
 * Other models (fisheye, FOV, double sphere, tangential OpenCV) make
 * visloc_ba_cuda_optimize return VLBA_DECLINED. */
enum vlba_camera_model {
  VLBA_CAMERA_PINHOLE = 0,
  VLBA_CAMERA_SIMPLE_PINHOLE = 1,
  VLBA_CAMERA_SIMPLE_RADIAL = 2,
  VLBA_CAMERA_RADIAL = 3,
  VLBA_CAMERA_OPENCV = 4,
  VLBA_CAMERA_OTHER = 255
};

typedef struct vlba_camera {
  uint32_t model;        /* enum vlba_camera_model */
  uint32_t num_params;   /* <= 8 */
  double params[8];
  /* Fixed rig extrinsic T_sensor<-rig of a BaRigObservation
   * (bundle/mod.rs:245-251).  Identity (1,0,0,0 / 0,0,0) for the monocular
   * BaObservation, whose pose is the camera's own T_camera<-world. */
  double sensor_from_rig_q[4]; /* w, i, j, k */
  double sensor_from_rig_t[3];
} vlba_camera;

/* ----------------------------------------------------------------- problem */
/* BundleAdjustment (bundle/mod.rs:530-622) restricted to the monocular and
 * rig observations.  Poses are T_world->camera (Pose::world_to_camera,
 * core/geometry/pose.rs:4-7): a unit quaternion (w, i, j, k) and a
 * translation.  pose_q, pose_t and landmarks are overwritten with the
 * optimised values on success, as the reference mutates `ba` in place. */
typedef struct vlba_problem {
  uint64_t num_poses;
  uint64_t num_landmarks;
  uint64_t num_observations;
  double* pose_q;                 /* [4 * num_poses] */
  double* pose_t;                 /* [3 * num_poses] */
  const uint8_t* pose_fixed;      /* [num_poses], nonzero = fixed; NULL = none */
  double* landmarks;              /* [3 * num_landmarks] */
  const uint8_t* landmark_fixed;  /* [num_landmarks]; NULL = none fixed */
  const uint32_t* obs_pose;       /* [num_observations] dense pose index */
  const uint32_t* obs_landmark;   /* [num_observations] dense landmark index */
  const double* obs_xy;           /* [2 * num_observations] pixel (u, v) */
  /* Per-observation camera index into `cameras`.  NULL: every observation
   * is a monocular BaObservation through cameras[0] (BundleAdjustment::camera).
   * Non-NULL: each observation is a BaRigObservation with its own camera and
   * sensor_from_rig. */
  const uint32_t* obs_camera;
  uint32_t num_cameras;
  const vlba_camera* cameras;
  /* External confidence weight per observation (ABI version 2), the
   * `observation_weights` of BundleAdjustment::optimize_with_observation_weights
   * (bundle/optimize.rs:43-53): it multiplies the robust-kernel IRLS weight in
   * the normal equations (normal_equations.rs:238,458) and each observation's
   * robust cost (problem.rs:497-560); 1 keeps the plain contribution, 0 drops
   * the residual.  Each must be finite and >= 0 (optimize.rs:628-650), else
   * VLBA_ERR_INVALID_OBSERVATION_WEIGHT with the observation's index.  NULL:
   * every weight is 1 (BundleAdjustment::optimize). */
  const double* obs_weight;
  /* Stereo observations (ABI version 3).  obs_kind[o] (NULL: every
   * observation is of kind 0):
   *   0  a monocular or rig observation as described above;
   *   1  BaStereoObservation (bundle/mod.rs:213-221), rectified stereo: left
   *      pixel obs_xy, observed right column u_r = obs_stereo[2o]; residual
   *      (u_l, v_l, u_r) with u_r predicted as u_l - fx stereo_baseline / z
   *      (normal_equations.rs:496-570);
   *   2  BaGeneralStereoObservation (mod.rs:223-237), calibrated stereo: left
   *      pixel obs_xy, right pixel (obs_stereo[2o], obs_stereo[2o+1]) through
   *      cameras[obs_right_camera[o]], whose sensor_from_rig is the rig
   *      transform T_right<-left (sqrt_qr.rs:465-518).
   * Kinds 1 and 2 project through cameras[0] (BundleAdjustment::camera) and
   * the right camera with their pinhole intrinsics, without distortion, as
   * the reference does; cameras[0] must then be PINHOLE or SIMPLE_PINHOLE
   * (check_stereo_camera_model, problem.rs:733-745). */
  const uint8_t* obs_kind;
  const double* obs_stereo;          /* [2 * num_observations] (kinds 1 and 2) */
  const uint32_t* obs_right_camera;  /* [num_observations] (kind 2) */
  double stereo_baseline;            /* BundleAdjustment::stereo_baseline; finite and > 0
                                        when an observation is of kind 1, else
                                        VLBA_ERR_MISSING_STEREO_BASELINE */
} vlba_problem;

/* ------------------------------------------------------------------ config */
enum vlba_robust_kernel {
  VLBA_KERNEL_NONE = 0,   /* RobustKernel::None */
  VLBA_KERNEL_HUBER = 1,  /* RobustKernel::Huber { delta } */
  VLBA_KERNEL_CAUCHY = 2  /* RobustKernel::Cauchy { c } */
};

/* BaConfig (bundle/mod.rs:626-752) plus the PCG controls of GpuBaSettings
 * (crates/ba-gpu/src/solver.rs:25-50).  visloc_ba_cuda_default_config fills
 * the reference's defaults (mod.rs:729-752). */
typedef struct vlba_config {
  uint32_t max_iterations;
  uint32_t has_initial_lambda;     /* 0 = None (pure Gauss-Newton) */
  double initial_lambda;
  double lambda_increase_factor;
  double lambda_decrease_factor;
  double max_lambda;
  double min_lambda;
  double step_tolerance;
  double cost_tolerance;
  uint32_t has_relative_cost_tolerance;
  uint32_t robust_kernel;          /* enum vlba_robust_kernel */
  double relative_cost_tolerance;
  double robust_parameter;         /* Huber delta or Cauchy c */
  uint32_t max_pcg_iterations;     /* per LM linear solve */
  uint32_t flags;                  /* VLBA_FLAG_* */
  double pcg_relative_tolerance;   /* stop once |r| <= tol |b| */
  /* Joint self-calibration switches of BaConfig (ABI version 4;
   * bundle/mod.rs:669-700).  This solver keeps the intrinsics fixed, so a
   * nonzero value in any of them makes every solving entry point return
   * VLBA_DECLINED before it looks at the problem, and the caller runs its
   * CPU solver -- the decline of GpuBundleAdjuster::check for
   * refine_intrinsics || refine_distortion (crates/ba-gpu/src/solver.rs:
   * 214-216).  refine_tangential_distortion and shared_focal only take
   * effect with refine_intrinsics in the reference (mod.rs:682-700) and are
   * declined here as well, so no config that could change the answer is
   * solved with the intrinsics held. */
  uint32_t refine_intrinsics;
  uint32_t refine_distortion;
  uint32_t refine_tangential_distortion;
  uint32_t shared_focal;
  uint32_t reserved[4];
} vlba_config;

/* Record per-iteration device phase times in vlba_iteration (costs a device
 * synchronisation per iteration; the analogue of VISLOC_BA_GPU_PROFILE,
 * solver.rs:571,622-628). */
#define VLBA_FLAG_PROFILE 1u

/* Run the initial cost and all max_iterations LM iterations as one CUDA graph,
 * captured at the first solve of an upload and replayed by later solves:
 * no host synchronisation between iterations (iterations after every problem
 * has finished cost only their launches).  Ignored with VLBA_FLAG_PROFILE. */
#define VLBA_FLAG_GRAPH 2u

/* Before the first solve of an upload, choose the launch shape (see
 * visloc_ba_cuda_autotune) unless one was tuned for a system of this shape
 * earlier in the process. */
#define VLBA_FLAG_AUTOTUNE 4u

/* ------------------------------------------------------------------ result */
/* BaIterationStats (bundle/mod.rs:755-763) plus solver diagnostics. */
typedef struct vlba_iteration {
  uint64_t iteration;
  double cost_before;
  double cost_after;
  double max_pose_step;
  double max_landmark_step;
  double lambda;
  uint32_t step_accepted;
  uint32_t pcg_iterations;
  double pcg_relative_residual;    /* |r| / |b| at PCG exit */
  /* Device time of the iteration's phases with VLBA_FLAG_PROFILE (else 0):
   * linearisation, reduced-system assembly, PCG, update + cost + decision. */
  double linearize_ms;
  double assemble_ms;
  double pcg_ms;
  double update_ms;
} vlba_iteration;

/* BaResult (bundle/mod.rs:765-771) plus diagnostics. */
typedef struct vlba_result {
  double initial_cost;
  double final_cost;
  uint32_t converged;
  uint32_t num_iterations;         /* total; entries beyond capacity dropped */
  uint64_t initial_nonprojectable;
  uint64_t final_nonprojectable;
  uint64_t total_pcg_iterations;
  uint64_t error_index;            /* id for MISSING_POSE / MISSING_LANDMARK; observation index for INVALID_OBSERVATION_WEIGHT */
  double device_ms;                /* device time of the LM iterations */
  double upload_ms;                /* host+device time of the upload */
  uint64_t kernel_launches;        /* kernels launched by the LM iterations */
  uint64_t upload_bytes;           /* host -> device bytes of the upload (ABI version 4) */
} vlba_result;

/* Device layout of a problem, computed on the host without touching the GPU
 * (the memory figure is what a solve allocates, for admission control). */
typedef struct vlba_plan_info {
  uint64_t variable_cameras;
  uint64_t variable_landmarks;
  uint64_t variable_observations;   /* observations of a variable landmark
                                       by a variable camera */
  uint64_t camera_pairs;            /* camera pairs sharing a variable
                                       landmark: off-diagonal Schur blocks */
  uint64_t schur_terms;             /* landmark terms summed into them */
  uint32_t tile_size;               /* Schur tiles are tile_size^2 blocks */
  uint32_t tile_rows;
  uint32_t tiles;
  uint32_t assembly_lanes;          /* lanes per off-diagonal block */
  uint64_t device_bytes;
  uint64_t upload_bytes;            /* host -> device bytes of an upload */
  double bytes_per_iteration;       /* algorithmic bytes of one LM iteration
                                       (linearisation + one trial) */
  double bytes_per_pcg_iteration;
} vlba_plan_info;

/* ------------------------------------------------------------ entry points */

/* ABI version of the loaded library (VLBA_ABI_VERSION). */
uint32_t visloc_ba_cuda_abi_version(void);

/* Reference defaults of BaConfig (mod.rs:729-752) and GpuBaSettings
 * (solver.rs:36-50: 100 PCG iterations, tolerance 1e-4). */
void visloc_ba_cuda_default_config(vlba_config* out);

/* Create a solver context on CUDA device `device`; NULL on failure.
 * Replaces GpuBundleAdjuster::new (solver.rs:130-190). */
void* visloc_ba_cuda_create(int device);

/* Release a context and all of its device memory. */
void visloc_ba_cuda_destroy(void* ctx);

/* Message of the last failure on `ctx` (valid until the next call on it). */
const char* visloc_ba_cuda_last_error(void* ctx);

/* Validation and eligibility only, no device work: the checks of
 * BundleAdjustment::optimize_weighted_backend (bundle/lm.rs:168-229) and of
 * GpuBundleAdjuster::check (solver.rs:212-251) that apply to this problem
 * type.  `error_index` (may be NULL) receives the offending id. */
int visloc_ba_cuda_check(const vlba_problem* problem, const vlba_config* config,
                         uint64_t* error_index);

/* Levenberg-Marquardt solve of `problem` in place.  Replaces
 * GpuBundleAdjuster::optimize (solver.rs:552-690) and the reference CPU
 * BundleAdjustment::optimize (bundle/optimize.rs:8-28 -> lm.rs:162-1017).
 * `iterations` (capacity `iterations_capacity`, may be 0/NULL) receives the
 * per-iteration trace of BaResult::iterations. */
int visloc_ba_cuda_optimize(void* ctx, vlba_problem* problem,
                            const vlba_config* config, vlba_result* result,
                            vlba_iteration* iterations,
                            uint32_t iterations_capacity);

/* The three phases of visloc_ba_cuda_optimize, for callers that solve the
 * same problem repeatedly or time the device solve alone:
 *   upload:          validate, build the device structures, copy the state;
 *   solve_uploaded:  LM from the uploaded initial state, device-resident;
 *   download:        copy the last solve's poses and landmarks back.
 * GpuBundleAdjuster::upload (solver.rs:253-385) is the reference's upload. */
int visloc_ba_cuda_upload(void* ctx, const vlba_problem* problem,
                          const vlba_config* config);
int visloc_ba_cuda_solve_uploaded(void* ctx, const vlba_config* config,
                                  vlba_result* result,
                                  vlba_iteration* iterations,
                                  uint32_t iterations_capacity);
int visloc_ba_cuda_download(void* ctx, vlba_problem* problem);

/* Host-only: validate `problem`, build its device layout and check every
 * index of that layout against the arrays it addresses; `pcg_iterations`
 * sets the PCG count of bytes_per_iteration.  No device is needed. */
int visloc_ba_cuda_plan(const vlba_problem* problem, const vlba_config* config,
                        double pcg_iterations, vlba_plan_info* info);

/* Robust cost and non-projectable count of `problem` as given, in FP64 on the
 * device: BundleAdjustment::robust_cost_weighted (bundle/problem.rs:497-560)
 * and nonprojectable_observation_count (problem.rs:252-304), the pair the
 * reference GPU path evaluates on the CPU (cost_and_nonprojectable,
 * solver.rs:696-727). */
int visloc_ba_cuda_cost(void* ctx, const vlba_problem* problem,
                        const vlba_config* config, double* cost,
                        uint64_t* nonprojectable);

/* ----------------------------------------------------------------- batches */
/* Many independent problems (local BA windows, pose-only refinements, whole
 * models) packed into one device layout and solved together: every kernel
 * launch covers all of them, each problem keeps its own LM state (lambda,
 * accept/reject, convergence) and stops on its own, and every sum is taken
 * per problem in a fixed order, so a problem's result is identical solved
 * alone or in any batch.  The reference solves such windows one call at a
 * time through BaAccelerator::optimize (ba_accel.rs:23-32); this is its
 * batched form.
 *
 * statuses[i] (may be NULL) receives problem i's validation status; problems
 * that fail validation are left out of the batch (the call still succeeds if
 * any problem remains).  results has n entries and iterations n x
 * iterations_capacity (row i for problem i); entries of problems left out are
 * zeroed.  The configs' VLBA_FLAG_* bits are combined. */
int visloc_ba_cuda_batch_optimize(void* ctx, uint32_t n, vlba_problem* const* problems,
                                  const vlba_config* const* configs, int* statuses,
                                  vlba_result* results, vlba_iteration* iterations,
                                  uint32_t iterations_capacity);
int visloc_ba_cuda_batch_upload(void* ctx, uint32_t n, const vlba_problem* const* problems,
                                const vlba_config* const* configs, int* statuses);
int visloc_ba_cuda_batch_solve_uploaded(void* ctx, vlba_result* results,
                                        vlba_iteration* iterations,
                                        uint32_t iterations_capacity);
int visloc_ba_cuda_batch_download(void* ctx, uint32_t n, vlba_problem* const* problems);

/* --------------------------------------------------------- reduced solves */
/* ReducedSolveAccelerator::solve (pipelines/slam/src/ba_accel.rs:50-72 and
 * :128-135): block-Jacobi preconditioned conjugate gradients on a reduced
 * camera system the caller has formed, in the reference's layout -- the
 * damped 6x6 diagonal blocks (f64, column-major, nalgebra Matrix6), the
 * sorted edges (a, b), a < b, and for each edge the (row b, column a)
 * block (f32, column-major), the right-hand side, and the stopping rule
 * |r| <= tol |rhs| within max_iterations.  The step (6 per node) and the
 * iteration count are returned.  Systems that carry cluster inverses or a
 * coarse level go to visloc_ba_cuda_reduced_solve_preconditioned below; the
 * accelerator-side elimination (empty offdiag) is not implemented, and a
 * shim returns None for it, so the caller eliminates on its CPU. */
typedef struct vlba_reduced_system {
  uint32_t num_nodes;
  uint32_t reserved;
  uint64_t num_edges;
  const double* diag;      /* [36 num_nodes] */
  const uint32_t* edges;   /* [2 num_edges] */
  const float* offdiag;    /* [36 num_edges] */
  const double* rhs;       /* [6 num_nodes] */
  double tol;
  uint32_t max_iterations;
  uint32_t reserved2;
} vlba_reduced_system;

int visloc_ba_cuda_reduced_solve(void* ctx, const vlba_reduced_system* system, double* x,
                                 uint32_t* iterations, double* relative_residual);

/* The preconditioners of ReducedCameraSystem::clusters and ::coarse
 * (pipelines/slam/src/ba_accel.rs:64-69; built by cluster_inverses and
 * coarse_correction, pipelines/slam/src/colmap_incremental/rig_ba_solver.rs:
 * 1101-1140 and 1235-1266; applied as in pcg_core, :1406-1480):
 *
 *   z = M r:  over each run c of cluster_size[c] consecutive nodes from
 *             cluster_first[c], z_run = cluster inverse c times r_run; the
 *             6x6 block-Jacobi inverse of the diagonal for nodes in no run;
 *             then, with a coarse level, z += P (P^T S P)^-1 P^T r, where P
 *             sums aggregates of coarse_group consecutive nodes over the
 *             leading coarse_nodes.
 *
 * Runs are ascending and disjoint, at most 1024 nodes each; each inverse is
 * (6 size)^2 doubles, column-major (nalgebra DMatrix), concatenated in run
 * order.  coarse_inverse is (6 m)^2 doubles, column-major, m =
 * ceil(coarse_nodes / coarse_group) <= 2048; coarse_nodes = 0 means no
 * coarse level.  The reference hands over its runs as (first node, inverse)
 * with all runs of one length k but the last: cluster_first[c] = c k. */
typedef struct vlba_reduced_preconditioner {
  uint32_t num_clusters;
  uint32_t reserved;
  const uint32_t* cluster_first;   /* [num_clusters] */
  const uint32_t* cluster_size;    /* [num_clusters] nodes */
  const double* cluster_inverse;   /* sum over runs of (6 size)^2 */
  uint32_t coarse_group;
  uint32_t coarse_nodes;
  const double* coarse_inverse;    /* [(6 m)^2] or null without a level */
} vlba_reduced_preconditioner;

/* visloc_ba_cuda_reduced_solve with the preconditioner above (null: block-
 * Jacobi, the same iteration as visloc_ba_cuda_reduced_solve up to the
 * order of its sums).  The iteration follows pcg_core: x = 0, r = b, z = M r,
 * p = z; per iteration q = S p, alpha = r.z / p.q, x += alpha p, r -= alpha
 * q, stop once |r| <= tol |b| or max_iterations have run, else z = M r and
 * p = z + beta p.  Vectors and S are f32, dots and scalars f64; every sum
 * runs in a fixed order, so repeated solves give identical steps.  A p.q
 * that is not positive and finite fails the solve as in pcg_core (which
 * returns None): VLBA_DECLINED, and the caller runs its CPU solver.  Edges
 * out of order or repeated are declined too, as the reference's solver does
 * (VLBA_ERR_INVALID_ARGUMENT for an edge that is not a < b < nodes).  A zero
 * right-hand side gives x = 0 after 0 iterations.
 *
 * Both reduced-solve entry points accept offdiag = NULL with num_edges > 0:
 * the blocks the context's last visloc_ba_cuda_reduced_eliminate formed, as
 * ReducedCameraSystem::offdiag empty means (ba_accel.rs:58-60).  The edges
 * must equal that elimination's, else VLBA_DECLINED (the reference's solve
 * returns None without resident blocks). */
int visloc_ba_cuda_reduced_solve_preconditioned(void* ctx, const vlba_reduced_system* system,
                                                const vlba_reduced_preconditioner* pre,
                                                double* x, uint32_t* iterations,
                                                double* relative_residual);

/* ReducedSolveAccelerator::eliminate (ba_accel.rs:136-144) on a
 * PointElimination (ba_accel.rs:74-120): the off-diagonal blocks of the
 * reduced camera system,
 *
 *   block(e) = extra(e) - sum over points p whose k-th and j-th nodes (k < j)
 *              are s and t of  hcp[p, j] V_p^-1 hcp[p, k]^T,
 *
 * for each edge e = (s, t), s < t, the (row t, column s) block, formed on the
 * device and kept there for the next solve with offdiag = NULL.  What
 * returns to the caller: the blocks of run_edges (the edges inside its
 * preconditioner runs, in that order) and, with coarse_group > 0, for each
 * aggregate pair g <= h of the coarse level the sum of the blocks of edges
 * from aggregate g to h within the leading coarse_nodes (coarse_sums[g m +
 * h], m = ceil(coarse_nodes / coarse_group); entries g > h are zero).
 *
 * Each term is a 6x6 product of FP32 copies of hcp and of hcp V^-1 (formed
 * in FP64), summed in FP64 in ascending point order, so the blocks do not
 * depend on scheduling and repeated eliminations give identical blocks.
 * The reference's per-node Cauchy-Schwarz bounds (`scale`) only scale its
 * fixed-point sums; FP64 sums in a fixed order need none, and there is no
 * field for them.  Its per-node slot lists (`slot_off`, `slots`) and edge
 * row offsets (`row_off`) are derived here from the edges and point_nodes.
 *
 * The structure (edges, point_off, point_nodes) is indexed once per
 * structure_id (nonzero) and kept while the id and the sizes stay the same;
 * hcp is uploaded again whenever linearization_id changes.  Every pair of
 * nodes of a point must be an edge.  VLBA_DECLINED when a returned block is
 * not finite (the reference's None). */
typedef struct vlba_point_elimination {
  uint64_t structure_id;
  uint64_t linearization_id;
  uint32_t num_nodes;
  uint32_t num_points;
  uint64_t num_edges;
  const uint32_t* edges;          /* [2 num_edges] (s, t), s < t, ascending */
  const uint64_t* point_off;      /* [num_points + 1] into point_nodes / hcp */
  const uint32_t* point_nodes;    /* ascending within each point */
  const double* hcp;              /* [18 point_off[num_points]] 6x3 column-major J_node^T J_point */
  const double* point_inverse;    /* [9 num_points] damped V_p^-1, 3x3 column-major */
  const uint8_t* point_used;      /* [num_points] 0: left out (None); NULL: all used */
  uint64_t num_extra;
  const uint32_t* extra_edge;     /* [num_extra] edge of each direct coupling */
  const double* extra_block;      /* [36 num_extra] column-major, added to its edge's block */
  uint64_t num_run_edges;
  const uint32_t* run_edges;      /* [num_run_edges] */
  uint32_t coarse_group;          /* nodes per aggregate; 0: no coarse sums */
  uint32_t coarse_nodes;          /* leading nodes the aggregates cover */
} vlba_point_elimination;

int visloc_ba_cuda_reduced_eliminate(void* ctx, const vlba_point_elimination* elimination,
                                     double* run_blocks /* [36 num_run_edges] */,
                                     double* coarse_sums /* [36 m m] or NULL without coarse */);

/* Device times of the context's last reduced solve and elimination, from
 * CUDA events on its stream: fill_ms the system's host-to-device copies and
 * the fill of S's tiles, pcg_ms the PCG loop (with the host's checks between
 * launches of the preconditioned loop), eliminate_ms the elimination's
 * uploads of this call and its kernels.  Diagnostics for measurement; no
 * counterpart in the reference. */
typedef struct vlba_reduced_timing {
  double fill_ms;
  double pcg_ms;
  double eliminate_ms;
  double reserved;
} vlba_reduced_timing;

int visloc_ba_cuda_reduced_timing(void* ctx, vlba_reduced_timing* out);

/* --------------------------------------------------------------- autotuner */
/* Launch shape of the uploaded system: the blocks of the persistent PCG
 * kernel and the share of the L2 that keeps tiles of S resident across PCG
 * iterations.  Neither changes any result (every sum's order is fixed by the
 * problem's layout), only the time.  visloc_ba_cuda_autotune times a fixed
 * number of PCG iterations for candidate shapes on the system assembled at the
 * uploaded state, applies the fastest and caches it for systems of the same
 * shape (tiles, tile rows and problems, by powers of two) for the process;
 * visloc_ba_cuda_set_launch_shape forces one (pcg_blocks 0: the largest
 * co-resident grid).  No counterpart in the reference (its shader workgroup
 * sizes are fixed). */
typedef struct vlba_launch_shape {
  int32_t pcg_blocks;
  int32_t reserved;
  double l2_resident_fraction;
  double pcg_iteration_us;   /* measured by the autotuner (0 when forced) */
} vlba_launch_shape;

int visloc_ba_cuda_autotune(void* ctx, vlba_launch_shape* chosen);
int visloc_ba_cuda_set_launch_shape(void* ctx, const vlba_launch_shape* shape);

/* ----------------------------------------------------------------- serving */
/* A request loop on one GPU for streams of independent solves (localisation
 * refinements, local windows, occasional global BAs).  A submitted ticket is
 * validated and planned on a host thread, then admitted into a batch by one
 * of `slots` worker slots as soon as a slot and device memory are free; the
 * batches of different slots overlap on the device.  A request of many
 * observations runs as a batch of its own.  Each slot owns
 * memory_bytes / slots of device memory, allocated once at creation
 * (memory_bytes 0: half of the free memory); a request that does not fit a
 * slot completes with VLBA_ERR_OUT_OF_MEMORY.  Results are the same as solving
 * the problem alone.  The problem's arrays are read while the ticket is
 * planned and written (the optimised state) when it completes: keep them
 * alive and untouched until visloc_ba_cuda_server_wait has returned for the
 * ticket.  The reference has no serving loop; its callers solve one problem
 * per BaAccelerator::optimize call (ba_accel.rs:23-32). */
typedef struct vlba_ticket_info {
  double latency_ms;   /* submit -> done */
  double queue_ms;     /* submit -> its batch started (planning included) */
  double solve_ms;     /* its batch's upload, LM and download */
  uint32_t batch_size; /* problems in its batch */
  uint32_t slot;
} vlba_ticket_info;

void* visloc_ba_cuda_server_create(int device, uint32_t slots, uint64_t memory_bytes,
                                   uint32_t max_batch);
/* Finishes the tickets already submitted, then stops. */
void visloc_ba_cuda_server_destroy(void* server);
int visloc_ba_cuda_server_submit(void* server, vlba_problem* problem,
                                 const vlba_config* config, uint64_t* ticket);
/* Wait up to timeout_ms (negative: no limit, 0: poll) for a ticket: its
 * status (VLBA_ERR_BUSY if still pending), result, iterations and timing.
 * A ticket whose status has been returned is released. */
int visloc_ba_cuda_server_wait(void* server, uint64_t ticket, double timeout_ms,
                               vlba_result* result, vlba_iteration* iterations,
                               uint32_t iterations_capacity, vlba_ticket_info* info);
const char* visloc_ba_cuda_server_last_error(void* server);

/* ------------------------------------------------------------- diagnostics */
/* Self-test of the bounded device waits every kernel uses (mbarrier waits,
 * row counters, the grid barrier give up after 2 s, set an error bit and let
 * the kernel return, so a lost arrival becomes VLBA_ERR_TIMEOUT instead of a
 * hung GPU): waits on a device flag that nothing sets for limit_ms and
 * returns VLBA_ERR_TIMEOUT with the time it waited.  The context stays usable
 * afterwards.  No reference counterpart. */
int visloc_ba_cuda_wait_probe(void* ctx, double limit_ms, double* waited_ms);

/* One damped linear step at the given state, without updating it: the step
 * of solve_step (bundle/normal_equations.rs:1621-1733) as this solver forms
 * it (linearisation, reduced system, PCG, back-substitution).  dp holds 6
 * values ([rho; omega]) per variable pose and dl 3 per variable landmark, in
 * index order; both may be NULL.  pcg_iterations / pcg_relative_residual may
 * be NULL. */
int visloc_ba_cuda_linear_step(void* ctx, const vlba_problem* problem,
                               const vlba_config* config, double lambda,
                               double* dp, double* dl, uint32_t* pcg_iterations,
                               double* pcg_relative_residual);

/* The damped reduced camera system S (dense, (6 Nc)^2 row-major, both
 * triangles, Nc = variable poses) and its right-hand side at `lambda`, as
 * assembled on the device. */
int visloc_ba_cuda_reduced_system(void* ctx, const vlba_problem* problem,
                                  const vlba_config* config, double lambda,
                                  double* s_dense, double* rhs);

/* --------------------------------------------------------------------- GNC */
/* GncKernel (pipelines/slam/src/gnc.rs:38-48). */
enum vlba_gnc_kernel {
  VLBA_GNC_GEMAN_MCCLURE = 0,          /* GncKernel::GemanMcClure (default) */
  VLBA_GNC_TRUNCATED_LEAST_SQUARES = 1 /* GncKernel::TruncatedLeastSquares */
};

/* GncConfig (gnc.rs:50-110); visloc_ba_cuda_default_gnc_config fills
 * GncConfig::default() (gnc.rs:100-110). */
typedef struct vlba_gnc_config {
  uint32_t kernel;             /* vlba_gnc_kernel */
  uint32_t max_outer;          /* cap on mu levels */
  uint32_t inner_iterations;   /* LM iterations per level */
  uint32_t has_auto_scale;     /* auto_scale: 0 = None */
  double c;                    /* inlier scale in pixels (a floor under auto_scale) */
  double anneal_factor;        /* geometric mu step, > 1 */
  double auto_scale;           /* k of median + k 1.4826 MAD when has_auto_scale */
  uint32_t auto_scale_readapt; /* re-estimate the scale at every level */
  uint32_t reserved;
} vlba_gnc_config;

/* BaGncResult (bundle/mod.rs:975-1000); the weight vector is returned
 * through `observation_weights`. */
typedef struct vlba_gnc_result {
  double initial_cost;         /* non-robust cost at the input estimate */
  double final_cost;           /* sum of w s at the recovered estimate */
  double inlier_cost;          /* sum of s over observations with w >= 0.5 */
  double inlier_scale;         /* the c the solve used */
  uint64_t observation_count;
  uint32_t outer_iterations;
  uint32_t converged;          /* the mu schedule reached its terminal level */
  uint64_t lm_iterations;      /* inner LM iterations, all levels */
  double device_ms;            /* device time of the inner solves */
} vlba_gnc_result;

void visloc_ba_cuda_default_gnc_config(vlba_gnc_config* gnc);

/* BundleAdjustment::optimize_gnc (bundle/lm.rs:28-142): anneal the GNC
 * surrogate from least squares to the robust cost, each level a short
 * weighted LM solve (config's lambda schedule and tolerances, no robust
 * kernel, gnc->inner_iterations iterations) from the previous level's state,
 * with the per-observation Black-Rangarajan weights of the level.  The
 * problem is uploaded once; residuals and weights move between host and
 * device per level.  problem->obs_weight must be NULL (GNC sets the weights).
 * On success the state is written back in place and, when
 * `observation_weights` is not NULL, it receives the final weight of every
 * observation in the problem's order (NaN where the observation cannot be
 * evaluated at the final estimate). */
int visloc_ba_cuda_optimize_gnc(void* ctx, vlba_problem* problem, const vlba_config* config,
                                const vlba_gnc_config* gnc, vlba_gnc_result* result,
                                double* observation_weights);

/* ----------------------------------------------------- allocation-free cost */
/* No counterpart in the reference: an addition for callers that cannot
 * allocate device memory when they need a cost -- a tracking thread with a
 * frame deadline, where cudaMalloc/cudaFree may synchronise the device and
 * stall it, or a process whose device memory belongs to another allocator.
 *
 * The same robust cost and non-projectable count as visloc_ba_cuda_cost, for
 * a problem whose arrays are already in DEVICE memory: pose_q, pose_t,
 * landmarks, obs_pose, obs_landmark, obs_xy, obs_camera, obs_weight,
 * obs_kind, obs_stereo and obs_right_camera are device pointers; `cameras`
 * (at most VLBA_NOALLOC_MAX_CAMERAS) is read on the host during the call;
 * pose_fixed and landmark_fixed are ignored.  `cost` (one double) and
 * `counts` (two words: non-projectable observations, and observations
 * skipped for a pose, landmark or camera index out of range, a weight that
 * is negative or not finite, or a stereo observation without a usable
 * baseline, right camera or pinhole cameras[0])
 * are device pointers, written by a kernel enqueued on `stream` (a
 * cudaStream_t of the current device; NULL = default stream); the call
 * returns without waiting for it.
 *
 * Nothing is allocated: the kernel's scratch is a fixed array of 1 MiB +
 * 256 B (a 256-byte header and 65,536 partials of 16 B) in the library's
 * device code, held by every GPU that loads the library until the process
 * exits, which limits a call to VLBA_NOALLOC_MAX_OBSERVATIONS observations
 * (larger problems return VLBA_ERR_INVALID_ARGUMENT).  All calls on a device
 * share that array: calls whose kernels may overlap on the GPU race and must
 * be serialised by the caller.  The first call on each device looks the
 * array's address up (set-up), and so does the first call after the
 * device's current context has changed (a cudaDeviceReset, after which the
 * array may sit elsewhere, or another context of the device made current);
 * make those calls before any stream capture.
 * `error` (capacity `error_capacity`, may be NULL) receives a message when
 * the status is not VLBA_OK. */
#define VLBA_NOALLOC_MAX_OBSERVATIONS 16777216ull
#define VLBA_NOALLOC_MAX_CAMERAS 16u
int visloc_ba_cuda_cost_noalloc(const vlba_problem* problem,
                                const vlba_config* config, void* stream,
                                double* cost, uint64_t* counts, char* error,
                                size_t error_capacity);

#ifdef __cplusplus
}
#endif

#endif /* VISLOC_BA_CUDA_H */
