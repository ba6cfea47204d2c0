// vlba_common.cuh -- device data layout shared by the kernels and the host.
//
// Layout in HBM (one or more problems packed back to back):
//   poses      f64 quaternion + translation, current and candidate copies, and
//              a derived f64 (R, t) table per copy (96 B per pose);
//   points     f64 xyz, current and candidate;
//   obs        sorted point-major: pose, point, variable-camera slot, camera
//              model, pixel (f64), and two linearisation records per obs:
//              H_o = w J_l^T J_l (upper 3x3, f32, plus point index and the
//              point's z) and e_o = w J_l^T r (f32); per trial, a copy of the
//              point's damped inverse and x, y next to each observation, so
//              that a Schur term reads three 32-byte records;
//   S          the reduced camera system in dense TB x TB tiles of 6x6 f32
//              blocks (lower block triangle; diagonal tiles stored full);
//   vectors    PCG x, r, z, p, q in f32, 6 per variable camera, tile padded.
//
// The pose Jacobian of every observation factors as J_p = J_l [I | -[X]x]
// (right perturbation of T_world->rig, bundle/normal_equations.rs:447-456 and
// sqrt_qr.rs:990-998), so H_o and e_o carry everything the Schur complement
// needs: W_o = J_p^T J_l = B^T H_o with B = [I | -[X]x].

#pragma once

#include <vector_types.h>

#include <cstdint>

#include "../../include/visloc_ba_cuda.h"

namespace vlba {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// Observation kinds (vlba_problem.obs_kind).
constexpr uint32_t kObsMono = 0;           // BaObservation / BaRigObservation
constexpr uint32_t kObsStereo = 1;         // BaStereoObservation (rectified)
constexpr uint32_t kObsGeneralStereo = 2;  // BaGeneralStereoObservation
constexpr int kBlock = 36;             // floats in a 6x6 block
// Every device wait (on an mbarrier, a counter or a flag that another block
// writes) gives up after this long, sets an error bit and lets its kernel
// return: a lost arrival turns into VLBA_ERR_TIMEOUT, never a hung GPU.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

// Camera of an observation (f64).  R/t is sensor_from_rig (identity for
// monocular observations).
struct DevCamera {
  double fx, fy, cx, cy, k1, k2;
  double R[9];
  double t[3];
  int radial;  // MonoProjection::Radial
  int rig;     // apply sensor_from_rig
  int pad[2];
};

// Per-problem LM settings (BaConfig + PCG controls).
struct LmParams {
  double initial_lambda;
  double lambda_increase_factor;
  double lambda_decrease_factor;
  double max_lambda;
  double min_lambda;
  double step_tolerance;
  double cost_tolerance;
  double relative_cost_tolerance;
  double robust_parameter;
  double pcg_relative_tolerance;
  uint32_t has_initial_lambda;
  uint32_t has_relative_cost_tolerance;
  uint32_t robust_kernel;
  uint32_t max_iterations;
  uint32_t max_pcg_iterations;
  uint32_t pad[3];
};

// Per-problem LM state, owned by the device (k_decide).
struct Ctrl {
  double lambda;
  double current_cost;
  double initial_cost;
  double cost_after;
  double max_pose_step;
  double max_landmark_step;
  double pcg_rel_res;
  double pad_d;
  unsigned long long current_nonproj;
  unsigned long long initial_nonproj;
  unsigned long long nonproj_after;
  unsigned long long total_pcg;
  uint32_t iteration;    // LM iterations (trials) performed
  uint32_t done;
  uint32_t converged;
  uint32_t relinearize;  // linearise before the next trial
  uint32_t cur;          // which state buffer (0/1) holds the current state
  uint32_t pcg_iters;
  uint32_t pcg_status;   // 0 converged, 1 iteration cap, 2 breakdown, 3 timeout
  uint32_t nonfinite;    // the step had a non-finite entry (singular system)
};

// PCG control words of one problem (written by the PCG kernel).
struct PcgState {
  double rz;
  double bnorm;
  double rnorm;
  uint32_t iters;
  uint32_t status;  // 0 running/converged, 1 cap, 2 breakdown
  uint32_t active;
  uint32_t pad;
};

// Off-diagonal blocks of at least this many terms are summed on kLongLanes
// lanes instead of the plan's lane count (a block's summation order then
// depends on its own length only, the same alone and in any batch).
constexpr uint32_t kLongBlockTerms = 1024;
constexpr int kLongLanes = 32;

// Everything the kernels touch.  Passed by value.
struct Dev {
  // sizes
  uint32_t num_problems;
  uint32_t num_poses;
  uint32_t num_points;
  uint32_t num_obs;
  uint32_t num_var_cams;       // padded slot count (multiple of TB per problem)
  uint32_t num_tile_rows;
  uint32_t num_tiles;
  uint32_t num_offdiag_blocks;
  uint32_t num_dup_pairs;
  uint32_t num_point_chunks;
  uint32_t tb;                  // tile size in blocks
  uint32_t group;               // lanes per off-diagonal block in assembly

  // problem ranges
  const uint32_t* prob_pose_begin;   // [num_problems + 1]
  const uint32_t* prob_point_begin;  // [num_problems + 1]
  const uint32_t* prob_tr_begin;     // tile rows [num_problems + 1]
  const uint32_t* prob_chunk_begin;  // point chunks [num_problems + 1]
  const uint32_t* pose_prob;         // [num_poses]
  const uint32_t* point_prob;        // [num_points]
  const uint32_t* slot_prob;         // [num_var_cams]
  const LmParams* params;            // [num_problems]
  Ctrl* ctrl;                        // [num_problems]
  PcgState* pcg;                     // [num_problems]
  vlba_iteration* records;           // [num_problems * max_records]
  uint32_t max_records;

  // state: two buffers each; Ctrl::cur selects the current one, the other
  // receives the candidate of a trial (an accepted step flips cur).
  double* pose_q[2];    // [4 N] quaternion (w, i, j, k)
  double* pose_t[2];    // [3 N]
  double* pose_rt[2];   // [12 N] derived R (row-major) and t
  double* points[2];    // [3 M]
  const double* init_pose_q;   // uploaded initial state (reset by copy on device)
  const double* init_pose_t;
  const double* init_points;
  const uint32_t* pose_slot;   // [N] variable slot or kNone
  const uint8_t* point_var;    // [M] 1 = variable
  double* pose_step;           // [N] |xi| of the last trial

  // cameras
  const DevCamera* cameras;

  // observations, point-major
  const uint32_t* pt_off;      // [M + 1]
  const uint32_t* obs_point;   // [K] point of each observation
  const uint32_t* obs_pose;    // [K]
  const uint32_t* obs_cam;     // [K] camera index
  const uint32_t* obs_slot;    // [K] variable slot of the pose or kNone
  const double2* obs_xy;       // [K]
  const double* obs_w;         // [K] external observation weights, or null (all 1)
  // Stereo observations (null when the plan has none): kind per observation
  // (kObsMono / kObsStereo / kObsGeneralStereo), its stereo data ((u_r,
  // baseline) rectified, the right pixel general) and right camera.
  const uint8_t* obs_kind;     // [K]
  const double2* obs_st;       // [K]
  const uint32_t* obs_rcam;    // [K]
  float4* obs_h;               // [2 K]: {h00,h01,h02,h11} {h12,h22,point,X.z}
  float4* obs_e;               // [K]:   {e0,e1,e2,w}
  float4* pt_p;                // [2 M]: each point's record, per trial:
                               //        {hinv00,01,02,11} {hinv12,22,X.x,X.y}

  // per-camera observation lists (indices into the point-major order)
  const uint32_t* cam_off;     // [num_var_cams + 1]
  const uint32_t* cam_obs;
  uint32_t* cam_pt;            // [cam_obs] each listed observation's point (set at upload)

  // per point, per linearisation / per trial
  float* pt_h;                 // [9 M] H_ll upper (6) + g_l (3)
  float4* pt_s;                // [4 M] {hinv00,01,02,11} {hinv12,22,X.x,X.y} {X.z,v0,v1,v2} {g0,g1,g2,ok}
  double* pt_c;                // [12 M] per trial, 96 bytes per point: its FP64 damped inverse
                               // {i00,i01,i02,i11,i12,i22}, v = H^-1 g {v0,v1,v2}, then
                               // X.x, X.y | X.z, ok as f32 pairs, one spare (zero inverse
                               // and v for a point without one)

  // per camera
  double* cam_hpp;             // [27 C] H_pp upper 21 + g_p 6 (f64)

  // reduced system
  float* tiles;                // [num_tiles * tb*tb * 36]
  const uint32_t* tile_ij;     // [num_tiles] (I << 16) | J
  const uint32_t* blk_off;     // [num_offdiag_blocks + 1] pair ranges
  // The assembly's blocks in the order it takes them: each one's term range
  // (first, end) and destination, at its place in that order.
  const uint2* ord_range;      // [num_offdiag_blocks]
  const uint2* ord_dst;        // [num_offdiag_blocks]
  // Blocks of at least kLongBlockTerms terms, summed on kLongLanes lanes
  // (the lane count of a block follows from its own length alone), listed
  // in any order: their term ranges and destinations, and their count.
  const uint2* long_range;     // [num_offdiag_blocks]
  const uint2* long_dst;       // [num_offdiag_blocks]
  uint32_t* num_long;          // [1] appended by the block order at upload
  uint32_t num_long_blocks;    // the same count, read back at upload
  const uint2* pairs;          // (k_i, k_j), sorted by block then point
  uint32_t* pair_pt;           // [pairs] each term's point (set at upload)
  const uint2* blk_dst;        // [num_offdiag_blocks] float offsets (block, mirror or kNone)
  const uint32_t* diag_dst;    // [num_var_cams] float offset of the diagonal block
  const uint32_t* dup_off;     // [num_var_cams + 1] same-camera pairs k != k'
  const uint2* dup_pairs;
  float* minv;                 // [36 C]
  float* rhs;                  // [6 C]

  // PCG
  float* x;
  float* r;
  float* z;
  float* p;
  float* q;
  float* partial;              // [list slots * tb * 6]: row-contiguous partials
  const uint2* tile_slot;      // [num_tiles] slot of the row side, column side
  const uint4* tile_meta;      // [num_tiles] {ij, row slot, column slot, problem}
  const uint32_t* tr_list_off; // [num_tile_rows + 1]
  const uint32_t* tr_list;     // partial indices (tile * 2 + side)
  const uint32_t* tr_prob;     // [num_tile_rows]
  double* dots;                // [16 * num_tile_rows]
  uint32_t l2_resident_tiles;  // tiles [0, n) are streamed with L2 evict_last
  unsigned int* barrier;       // [kBarrierWords]: [0] grid-barrier arrivals, [2] active problems
                               // problems, -, group counts
  unsigned int* error;         // [1] device error flags
  // Optional PCG phase trace (globaltimer ns): [iteration][block][kTracePhases]
  // for iterations < kTraceIters; null unless VLBA_TRACE_PCG is set.
  unsigned long long* trace;

  // reductions
  const uint32_t* chunk_point_begin;  // [num_point_chunks + 1]
  double* chunk_cost;
  unsigned long long* chunk_bad;
  double* chunk_step;
};

constexpr int kBarrierWords = 4;  // PCG grid-barrier and active-count words
constexpr int kTracePhases = 6;
constexpr int kTraceIters = 64;

enum ErrorBits : unsigned int {
  kErrBarrierTimeout = 1u,
  kErrTmaTimeout = 2u,
};

#ifdef __CUDACC__
// Nanoseconds of the GPU's global timer (deadlines of the bounded waits).
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
#endif

}  // namespace vlba
