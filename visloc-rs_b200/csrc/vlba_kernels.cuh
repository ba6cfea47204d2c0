// vlba_kernels.cuh -- declarations of the LM-step kernels (vlba_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "vlba_common.cuh"

namespace vlba {

// Launch helpers; every kernel reads the per-problem Ctrl and skips problems
// that are done (so a batch keeps running while some problems finish).
cudaError_t launch_pose_table(const Dev& d, cudaStream_t s);
cudaError_t launch_cost(const Dev& d, bool trial, cudaStream_t s);
cudaError_t launch_decide(const Dev& d, bool init, cudaStream_t s);
cudaError_t launch_linearize(const Dev& d, cudaStream_t s);
cudaError_t launch_point_prep(const Dev& d, cudaStream_t s);
cudaError_t launch_offdiag(const Dev& d, cudaStream_t s);
cudaError_t launch_cam_diag(const Dev& d, cudaStream_t s);
// ord_range / ord_dst: the blocks of each window of 256 sorted by the loop
// passes they take at d.group lanes (longest first, ties in plan order).
cudaError_t launch_block_order(const Dev& d, cudaStream_t s);
// pair_pt[q] = obs_point[pairs[q].x] for the n Schur terms.
cudaError_t launch_pair_points(const Dev& d, uint64_t n, cudaStream_t s);
// cam_pt[i] = obs_point[cam_obs[i]] for the n listed observations.
cudaError_t launch_cam_points(const Dev& d, uint32_t n, cudaStream_t s);
cudaError_t launch_pcg(const Dev& d, int sm_count, cudaStream_t s);
cudaError_t launch_pose_update(const Dev& d, cudaStream_t s);
cudaError_t launch_pcg_setup(const Dev& d, cudaStream_t s);
// Fill the tiles, preconditioner and rhs of a reduced system given directly
// (device arrays in the reference's layout; the off-diagonal blocks f32, or
// f64 when offdiag is null).
cudaError_t launch_reduced_fill(const Dev& d, uint32_t n, uint64_t ne, const double* diag,
                                const float* offdiag, const double* offdiag64, const double* rhs,
                                cudaStream_t s);
// Bounded-wait self-test: waits on `flag` (which nothing sets) for limit_ns.
cudaError_t launch_wait_probe(const unsigned int* flag, unsigned long long limit_ns,
                              unsigned int* err, unsigned long long* waited, cudaStream_t s);
// Copy each problem's current state into state buffer 0 (for a bulk download).
cudaError_t launch_state_to_front(const Dev& d, cudaStream_t s);
// Squared reprojection residual per observation (plan order) at the state in
// buffer 0; NaN where it cannot be evaluated.
cudaError_t launch_sq_residuals(const Dev& d, double* out, cudaStream_t s);

// Scalars of a preconditioned reduced solve (vlba_reduced.cu), on the device.
struct RpScalars {
  double alpha, beta, rz, bnorm, rnorm;
  uint32_t iters;
  uint32_t done;    // the loop is over: every kernel returns at once
  uint32_t failed;  // p.q not positive and finite
  uint32_t arrive;  // blocks of the running row kernel that have finished (reset by the last)
};

// The preconditioner and work arrays of a preconditioned reduced solve.
struct RpData {
  RpScalars* sc;
  double* dots;                // [3 num_tile_rows]: per tile row p.q, r.z, r.r
  uint32_t num_clusters;
  uint32_t max_cluster_rows;   // 6 x the longest run
  const uint32_t* cl_first;    // [num_clusters] first node
  const uint32_t* cl_size;     // [num_clusters] nodes
  const uint64_t* cl_off;      // [num_clusters] float offset of the inverse
  const float* cl_mat;         // column-major run inverses
  uint32_t coarse_m;           // aggregates (0: no coarse level)
  uint32_t coarse_group;
  uint32_t coarse_nodes;
  uint32_t max_iterations;
  const float* coarse_inv;     // [(6 m)^2] row-major
  float* rc;                   // [6 m] P^T r
  float* yc;                   // [6 m]
  double tol;
};

// x = 0, r = b, z = M r, p = z and the initial scalars (sc zeroed first).
cudaError_t launch_rp_init(const Dev& d, const RpData& rp, cudaStream_t s);
// One iteration; a no-op once sc->done is set.
cudaError_t launch_rp_iteration(const Dev& d, const RpData& rp, cudaStream_t s);

// Floats between consecutive FP32 camera-point blocks of an elimination: the
// 18 entries of a 6x3 block padded to 80 bytes (16-byte aligned loads).
constexpr int kElRec = 20;

// A point elimination on the device (vlba_reduced.cu): the pair index of the
// structure, this call's camera-point blocks and point inverses, the blocks.
struct ElimDev {
  uint32_t n;
  uint32_t num_points;
  uint64_t num_edges;
  uint64_t num_obs;
  uint64_t num_run;
  uint32_t coarse_m;           // aggregates (0: no coarse sums)
  uint32_t coarse_group;
  uint32_t coarse_nodes;
  uint32_t pad;
  const uint32_t* row_off;     // [n + 1]
  const uint32_t* edge_t;      // [num_edges]
  const uint32_t* pair_off;    // [num_edges + 1]
  const uint2* pairs;          // (o_s, o_t), ascending point within an edge
  const uint32_t* obs_point;   // [num_obs]
  const double* hcp64;         // [18 num_obs] 6x3 column-major
  const double* vinv64;        // [9 num_points] 3x3 column-major
  const uint8_t* used;         // [num_points] or null (all used)
  float* hcp32;                // [kElRec num_obs]
  float* sk32;                 // [kElRec num_obs] hcp V^-1 (zero for a point left out)
  const int32_t* extra_of;     // [num_edges] row of extra64 or -1; null: none
  const double* extra64;       // [36 rows]
  double* blocks;              // [36 num_edges] column-major (row t, column s)
  const uint32_t* run_edges;   // [num_run]
  double* run_out;             // [36 num_run]
  double* coarse_out;          // [36 m m]
  // The structure's pair index, built on the device: per node its blocks in
  // point order, each block's point and the points' block ranges; per edge
  // a count (then a write cursor); the pairs written; an error flag.
  const uint32_t* slot_off;    // [n + 1]
  const uint32_t* slot_obs;    // [num_obs]
  const uint32_t* point_off;   // [num_points + 1]
  const uint32_t* point_nodes; // [num_obs]
  uint32_t* cursor;            // [num_edges]
  uint2* pairs_out;            // [pairs]
  unsigned int* err;           // bit 0: a pair of a point's nodes has no edge
};

// The pair index: write = false counts each edge's pairs into cursor (zeroed
// first); write = true writes them at cursor (set to the edges' offsets).
cudaError_t launch_el_index(const ElimDev& e, bool write, cudaStream_t s);
cudaError_t launch_el_prepare(const ElimDev& e, cudaStream_t s);
cudaError_t launch_el_blocks(const ElimDev& e, cudaStream_t s);
cudaError_t launch_el_outputs(const ElimDev& e, cudaStream_t s);

// The Schur terms of one problem built on the device (vlba_pairs.cu): the
// arrays of its plan the builders read, their scratch and outputs.
struct RowsDev {
  uint32_t nvar;               // variable camera slots (rows)
  const uint32_t* cam_off;     // [nvar + 1] into cam_obs
  const uint32_t* cam_obs;     // per slot, its observations ascending
  const uint32_t* obs_point;
  const uint32_t* obs_slot;
  const uint8_t* point_var;
  const uint32_t* pt_off;
  uint2* tri;                  // [nvar (nvar - 1) / 2] per-row (column, terms) scratch
  uint32_t* row_nblk;          // [nvar]
  uint32_t* row_blk;           // [nvar + 1]
  uint32_t* col;               // [nvar (nvar - 1) / 2] packed columns
  uint32_t* count;             // [nvar (nvar - 1) / 2] packed term counts
  uint32_t* flags;             // bit 0: a point seen twice by one slot; bit 1: a term
                               // outside its block or a block left short
};

// Count each row's terms per column and pack the rows' (column, count)
// lists by the prefix of their lengths (row_blk).
cudaError_t launch_rows_count(const RowsDev& r, cudaStream_t s);
// Write every term at its place: per block in point order (the host order).
// max_row_blocks: the most blocks of any row (sizes the per-row state).
cudaError_t launch_rows_place(const RowsDev& r, const uint32_t* blk_off, const uint32_t* row_blk,
                              const uint32_t* blk_col, uint32_t max_row_blocks, uint2* pairs,
                              uint32_t* pair_pt, cudaStream_t s);
size_t rows_count_smem(uint32_t nvar);
// Shared memory of the placement with `warps` warps per row.
size_t rows_place_smem(uint32_t nvar, uint32_t max_row_blocks, int warps);

// Occupancy-derived grid of the persistent PCG kernel (0 if it cannot run).
int pcg_grid_size(int tb, int sm_count);
size_t pcg_smem_bytes(int tb);
// Tile rows one PCG block can own (a launch covers grid x this many rows).
int pcg_rows_per_block();

}  // namespace vlba
