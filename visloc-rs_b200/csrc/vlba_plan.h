// vlba_plan.h -- host-side construction of the device layout of one or more
// bundle-adjustment problems (the analogue of GpuBundleAdjuster::upload,
// crates/ba-gpu/src/solver.rs:253-385, extended to the explicit reduced
// camera system and to batches).  Pure C++; no CUDA calls.
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <utility>
#include <functional>
#include <vector>

#include "vlba_common.cuh"

namespace vlba {

struct PairIdx {
  uint32_t a, b;
};

// Asks the kernel to back [p, p + bytes) with transparent huge pages (where
// it only does so on request): the builder's scatters write into many
// streams across arrays of hundreds of MB, which 4 KB pages make
// TLB-bound.  A hint only.
void advise_huge_pages(void* p, size_t bytes);

// Page-locking of the large plan arrays an upload copies, so that the copies
// go from them straight to the device instead of through staging buffers.
// While a PinScope is alive on a thread, the arrays of 8 MB or more that it
// allocates are page-locked (where the device allows it; else they stay
// pageable) until they are freed; a plan rebuilt in place keeps them.
struct PinScope {
  PinScope();
  ~PinScope();
};
bool pin_requested();
void pin_allocation(void* p, size_t bytes);
void unpin_allocation(void* p);
// [p, p + bytes) lies inside one page-locked allocation.
bool pinned_range(const void* p, size_t bytes);

// Allocator whose resize() leaves new elements uninitialised, for the large
// pair arrays that the builder sizes first and then writes in full (from
// several threads, which then also take the page faults).  Allocations of 8 MB
// or more are advised huge pages before their first touch, and page-locked
// inside a PinScope.
template <typename T>
struct NoInit : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = NoInit<U>;
  };
  NoInit() noexcept = default;
  template <typename U>
  NoInit(const NoInit<U>&) noexcept {}
  T* allocate(size_t n) {
    T* p = std::allocator<T>::allocate(n);
    if (n * sizeof(T) >= (8u << 20)) {
      advise_huge_pages(p, n * sizeof(T));
      if (pin_requested()) pin_allocation(p, n * sizeof(T));
    }
    return p;
  }
  void deallocate(T* p, size_t n) {
    if (n * sizeof(T) >= (8u << 20)) unpin_allocation(p);
    std::allocator<T>::deallocate(p, n);
  }
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
using PairList = std::vector<PairIdx, NoInit<PairIdx>>;

struct Plan {
  uint32_t tb = 16;
  uint32_t group = 8;
  uint32_t num_problems = 0;

  std::vector<uint32_t> prob_pose_begin, prob_point_begin, prob_obs_begin, prob_tr_begin,
      prob_chunk_begin, prob_camera_begin;
  std::vector<uint32_t> pose_prob, point_prob, slot_prob;
  std::vector<LmParams> params;

  std::vector<double> pose_q, pose_t;
  std::vector<uint32_t> pose_slot;
  std::vector<uint8_t> point_var;
  std::vector<DevCamera> cameras;

  // Observation-scale arrays are sized first and then written in full, so
  // their resize leaves them uninitialised.
  template <typename T>
  using ObsArray = std::vector<T, NoInit<T>>;
  std::vector<uint32_t> pt_off;
  ObsArray<double> points;  // 3 per landmark
  ObsArray<uint32_t> obs_point, obs_pose, obs_cam, obs_slot;
  ObsArray<double> obs_xy;  // 2 per obs
  // External weight per observation; empty when no problem of the plan has
  // weights (a problem without them gets 1 in a plan that has them).
  ObsArray<double> obs_w;
  // Each observation's index in its problem's own order (host only: results
  // per observation go back to the caller in that order).
  ObsArray<uint32_t> obs_src;
  // Stereo observations, present when some problem has them (empty
  // otherwise): kind, stereo data (2 per observation: u_r and the baseline
  // for rectified stereo, the right pixel for general stereo) and the right
  // camera (general stereo).
  ObsArray<uint8_t> obs_kind;
  ObsArray<double> obs_st;
  ObsArray<uint32_t> obs_rcam;
  std::vector<uint32_t> cam_off;
  ObsArray<uint32_t> cam_obs;

  uint32_t num_var_cams = 0;  // padded slots
  uint32_t num_tile_rows = 0;
  std::vector<uint32_t> tile_ij;
  std::vector<uint32_t> blk_off;
  PairList pairs;  // per block, its (row-slot observation, column-slot observation) terms
  std::vector<PairIdx> blk_dst;
  std::vector<uint32_t> diag_dst;
  std::vector<uint32_t> dup_off;
  PairList dup_pairs;
  std::vector<uint32_t> tr_list_off, tr_list, tr_prob;
  std::vector<PairIdx> tile_slot;  // per tile: partial slot of its row side, column side
  std::vector<uint32_t> tile_meta;  // per tile: ij, row slot, column slot (or kNone), problem
  std::vector<uint32_t> chunk_point_begin;

  // Builder working memory (each term's column), kept with the plan so that
  // a rebuild in place reuses its pages; never uploaded.
  std::vector<uint32_t, NoInit<uint32_t>> scratch;

  // statistics (per plan)
  uint64_t real_var_cams = 0;
  uint64_t var_points = 0;
  uint64_t var_obs = 0;          // observations with a variable point
  uint64_t camera_pairs = 0;     // nonzero off-diagonal blocks (N_e)
  uint64_t num_pairs = 0;        // point contributions to those blocks
  // The terms (pairs) are not on the host: the device writes num_pairs of
  // them at upload, per block in point order as the host build would; the
  // block structure (blk_off, blk_dst, tiles) and blk_col, each block's
  // column slot, are the host's.
  bool pairs_on_device = false;
  std::vector<uint32_t> blk_col;
  std::vector<uint32_t> row_blk;   // [num_var_cams + 1] first block of each row

  size_t device_bytes() const;
  size_t upload_bytes() const;  // bytes copied host -> device by an upload
};

// Per-problem outcome of validation (BaError order of lm.rs:168-229).
struct Validation {
  int status = VLBA_OK;
  uint64_t error_index = 0;
};

// Resolve a vlba_camera into DevCamera; false if the model is outside the
// radial pinhole family (the caller declines).
bool resolve_camera(const vlba_camera& c, DevCamera* out);

// Validate one problem and its config without building anything.
Validation validate_problem(const vlba_problem* p, const vlba_config* cfg);

LmParams make_params(const vlba_config* cfg);

// The off-diagonal block structure of one problem's reduced system, found
// elsewhere (on the device) from the plan's point-major observations: per
// variable slot i, its columns j < i that share a variable point with it,
// ascending, and the number of terms (shared points) of each.  The builder
// then lays out everything but the terms themselves, which the device
// writes in the same order as the host build (Plan::pairs_on_device).
struct RowBlocks {
  std::vector<uint32_t> row_off;  // [nvar + 1] into col / count
  std::vector<uint32_t> col;      // per row, ascending
  std::vector<uint32_t> count;    // terms of each (row, col) block
};
// Returns false when some point has two observations in one slot (same-
// camera terms), which the host build handles, or when the device cannot
// take the problem; the builder then builds the terms on the host.
using RowBlocksFn = std::function<bool(const Plan& P, uint32_t nvar, RowBlocks* out)>;

// Build the plan for `n` problems (all must have validated OK); with n > 1
// each problem is built on its own host thread and the parts are merged;
// one large problem splits its pair counting over up to `max_threads` threads
// (0: all the host's).  `tb` is the tile size in blocks.  With n == 1 and
// `device_rows`, the block structure comes from device_rows and the terms are
// left to the device (Plan::pairs_on_device) when it succeeds.  Throws
// std::runtime_error on internal inconsistency.
void build_plan(const vlba_problem* const* problems, const vlba_config* const* configs,
                uint32_t n, uint32_t tb, Plan* plan, uint32_t max_threads = 0,
                const RowBlocksFn* device_rows = nullptr);

// The layout of a reduced camera system given directly (n nodes, sorted
// edges (a, b), a < b): its tiles, block destinations and PCG lists, with no
// observations; `params` carries the PCG tolerance and iteration cap.
void build_reduced_plan(uint32_t n, const uint32_t* edges, uint64_t ne, uint32_t tb,
                        const LmParams& params, Plan* plan);

// The structure of a point elimination (ReducedSolveAccelerator::eliminate)
// from which the device builds its pair index: the sorted edges by first
// node, and per node its camera-point blocks in ascending point order.
struct ElimIndex {
  uint32_t n = 0;
  uint32_t num_points = 0;
  uint64_t num_edges = 0;
  uint64_t num_obs = 0;
  std::vector<uint32_t> row_off;                      // [n + 1] edges (s, _)
  std::vector<uint32_t> edge_t;                       // [num_edges] second node
  std::vector<uint32_t> slot_off;                     // [n + 1]
  std::vector<uint32_t, NoInit<uint32_t>> slot_obs;   // [num_obs] blocks by node, then point
  std::vector<uint32_t, NoInit<uint32_t>> obs_point;  // [num_obs]
  std::vector<uint32_t> point_off;                    // [num_points + 1] (32-bit)
};

// Builds it for n nodes, ne sorted edges and num_points points (their nodes
// point_nodes[point_off[p] .. point_off[p + 1]], ascending) on the host's
// threads.  Returns an empty string, or the first inconsistency found
// (unsorted edges, a node out of range or out of order, a size past the
// 32-bit indices); a pair of nodes with no edge is found on the device.
std::string build_elimination_index(uint32_t n, const uint32_t* edges, uint64_t ne,
                                    uint32_t num_points, const uint64_t* point_off,
                                    const uint32_t* point_nodes, ElimIndex* out);

// Concatenate plans (built by build_plan) into one batch plan: indices are
// offset, each problem's layout and order are kept, so a problem solves the
// same in the merged plan as in its own.
void merge_plans(const std::vector<const Plan*>& parts, Plan* out);

// Bounds-check every index array of the plan against the arrays it indexes.
// Returns an empty string when the plan is consistent.
std::string check_plan(const Plan& plan);

// Algorithmic bytes of one LM iteration (linearisation + one trial with
// `pcg_iterations` PCG iterations) under the byte model of the headline
// roofline: B_lin + B_asm + k B_pcg + B_bs + B_cost.
double algorithmic_bytes(const Plan& plan, double pcg_iterations, double* b_pcg_out);

}  // namespace vlba
