// vlba_solver.cu -- solver context, device upload, the LM driver and the C ABI
// of include/visloc_ba_cuda.h.
//
// The LM loop runs on the device (k_decide owns accept/reject and lambda);
// the host only issues the per-iteration kernel sequence and polls a 4-byte
// "all done" word per iteration.  The reference's host loop instead reads
// back the step and evaluates the cost on the CPU every iteration
// (crates/ba-gpu/src/solver.rs:514-548, 696-727).

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <unordered_map>
#include <string>
#include <vector>

#include "vlba_kernels.cuh"
#include "vlba_gnc.h"
#include "vlba_plan.h"

namespace vlba {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const char* what)
      : std::runtime_error(std::string(what) + ": " + cudaGetErrorString(c)), code(c) {}
};

#define VLBA_CUDA(expr)                                   \
  do {                                                    \
    cudaError_t e_ = (expr);                              \
    if (e_ != cudaSuccess) throw ::vlba::CudaError(e_, #expr);    \
  } while (0)

struct Status : std::runtime_error {
  int code;
  uint64_t index;
  Status(int c, const std::string& m, uint64_t i = 0) : std::runtime_error(m), code(c), index(i) {}
};

// A device allocation freed with its holder (cudaFree waits for the work
// that uses it).
struct DeviceArray {
  void* p = nullptr;
  size_t bytes = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  void alloc(size_t n) {
    reset();
    VLBA_CUDA(cudaMalloc(&p, std::max<size_t>(n, 16)));
    bytes = n;
  }
  // At least n bytes, keeping the allocation when it is large enough.
  void ensure(size_t n) {
    if (!p || bytes < n) alloc(n);
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// The state of the context's last point elimination: the structure's pair
// index on the device (kept while the structure id and sizes stay the same),
// the camera-point blocks (kept while the linearization id does), and the
// blocks it formed, which a reduced solve with no off-diagonal blocks uses.
struct ElimState {
  uint64_t structure_id = 0;
  uint64_t linearization_id = 0;
  bool hcp_valid = false;
  bool blocks_valid = false;
  uint32_t n = 0, num_points = 0;
  uint64_t num_edges = 0, num_obs = 0, num_pairs = 0;
  std::vector<uint32_t> edges;  // the structure's edges (2 per edge), for the solve's check
  DeviceArray row_off, edge_t, pair_off, pairs, obs_point, slot_off, slot_obs, point_off32,
      point_nodes, cursor, flag;
  DeviceArray hcp64, hcp32, sk32, vinv64, used, extra_of, extra64, blocks, run_edges, run_out,
      coarse_out;
};

// A slab allocation that does not fit (the upload is redone on a larger slab).
struct SlabFull : std::runtime_error {
  size_t need;
  explicit SlabFull(size_t n) : std::runtime_error("slab exhausted"), need(n) {}
};

// Device memory owned by a context: bump allocation inside one slab.  A
// context's slab grows to the largest upload it has seen (capacity-grown, so
// repeated solves of similar sizes allocate nothing); a serving slot's slab
// is fixed at creation (use_slab) and never grows.
class Arena {
 public:
  ~Arena() {
    release();
    if (slab_) cudaFree(slab_);
  }
  void use_slab(size_t bytes) {
    set_slab(bytes);
    growable_ = false;
  }
  // Make room for an upload of about `bytes` and reset the bump pointer.
  void reserve(size_t bytes) {
    release();
    if (slab_ && slab_size_ >= bytes) return;
    if (!growable_) throw CudaError(cudaErrorMemoryAllocation, "request exceeds the slot's memory");
    set_slab(bytes);
  }
  bool growable() const { return growable_; }
  size_t capacity() const { return slab_size_; }
  template <typename T>
  T* alloc(size_t count) {
    if (count == 0) count = 1;
    const size_t need = count * sizeof(T);
    if (slab_) {
      const size_t off = (slab_used_ + 255) / 256 * 256;
      if (off + need > slab_size_) {
        if (growable_) throw SlabFull(off + need);
        throw CudaError(cudaErrorMemoryAllocation, "slab exhausted");
      }
      slab_used_ = off + need;
      bytes_ += need;
      return reinterpret_cast<T*>(static_cast<char*>(slab_) + off);
    }
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw CudaError(e, "cudaMalloc");
    }
    ptrs_.push_back(p);
    bytes_ += need;
    return static_cast<T*>(p);
  }
  void release() {
    for (void* p : ptrs_) cudaFree(p);
    ptrs_.clear();
    bytes_ = 0;
    slab_used_ = 0;
  }
  size_t bytes() const { return bytes_; }

 private:
  void set_slab(size_t bytes) {
    release();
    if (slab_) cudaFree(slab_);
    slab_ = nullptr;
    slab_size_ = 0;
    const cudaError_t e = cudaMalloc(&slab_, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      slab_ = nullptr;
      throw CudaError(e, "cudaMalloc (slab)");
    }
    slab_size_ = bytes;
  }
  std::vector<void*> ptrs_;
  size_t bytes_ = 0;
  void* slab_ = nullptr;
  size_t slab_size_ = 0, slab_used_ = 0;
  bool growable_ = true;
};

// Serialises the persistent PCG kernels of several contexts sharing a GPU
// (each launch waits for the previous one of any context): two cooperative
// grids never wait on each other's resources.
struct PcgGate {
  std::mutex mu;
  cudaEvent_t last = nullptr;
};

struct Context {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  // The camera-diagonal sums run on `side` beside the off-diagonal assembly
  // (fork and join events on `stream`; both kernels are latency-bound and
  // write disjoint blocks).
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaEvent_t ev[6] = {};
  std::string error;
  Arena arena;
  Plan plan;
  Dev dev;
  bool uploaded = false;
  int pcg_grid = 0;
  uint32_t flags = 0;  // flags of the uploaded config
  size_t l2_bytes = 0;
  double l2_fraction = 0.5;  // share of the L2 that keeps S resident in PCG
  int pcg_grid_hint = 0;     // blocks of the PCG launch (trace sizing)
  // the uploaded problems' sizes (for download)
  std::vector<uint64_t> num_poses, num_points;
  // batch upload: input index -> problem of the plan (-1: failed validation)
  std::vector<int> batch_slot;
  // the LM loop of the current upload captured as one graph (VLBA_FLAG_GRAPH)
  cudaGraphExec_t graph = nullptr;
  uint32_t graph_iters = 0;
  PcgGate* gate = nullptr;  // set for the slots of a server
  bool tuned = false;       // the launch shape of this upload has been chosen
  // Pinned staging for uploads and downloads: two buffers of stage_cap bytes,
  // each refilled once the device copy out of it (its event) has completed.
  char* stage[2] = {nullptr, nullptr};
  size_t stage_cap = 0;
  cudaEvent_t stage_ev[2] = {};
  // Per-observation squared residuals of a GNC solve (grown on demand).
  double* gnc_sq = nullptr;
  size_t gnc_cap = 0;
  // The last point elimination (ReducedSolveAccelerator::eliminate).
  std::unique_ptr<ElimState> elim;
  // Device times of the last reduced solve and elimination.
  vlba_reduced_timing reduced_ms{};
  // Uploads of a plan (any entry point); the reduced system's layout is
  // reused while no other plan replaced it and its edges stay the same.
  uint64_t plan_generation = 0;
  uint64_t reduced_generation = ~0ull;
  std::vector<uint32_t> reduced_edges;
  uint32_t reduced_nodes = 0;
  // The reduced system's diagonal, rhs and blocks as copied from the caller,
  // and the preconditioner of a preconditioned solve.
  DeviceArray reduced_in, reduced_pre;
  // Scratch of the device-built Schur terms (vlba_pairs.cu): the plan arrays
  // the row counts read, the per-row lists and the flags.
  DeviceArray rows_in, rows_out;
  // Where rows_in holds the plan arrays the row counts read (byte offsets of
  // cam_off, cam_obs, obs_point, obs_slot, point_var, pt_off), valid for the
  // plan built last with its terms on the device: its upload copies them from
  // there instead of from the host again.
  size_t rows_in_at[6] = {0, 0, 0, 0, 0, 0};
  uint64_t last_upload_bytes = 0;
  // Host milliseconds of the last upload's device-side steps (for the
  // VLBA_TRACE_UPLOAD line): array copies issued, then the device terms.
  double up_copy_ms = 0.0, up_terms_ms = 0.0, up_flush_ms = 0.0;
};

namespace {

void set_device(Context* c) { VLBA_CUDA(cudaSetDevice(c->device)); }

void drop_graph(Context* c) {
  if (c->graph) cudaGraphExecDestroy(c->graph);
  c->graph = nullptr;
  c->graph_iters = 0;
}

// L2-resident share of S: the leading tiles up to a fraction of the L2.
uint32_t l2_tiles(const Context* c, double frac) {
  const double tile_bytes = (double)c->plan.tb * c->plan.tb * kBlock * 4.0;
  return (uint32_t)std::min<double>((double)c->plan.tile_ij.size(),
                                    frac * (double)c->l2_bytes / tile_bytes);
}

// ---------------------------------------------------------------- autotuner
// Launch shapes that leave every result bit for bit the same (the PCG's
// blocks and the L2-resident share of S: every sum's order is fixed by the
// plan, not by which block or warp computes it), chosen by timing a fixed
// number of PCG iterations on the uploaded system and cached per system
// shape for the process.  The tile size and the assembly's lane count set
// summation orders, so they are not tuned: a problem must solve the same
// alone and in any batch.
struct ShapeKey {
  uint32_t tiles, rows, problems;
  bool operator<(const ShapeKey& o) const {
    return std::tie(tiles, rows, problems) < std::tie(o.tiles, o.rows, o.problems);
  }
};
struct LaunchShape {
  int pcg_grid = 0;
  double l2_fraction = 0.5;
  double pcg_iteration_us = 0.0;
};
std::mutex g_tune_mu;
std::map<ShapeKey, LaunchShape> g_tune_cache;

uint32_t log2_bucket(uint64_t v) {
  uint32_t b = 0;
  while (v > 1) {
    v >>= 1;
    ++b;
  }
  return b;
}

ShapeKey shape_key(const Plan& P) {
  return ShapeKey{log2_bucket(P.tile_ij.size()), log2_bucket(P.num_tile_rows),
                  log2_bucket(P.num_problems)};
}

int pcg_grid_max(const Context* c) {
  const Plan& P = c->plan;
  const int g = P.num_tile_rows ? pcg_grid_size((int)P.tb, c->sm_count) : 0;
  return std::min<int>(g, (int)std::max<size_t>(P.tile_ij.size(), P.num_tile_rows));
}

int pcg_grid_min(const Context* c) {
  const int per = pcg_rows_per_block();
  return (int)((c->plan.num_tile_rows + per - 1) / per);
}

void apply_shape(Context* c, const LaunchShape& sh) {
  const int gmax = pcg_grid_max(c), gmin = std::max(1, pcg_grid_min(c));
  if (gmax > 0) c->pcg_grid = std::max(gmin, std::min(gmax, sh.pcg_grid > 0 ? sh.pcg_grid : gmax));
  c->dev.l2_resident_tiles = l2_tiles(c, std::max(0.0, std::min(1.0, sh.l2_fraction)));
}

// memcpy, split over host threads from 8 MB up.
void par_memcpy(void* dst, const void* src, size_t n) {
  const size_t kPart = 4u << 20;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned T = (unsigned)std::min<size_t>(std::min(hw, 16u), n / kPart);
  char* d = static_cast<char*>(dst);
  const char* s = static_cast<const char*>(src);
  if (T <= 1) {
    std::memcpy(d, s, n);
    return;
  }
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < T; ++t)
    pool.emplace_back([=] {
      const size_t a = n * t / T, e = n * (t + 1) / T;
      std::memcpy(d + a, s + a, e - a);
    });
  std::memcpy(d, s, n / T);
  for (auto& th : pool) th.join();
}

// The context's two pinned staging buffers with at least `want` bytes each
// (at most 64 MB); false when no pinned memory can be had.  They grow to at
// least 16 MB and at least double, so that uploads of growing sizes (a
// serving slot's batches) reallocate them a few times at most: freeing
// pinned memory waits for the device.
constexpr size_t kStageMax = 64u << 20;
bool reserve_stage(Context* c, size_t want) {
  constexpr size_t kMin = 16u << 20, kGrain = 1u << 20;
  want = std::min(kStageMax, (want + kGrain - 1) / kGrain * kGrain);
  if (c->stage_cap >= want) return true;
  want = std::min(kStageMax, std::max({want, kMin, 2 * c->stage_cap}));
  for (int i = 0; i < 2; ++i) {
    if (c->stage_ev[i]) VLBA_CUDA(cudaEventSynchronize(c->stage_ev[i]));
    else VLBA_CUDA(cudaEventCreateWithFlags(&c->stage_ev[i], cudaEventDisableTiming));
    if (c->stage[i]) cudaFreeHost(c->stage[i]);
    c->stage[i] = nullptr;
  }
  c->stage_cap = 0;
  for (int i = 0; i < 2; ++i) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, want, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      if (c->stage[0]) cudaFreeHost(c->stage[0]);
      c->stage[0] = nullptr;
      return false;
    }
    c->stage[i] = static_cast<char*>(p);
  }
  c->stage_cap = want;
  return true;
}

// Host -> device copies of an upload through the context's pinned staging
// buffers: the host copies the next piece into one buffer (on several
// threads when it is large) while the device copies the previous piece out
// of the other.  Copies from pageable memory directly when no pinned memory
// can be had.
class Stager {
 public:
  explicit Stager(Context* c) : c_(c) {}
  template <typename T, typename A>
  T* up(Arena& arena, const std::vector<T, A>& v) {
    T* p = arena.alloc<T>(v.size());
    add(p, v.data(), v.size() * sizeof(T));
    return p;
  }
  void add(void* dst, const void* src, size_t bytes) {
    if (!bytes) return;
    const Item it{static_cast<char*>(dst), static_cast<const char*>(src), bytes};
    // Page-locked plan arrays go straight to the device.
    if (pinned_range(src, bytes)) direct_.push_back(it);
    else items_.push_back(it);
  }
  void flush(cudaStream_t s) {
    for (const Item& it : direct_)
      VLBA_CUDA(cudaMemcpyAsync(it.dst, it.src, it.bytes, cudaMemcpyHostToDevice, s));
    direct_.clear();
    size_t total = 0;
    for (const Item& it : items_) total += it.bytes;
    if (total == 0) return;
    if (!reserve_stage(c_, total)) {
      for (const Item& it : items_)
        VLBA_CUDA(cudaMemcpyAsync(it.dst, it.src, it.bytes, cudaMemcpyHostToDevice, s));
      items_.clear();
      return;
    }
    const size_t cap = c_->stage_cap;
    int b = 0;
    size_t fill = 0;
    struct Piece {
      char* dst;
      size_t off, bytes;
    };
    std::vector<Piece> pending;
    VLBA_CUDA(cudaEventSynchronize(c_->stage_ev[0]));
    auto issue = [&]() {
      for (const Piece& q : pending)
        VLBA_CUDA(cudaMemcpyAsync(q.dst, c_->stage[b] + q.off, q.bytes, cudaMemcpyHostToDevice, s));
      VLBA_CUDA(cudaEventRecord(c_->stage_ev[b], s));
      pending.clear();
      b ^= 1;
      fill = 0;
      VLBA_CUDA(cudaEventSynchronize(c_->stage_ev[b]));
    };
    for (const Item& it : items_) {
      for (size_t off = 0; off < it.bytes;) {
        const size_t n = std::min(it.bytes - off, cap - fill);
        if (n == 0) {
          issue();
          continue;
        }
        par_memcpy(c_->stage[b] + fill, it.src + off, n);
        pending.push_back(Piece{it.dst + off, fill, n});
        fill = std::min(cap, (fill + n + 255) / 256 * 256);
        off += n;
      }
    }
    if (!pending.empty()) issue();
    items_.clear();
  }

 private:
  struct Item {
    char* dst;
    const char* src;
    size_t bytes;
  };
  Context* c_;
  std::vector<Item> items_, direct_;
};

// Upload a built plan: allocate and fill every device array of Dev.
void check_launch(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(e, what);
}

// `before_kernels` (if set) runs before the first kernel that reads the
// plan's arrays: the copies may start while the host still checks the plan.
void upload_plan_once(Context* c, uint32_t max_records, const std::function<void()>& before_kernels) {
  Plan& P = c->plan;
  cudaStream_t s = c->stream;
  drop_graph(c);  // its kernels hold the old device pointers
  c->arena.release();
  c->uploaded = false;
  Dev d;
  std::memset(&d, 0, sizeof d);
  const auto u0 = std::chrono::steady_clock::now();
  const size_t npose = P.pose_prob.size(), npt = P.point_prob.size(), nobs = P.obs_pose.size();
  d.num_problems = P.num_problems;
  d.num_poses = (uint32_t)npose;
  d.num_points = (uint32_t)npt;
  d.num_obs = (uint32_t)nobs;
  d.num_var_cams = P.num_var_cams;
  d.num_tile_rows = P.num_tile_rows;
  d.num_tiles = (uint32_t)P.tile_ij.size();
  d.num_offdiag_blocks = (uint32_t)P.blk_dst.size();
  d.num_dup_pairs = (uint32_t)P.dup_pairs.size();
  d.num_point_chunks = (uint32_t)P.chunk_point_begin.size() - 1;
  d.tb = P.tb;
  d.group = P.group;
  Arena& A = c->arena;
  Stager st(c);
  d.prob_pose_begin = st.up(A, P.prob_pose_begin);
  d.prob_point_begin = st.up(A, P.prob_point_begin);
  d.prob_tr_begin = st.up(A, P.prob_tr_begin);
  d.prob_chunk_begin = st.up(A, P.prob_chunk_begin);
  d.pose_prob = st.up(A, P.pose_prob);
  d.point_prob = st.up(A, P.point_prob);
  d.slot_prob = st.up(A, P.slot_prob);
  d.params = st.up(A, P.params);
  d.ctrl = A.alloc<Ctrl>(P.num_problems);
  d.pcg = A.alloc<PcgState>(P.num_problems);
  d.max_records = max_records;
  d.records = A.alloc<vlba_iteration>((size_t)P.num_problems * (max_records ? max_records : 1));
  for (int b = 0; b < 2; ++b) {
    d.pose_q[b] = A.alloc<double>(4 * npose);
    d.pose_t[b] = A.alloc<double>(3 * npose);
    d.pose_rt[b] = A.alloc<double>(12 * npose);
    d.points[b] = A.alloc<double>(3 * npt);
  }
  d.init_pose_q = st.up(A, P.pose_q);
  d.init_pose_t = st.up(A, P.pose_t);
  d.init_points = st.up(A, P.points);
  // With the terms built on the device, the arrays its row counts read are
  // on the device already: copied from there, not sent again.
  auto from_rows = [&](const auto& v, int k) {
    using T = typename std::decay_t<decltype(v)>::value_type;
    T* p = A.alloc<T>(v.size());
    if (!v.empty())
      VLBA_CUDA(cudaMemcpyAsync(p, c->rows_in.as<char>() + c->rows_in_at[k], v.size() * sizeof(T),
                                cudaMemcpyDeviceToDevice, s));
    return p;
  };
  const bool reuse = P.pairs_on_device;
  d.pose_slot = st.up(A, P.pose_slot);
  d.point_var = reuse ? from_rows(P.point_var, 4) : st.up(A, P.point_var);
  d.pose_step = A.alloc<double>(npose);
  d.cameras = st.up(A, P.cameras);
  d.pt_off = reuse ? from_rows(P.pt_off, 5) : st.up(A, P.pt_off);
  d.obs_point = reuse ? from_rows(P.obs_point, 2) : st.up(A, P.obs_point);
  d.obs_pose = st.up(A, P.obs_pose);
  d.obs_cam = st.up(A, P.obs_cam);
  d.obs_slot = reuse ? from_rows(P.obs_slot, 3) : st.up(A, P.obs_slot);
  {
    double2* xy = A.alloc<double2>(nobs);
    st.add(xy, P.obs_xy.data(), nobs * 16);
    d.obs_xy = xy;
  }
  d.obs_w = P.obs_w.empty() ? nullptr : st.up(A, P.obs_w);
  d.obs_kind = P.obs_kind.empty() ? nullptr : st.up(A, P.obs_kind);
  d.obs_st = P.obs_kind.empty() ? nullptr : reinterpret_cast<const double2*>(st.up(A, P.obs_st));
  d.obs_rcam = P.obs_kind.empty() ? nullptr : st.up(A, P.obs_rcam);
  d.obs_h = A.alloc<float4>(2 * nobs);
  d.obs_e = A.alloc<float4>(nobs);
  d.pt_p = A.alloc<float4>(2 * npt);
  d.cam_off = reuse ? from_rows(P.cam_off, 0) : st.up(A, P.cam_off);
  d.cam_obs = reuse ? from_rows(P.cam_obs, 1) : st.up(A, P.cam_obs);
  d.cam_pt = A.alloc<uint32_t>(P.cam_obs.size());
  d.pt_h = A.alloc<float>(9 * npt);
  d.pt_s = A.alloc<float4>(4 * npt);
  d.pt_c = A.alloc<double>(12 * npt);
  d.cam_hpp = nullptr;
  const size_t tile_floats = (size_t)P.tb * P.tb * kBlock;
  d.tiles = A.alloc<float>(P.tile_ij.size() * tile_floats);
  VLBA_CUDA(cudaMemsetAsync(d.tiles, 0, P.tile_ij.size() * tile_floats * 4, s));
  d.tile_ij = st.up(A, P.tile_ij);
  d.blk_off = st.up(A, P.blk_off);
  uint2* dev_pairs = nullptr;
  const uint32_t* dev_row_blk = nullptr;
  const uint32_t* dev_blk_col = nullptr;
  if (P.pairs_on_device) {
    dev_pairs = A.alloc<uint2>(P.num_pairs);
    d.pairs = dev_pairs;
    dev_row_blk = st.up(A, P.row_blk);
    dev_blk_col = st.up(A, P.blk_col);
  } else {
    d.pairs = reinterpret_cast<const uint2*>(st.up(A, P.pairs));
  }
  const uint64_t npairs = P.pairs_on_device ? P.num_pairs : P.pairs.size();
  d.pair_pt = A.alloc<uint32_t>(npairs);
  d.blk_dst = reinterpret_cast<const uint2*>(st.up(A, P.blk_dst));
  d.ord_range = A.alloc<uint2>(P.blk_dst.size());
  d.ord_dst = A.alloc<uint2>(P.blk_dst.size());
  d.long_range = A.alloc<uint2>(P.blk_dst.size());
  d.long_dst = A.alloc<uint2>(P.blk_dst.size());
  d.num_long = A.alloc<uint32_t>(1);
  d.diag_dst = st.up(A, P.diag_dst);
  d.dup_off = st.up(A, P.dup_off);
  d.dup_pairs = reinterpret_cast<const uint2*>(st.up(A, P.dup_pairs));
  const size_t nvec = (size_t)P.num_var_cams * 6;
  d.minv = A.alloc<float>(36 * (size_t)P.num_var_cams);
  d.rhs = A.alloc<float>(nvec);
  d.x = A.alloc<float>(nvec);
  d.r = A.alloc<float>(nvec);
  d.z = A.alloc<float>(nvec);
  d.p = A.alloc<float>(nvec);
  d.q = A.alloc<float>(nvec);
  VLBA_CUDA(cudaMemsetAsync(d.x, 0, nvec * 4, s));
  d.partial = A.alloc<float>(P.tr_list.size() * (size_t)P.tb * 6);
  d.tile_slot = reinterpret_cast<const uint2*>(st.up(A, P.tile_slot));
  d.tile_meta = reinterpret_cast<const uint4*>(st.up(A, P.tile_meta));
  d.tr_list_off = st.up(A, P.tr_list_off);
  d.tr_list = st.up(A, P.tr_list);
  d.tr_prob = st.up(A, P.tr_prob);
  d.dots = A.alloc<double>(9 * (size_t)(P.num_tile_rows ? P.num_tile_rows : 1));
  d.l2_resident_tiles = l2_tiles(c, c->l2_fraction);
  d.trace = nullptr;
  if (std::getenv("VLBA_TRACE_PCG") && c->pcg_grid_hint > 0)
    d.trace = A.alloc<unsigned long long>((size_t)kTraceIters * c->pcg_grid_hint *
                                          (kTracePhases + 2 * 32 + 32 * 8 * 4));
  d.barrier = A.alloc<unsigned int>(kBarrierWords);
  d.error = A.alloc<unsigned int>(1);
  VLBA_CUDA(cudaMemsetAsync(d.barrier, 0, 4 * kBarrierWords, s));
  VLBA_CUDA(cudaMemsetAsync(d.error, 0, 4, s));
  d.chunk_point_begin = st.up(A, P.chunk_point_begin);
  const size_t nch = P.chunk_point_begin.size() - 1;
  d.chunk_cost = A.alloc<double>(nch);
  d.chunk_bad = A.alloc<unsigned long long>(nch);
  d.chunk_step = A.alloc<double>(nch);
  const auto uf = std::chrono::steady_clock::now();
  st.flush(s);
  c->dev = d;
  const auto u1 = std::chrono::steady_clock::now();
  c->up_flush_ms = std::chrono::duration<double, std::milli>(u1 - uf).count();
  c->up_copy_ms = std::chrono::duration<double, std::milli>(u1 - u0).count();
  if (before_kernels) before_kernels();
  check_launch(launch_cam_points(d, (uint32_t)P.cam_obs.size(), s), "camera lists");
  check_launch(launch_block_order(d, s), "block order");
  uint32_t num_long = 0;
  if (d.num_offdiag_blocks)
    VLBA_CUDA(cudaMemcpyAsync(&num_long, d.num_long, 4, cudaMemcpyDeviceToHost, s));
  if (P.pairs_on_device) {
    // The terms, from the uploaded point-major observations and per-slot
    // lists, at the places the host laid out; checked as they are written.
    RowsDev r{};
    r.nvar = P.row_blk.size() > 0 ? (uint32_t)P.row_blk.size() - 1 : 0u;
    r.cam_off = d.cam_off;
    r.cam_obs = d.cam_obs;
    r.obs_point = d.obs_point;
    r.obs_slot = d.obs_slot;
    r.point_var = d.point_var;
    r.pt_off = d.pt_off;
    c->rows_out.ensure(16);
    r.flags = c->rows_out.as<uint32_t>();
    VLBA_CUDA(cudaMemsetAsync(r.flags, 0, 4, s));
    uint32_t max_row_blocks = 0;
    for (uint32_t i = 0; i < r.nvar; ++i)
      max_row_blocks = std::max(max_row_blocks, P.row_blk[i + 1] - P.row_blk[i]);
    check_launch(launch_rows_place(r, d.blk_off, dev_row_blk, dev_blk_col, max_row_blocks, dev_pairs,
                                   d.pair_pt, s),
                 "Schur terms");
    uint32_t flags = 0;
    VLBA_CUDA(cudaMemcpyAsync(&flags, r.flags, 4, cudaMemcpyDeviceToHost, s));
    VLBA_CUDA(cudaStreamSynchronize(s));
    if (flags) throw std::runtime_error("device Schur terms do not match the plan's blocks");
  }
  if (!P.pairs_on_device) check_launch(launch_pair_points(d, npairs, s), "term points");
  c->up_terms_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - u1).count();
  // Co-resident grid, but no more blocks than tiles or tile rows to work on
  // (fewer blocks make the grid barriers cheaper on small systems).
  c->pcg_grid = P.num_tile_rows ? pcg_grid_size((int)P.tb, c->sm_count) : 0;
  c->pcg_grid = std::min<int>(c->pcg_grid,
                              (int)std::max<size_t>(P.tile_ij.size(), P.num_tile_rows));
  if (c->pcg_grid > 0 && (size_t)c->pcg_grid * pcg_rows_per_block() < P.num_tile_rows)
    throw Status(VLBA_ERR_INVALID_ARGUMENT,
                 "reduced system too large: more than " + std::to_string(pcg_rows_per_block()) +
                     " tile rows per PCG block");
  if (P.num_tile_rows && c->pcg_grid <= 0)
    throw Status(VLBA_ERR_CUDA, "the PCG kernel cannot be made co-resident on this device");
  // A launch shape tuned earlier for a system of this shape.
  c->tuned = false;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(shape_key(P));
    if (it != g_tune_cache.end()) {
      apply_shape(c, it->second);
      c->tuned = true;
    }
  }
  if (c->dev.trace && c->pcg_grid > c->pcg_grid_hint) c->dev.trace = nullptr;  // sized for fewer blocks
  VLBA_CUDA(cudaStreamSynchronize(s));
  if (num_long > c->dev.num_offdiag_blocks)
    throw std::runtime_error("long off-diagonal block count out of range");
  c->dev.num_long_blocks = num_long;
  c->uploaded = true;
}

void upload_plan(Context* c, uint32_t max_records,
                 const std::function<void()>& before_kernels = nullptr) {
  ++c->plan_generation;
  const size_t est = c->plan.device_bytes() + (size_t)max_records * sizeof(vlba_iteration) *
                                                   c->plan.num_problems + (4u << 20);
  if (c->arena.growable()) c->arena.reserve(std::max(est, c->arena.capacity()));
  try {
    upload_plan_once(c, max_records, before_kernels);
  } catch (const SlabFull& f) {
    // The estimate was short: one retry on a slab with room to spare.
    c->arena.reserve(std::max(2 * c->arena.capacity(), f.need + f.need / 2));
    upload_plan_once(c, max_records, before_kernels);
  }
}

// Reset the state to the uploaded initial values and the LM control words.
void reset_state(Context* c) {
  Dev& d = c->dev;
  const Plan& P = c->plan;
  cudaStream_t s = c->stream;
  VLBA_CUDA(cudaMemcpyAsync(d.pose_q[0], d.init_pose_q, P.pose_q.size() * 8, cudaMemcpyDeviceToDevice, s));
  VLBA_CUDA(cudaMemcpyAsync(d.pose_t[0], d.init_pose_t, P.pose_t.size() * 8, cudaMemcpyDeviceToDevice, s));
  VLBA_CUDA(cudaMemcpyAsync(d.points[0], d.init_points, P.points.size() * 8, cudaMemcpyDeviceToDevice, s));
  VLBA_CUDA(cudaMemsetAsync(d.ctrl, 0, sizeof(Ctrl) * P.num_problems, s));
  VLBA_CUDA(cudaMemsetAsync(d.error, 0, 4, s));
}


struct RunStats {
  double device_ms = 0.0;
  uint64_t launches = 0;
};

struct PhaseTimes {
  std::vector<double> lin, assemble, pcg, update;
};

// VLBA_TRACE_PCG: per-phase device time of the PCG iterations (mean over
// blocks of each phase's span, and the iteration's wall span), to stderr.
void dump_trace(Context* c) {
  const Dev& d = c->dev;
  const int G = c->pcg_grid;
  std::vector<unsigned long long> t((size_t)kTraceIters * G * kTracePhases);
  VLBA_CUDA(cudaMemcpyAsync(t.data(), d.trace, t.size() * 8, cudaMemcpyDeviceToHost, c->stream));
  PcgState pg;
  VLBA_CUDA(cudaMemcpyAsync(&pg, d.pcg, sizeof pg, cudaMemcpyDeviceToHost, c->stream));
  VLBA_CUDA(cudaStreamSynchronize(c->stream));
  const int iters = std::min<int>((int)pg.iters, kTraceIters - 1);
  double acc[kTracePhases] = {0};
  double wall = 0.0;
  for (int k = 0; k < iters; ++k) {
    unsigned long long lo = ~0ull, hi = 0;
    for (int b = 0; b < G; ++b) {
      const unsigned long long* r = &t[((size_t)k * G + b) * kTracePhases];
      for (int ph = 1; ph < kTracePhases; ++ph) acc[ph] += (double)(r[ph] - r[ph - 1]) / G;
      lo = std::min(lo, r[0]);
      hi = std::max(hi, r[kTracePhases - 1]);
    }
    wall += (double)(hi - lo);
  }
  const char* path = std::getenv("VLBA_TRACE_PCG");
  if (path && path[0] == '/') {  // raw dump: G, iterations, then the stamps
    if (FILE* f = std::fopen(path, "ab")) {
      const int32_t hdr[3] = {G, iters, kTracePhases};
      std::fwrite(hdr, sizeof hdr, 1, f);
      std::fwrite(t.data(), 8, (size_t)iters * G * kTracePhases, f);
      // Per-warp marks (warps per block from the kernel's configuration).
      const size_t tw = (size_t)G * 8;
      std::vector<unsigned long long> w((size_t)kTraceIters * tw * 2);
      VLBA_CUDA(cudaMemcpy(w.data(), d.trace + (size_t)kTraceIters * G * kTracePhases,
                           w.size() * 8, cudaMemcpyDeviceToHost));
      std::fwrite(w.data(), 8, (size_t)iters * tw * 2, f);
      std::vector<unsigned long long> tt((size_t)kTraceIters * tw * 8 * 4);
      VLBA_CUDA(cudaMemcpy(tt.data(), d.trace + (size_t)kTraceIters * G * kTracePhases +
                                          (size_t)kTraceIters * tw * 2,
                           tt.size() * 8, cudaMemcpyDeviceToHost));
      std::fwrite(tt.data(), 8, (size_t)iters * tw * 8 * 4, f);
      std::fclose(f);
    }
  }
  if (iters > 0)
    std::fprintf(stderr,
                 "vlba pcg trace: %u iterations, per iteration (us): status %.2f tiles %.2f "
                 "arrive+reduce %.2f barrier1 %.2f update %.2f barrier2 %.2f | span %.2f\n",
                 pg.iters, acc[1] / iters / 1e3, acc[2] / iters / 1e3, 0.0, acc[3] / iters / 1e3,
                 acc[4] / iters / 1e3, acc[5] / iters / 1e3, wall / iters / 1e3);
}

// The device LM loop over all uploaded problems.
// The kernels of one LM iteration (trial), in order; `ev` (4 events or null)
// brackets the phases for profiling.  Returns the number of launches.
uint64_t enqueue_iteration(Context* c, cudaEvent_t* ev) {
  Dev& d = c->dev;
  cudaStream_t s = c->stream;
  if (ev) VLBA_CUDA(cudaEventRecord(ev[0], s));
  check_launch(launch_linearize(d, s), "linearize");
  if (ev) VLBA_CUDA(cudaEventRecord(ev[1], s));
  check_launch(launch_point_prep(d, s), "point prep");
  // Camera blocks on the side stream beside the off-diagonal blocks.
  VLBA_CUDA(cudaEventRecord(c->fork, s));
  VLBA_CUDA(cudaStreamWaitEvent(c->side, c->fork, 0));
  check_launch(launch_cam_diag(d, c->side), "camera blocks");
  VLBA_CUDA(cudaEventRecord(c->join, c->side));
  check_launch(launch_offdiag(d, s), "off-diagonal blocks");
  VLBA_CUDA(cudaStreamWaitEvent(s, c->join, 0));
  check_launch(launch_pcg_setup(d, s), "pcg setup");
  if (ev) VLBA_CUDA(cudaEventRecord(ev[2], s));
  if (c->gate && d.num_tile_rows) {
    std::lock_guard<std::mutex> lock(c->gate->mu);
    VLBA_CUDA(cudaStreamWaitEvent(s, c->gate->last, 0));
    check_launch(launch_pcg(d, c->pcg_grid, s), "pcg");
    VLBA_CUDA(cudaEventRecord(c->gate->last, s));
  } else {
    check_launch(launch_pcg(d, c->pcg_grid, s), "pcg");
  }
  if (d.trace) dump_trace(c);
  if (ev) VLBA_CUDA(cudaEventRecord(ev[3], s));
  check_launch(launch_pose_update(d, s), "pose update");
  check_launch(launch_cost(d, true, s), "trial cost");
  check_launch(launch_decide(d, false, s), "decide");
  if (ev) VLBA_CUDA(cudaEventRecord(ev[4], s));
  // linearize, point prep, pcg setup, pose update, cost, decide always;
  // off-diagonal (short and long blocks), camera-diagonal and PCG kernels
  // when the system has them.
  return 6 + (d.num_offdiag_blocks ? 1 : 0) + (d.num_long_blocks ? 1 : 0) + (d.num_var_cams ? 1 : 0) +
         (d.num_tile_rows ? 1 : 0);
}

uint64_t enqueue_initial(Context* c) {
  Dev& d = c->dev;
  cudaStream_t s = c->stream;
  check_launch(launch_pose_table(d, s), "pose table");
  check_launch(launch_cost(d, false, s), "initial cost");
  check_launch(launch_decide(d, true, s), "init");
  return 3;
}

void check_device_error(Context* c) {
  unsigned int err = 0;
  VLBA_CUDA(cudaMemcpyAsync(&err, c->dev.error, 4, cudaMemcpyDeviceToHost, c->stream));
  VLBA_CUDA(cudaStreamSynchronize(c->stream));
  if (err)
    throw Status(VLBA_ERR_TIMEOUT,
                 "a bounded device wait gave up (error bits " + std::to_string(err) + ")");
}

// The LM loop with VLBA_FLAG_GRAPH: the initial cost and max_iters
// iterations captured once per upload as one CUDA graph and replayed; no
// host synchronisation between iterations (the kernels of a problem that has
// finished return at once).
RunStats run_lm_graph(Context* c, uint32_t max_iters) {
  cudaStream_t s = c->stream;
  RunStats st;
  uint64_t launches = 0;
  if (!c->graph || c->graph_iters != max_iters) {
    drop_graph(c);
    cudaGraph_t g = nullptr;
    VLBA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      launches += enqueue_initial(c);
      for (uint32_t it = 0; it < max_iters; ++it) launches += enqueue_iteration(c, nullptr);
    } catch (...) {
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    VLBA_CUDA(cudaStreamEndCapture(s, &g));
    const cudaError_t e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      c->graph = nullptr;
      throw CudaError(e, "cudaGraphInstantiate");
    }
    c->graph_iters = max_iters;
  } else {
    launches = 3;
    for (uint32_t it = 0; it < max_iters; ++it) {
      const Dev& d = c->dev;
      launches += 6 + (d.num_offdiag_blocks ? 1 : 0) + (d.num_var_cams ? 1 : 0) +
                  (d.num_tile_rows ? 1 : 0);
    }
  }
  VLBA_CUDA(cudaEventRecord(c->ev[0], s));
  VLBA_CUDA(cudaGraphLaunch(c->graph, s));
  VLBA_CUDA(cudaEventRecord(c->ev[5], s));
  check_device_error(c);
  float ms = 0.f;
  VLBA_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[5]));
  st.device_ms = ms;
  st.launches = launches;
  return st;
}

LaunchShape autotune(Context* c);

RunStats run_lm(Context* c, bool profile, PhaseTimes* pt) {
  if ((c->flags & VLBA_FLAG_AUTOTUNE) && !c->tuned) {
    autotune(c);
    reset_state(c);
  }
  Dev& d = c->dev;
  cudaStream_t s = c->stream;
  uint32_t max_iters = 0;
  for (const LmParams& lp : c->plan.params) max_iters = std::max(max_iters, lp.max_iterations);
  if ((c->flags & VLBA_FLAG_GRAPH) && !profile && !d.trace) return run_lm_graph(c, max_iters);
  RunStats st;
  std::vector<Ctrl> ctrl(c->plan.num_problems);
  VLBA_CUDA(cudaEventRecord(c->ev[0], s));
  st.launches += enqueue_initial(c);
  for (uint32_t it = 0; it < max_iters; ++it) {
    st.launches += enqueue_iteration(c, profile ? c->ev + 1 : nullptr);
    // Poll the per-problem control words (one small copy per iteration).
    VLBA_CUDA(cudaMemcpyAsync(ctrl.data(), d.ctrl, sizeof(Ctrl) * ctrl.size(), cudaMemcpyDeviceToHost, s));
    unsigned int err = 0;
    VLBA_CUDA(cudaMemcpyAsync(&err, d.error, 4, cudaMemcpyDeviceToHost, s));
    VLBA_CUDA(cudaStreamSynchronize(s));
    if (profile) {
      float a = 0.f, b = 0.f, e = 0.f, f = 0.f;
      VLBA_CUDA(cudaEventElapsedTime(&a, c->ev[1], c->ev[2]));
      VLBA_CUDA(cudaEventElapsedTime(&b, c->ev[2], c->ev[3]));
      VLBA_CUDA(cudaEventElapsedTime(&e, c->ev[3], c->ev[4]));
      VLBA_CUDA(cudaEventElapsedTime(&f, c->ev[4], c->ev[5]));
      pt->lin.push_back(a);
      pt->assemble.push_back(b);
      pt->pcg.push_back(e);
      pt->update.push_back(f);
    }
    if (err) throw Status(VLBA_ERR_TIMEOUT, "a bounded device wait gave up (error bits " + std::to_string(err) + ")");
    bool all_done = true;
    for (const Ctrl& x : ctrl) all_done = all_done && x.done;
    if (all_done) break;
  }
  VLBA_CUDA(cudaEventRecord(c->ev[5], s));
  VLBA_CUDA(cudaEventSynchronize(c->ev[5]));
  float ms = 0.f;
  VLBA_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[5]));
  st.device_ms = ms;
  return st;
}

// Times kIters PCG iterations (tolerance 0) on the system assembled at the
// uploaded initial state for each candidate shape; keeps the fastest.
LaunchShape autotune(Context* c) {
  constexpr uint32_t kIters = 16;
  Dev& d = c->dev;
  Plan& P = c->plan;
  cudaStream_t s = c->stream;
  LaunchShape best;
  best.pcg_grid = c->pcg_grid;
  best.l2_fraction = c->l2_fraction;
  if (!d.num_tile_rows) {
    c->tuned = true;
    return best;
  }
  std::vector<LmParams> tmp = P.params;
  for (LmParams& lp : tmp) {
    lp.pcg_relative_tolerance = 0.0;
    lp.max_pcg_iterations = kIters;
  }
  VLBA_CUDA(cudaMemcpyAsync(const_cast<LmParams*>(d.params), tmp.data(), tmp.size() * sizeof(LmParams),
                            cudaMemcpyHostToDevice, s));
  reset_state(c);
  enqueue_initial(c);
  check_launch(launch_linearize(d, s), "linearize");
  check_launch(launch_point_prep(d, s), "point prep");
  check_launch(launch_offdiag(d, s), "off-diagonal blocks");
  check_launch(launch_cam_diag(d, s), "camera blocks");
  const int gmax = pcg_grid_max(c), gmin = std::max(1, pcg_grid_min(c));
  std::vector<int> grids;
  for (double f : {1.0, 0.75, 0.5, 0.375, 0.25, 0.125}) {
    const int g = std::max(gmin, (int)(f * gmax));
    if (std::find(grids.begin(), grids.end(), g) == grids.end()) grids.push_back(g);
  }
  double best_ms = 1e30;
  for (int g : grids)
    for (double frac : {0.5, 0.0, 0.9}) {
      LaunchShape sh;
      sh.pcg_grid = g;
      sh.l2_fraction = frac;
      apply_shape(c, sh);
      float ms = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        VLBA_CUDA(cudaEventRecord(c->ev[0], s));
        check_launch(launch_pcg_setup(d, s), "pcg setup");
        check_launch(launch_pcg(d, c->pcg_grid, s), "pcg");
        VLBA_CUDA(cudaEventRecord(c->ev[1], s));
        VLBA_CUDA(cudaEventSynchronize(c->ev[1]));
        float t = 0.f;
        VLBA_CUDA(cudaEventElapsedTime(&t, c->ev[0], c->ev[1]));
        if (rep > 0) ms = std::min(ms, t);  // the first run warms the caches
      }
      if (ms < best_ms) {
        best_ms = ms;
        best = sh;
      }
    }
  check_device_error(c);
  VLBA_CUDA(cudaMemcpyAsync(const_cast<LmParams*>(d.params), P.params.data(),
                            P.params.size() * sizeof(LmParams), cudaMemcpyHostToDevice, s));
  VLBA_CUDA(cudaStreamSynchronize(s));
  best.pcg_iteration_us = 1e3 * best_ms / kIters;
  apply_shape(c, best);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[shape_key(P)] = best;
  }
  c->tuned = true;
  return best;
}

void fill_result(Context* c, uint32_t prob, vlba_result* res, vlba_iteration* its, uint32_t cap,
                 const PhaseTimes* pt) {
  Ctrl ctrl;
  VLBA_CUDA(cudaMemcpy(&ctrl, c->dev.ctrl + prob, sizeof ctrl, cudaMemcpyDeviceToHost));
  if (res) {
    res->initial_cost = ctrl.initial_cost;
    res->final_cost = ctrl.current_cost;
    res->converged = ctrl.converged;
    res->num_iterations = ctrl.iteration;
    res->initial_nonprojectable = ctrl.initial_nonproj;
    res->final_nonprojectable = ctrl.current_nonproj;
    res->total_pcg_iterations = ctrl.total_pcg;
  }
  const uint32_t n = std::min(std::min(ctrl.iteration, cap), c->dev.max_records);
  if (its && n) {
    VLBA_CUDA(cudaMemcpy(its, c->dev.records + (size_t)prob * c->dev.max_records,
                         n * sizeof(vlba_iteration), cudaMemcpyDeviceToHost));
    if (pt)
      for (uint32_t i = 0; i < n && i < pt->lin.size(); ++i) {
        its[i].linearize_ms = pt->lin[i];
        its[i].assemble_ms = pt->assemble[i];
        its[i].pcg_ms = pt->pcg[i];
        its[i].update_ms = pt->update[i];
      }
  }
}

void download_problem(Context* c, uint32_t prob, vlba_problem* p) {
  Ctrl ctrl;
  VLBA_CUDA(cudaMemcpy(&ctrl, c->dev.ctrl + prob, sizeof ctrl, cudaMemcpyDeviceToHost));
  const uint32_t b = ctrl.cur;
  const uint32_t pose0 = c->plan.prob_pose_begin[prob], pt0 = c->plan.prob_point_begin[prob];
  const size_t np = c->plan.prob_pose_begin[prob + 1] - pose0;
  const size_t nl = c->plan.prob_point_begin[prob + 1] - pt0;
  if (np != p->num_poses || nl != p->num_landmarks)
    throw Status(VLBA_ERR_INVALID_ARGUMENT, "download: problem sizes differ from the upload");
  VLBA_CUDA(cudaMemcpy(p->pose_q, c->dev.pose_q[b] + 4 * (size_t)pose0, np * 32, cudaMemcpyDeviceToHost));
  VLBA_CUDA(cudaMemcpy(p->pose_t, c->dev.pose_t[b] + 3 * (size_t)pose0, np * 24, cudaMemcpyDeviceToHost));
  VLBA_CUDA(cudaMemcpy(p->landmarks, c->dev.points[b] + 3 * (size_t)pt0, nl * 24, cudaMemcpyDeviceToHost));
}

// Results of every problem of the plan with two bulk copies; `slot[i]` maps
// output i to a problem of the plan (-1: zeroed entry).
void fill_results_bulk(Context* c, const std::vector<int>& slot, vlba_result* res,
                       vlba_iteration* its, uint32_t cap, const RunStats& st,
                       const PhaseTimes* pt) {
  const Dev& d = c->dev;
  const uint32_t np = c->plan.num_problems;
  std::vector<Ctrl> ctrl(np);
  VLBA_CUDA(cudaMemcpy(ctrl.data(), d.ctrl, sizeof(Ctrl) * np, cudaMemcpyDeviceToHost));
  std::vector<vlba_iteration> rec;
  if (its && cap) {
    rec.resize((size_t)np * d.max_records);
    VLBA_CUDA(cudaMemcpy(rec.data(), d.records, rec.size() * sizeof(vlba_iteration),
                         cudaMemcpyDeviceToHost));
  }
  for (size_t i = 0; i < slot.size(); ++i) {
    if (res) std::memset(res + i, 0, sizeof *res);
    if (its && cap) std::memset(its + i * cap, 0, sizeof(vlba_iteration) * cap);
    if (slot[i] < 0) continue;
    const Ctrl& x = ctrl[slot[i]];
    if (res) {
      res[i].initial_cost = x.initial_cost;
      res[i].final_cost = x.current_cost;
      res[i].converged = x.converged;
      res[i].num_iterations = x.iteration;
      res[i].initial_nonprojectable = x.initial_nonproj;
      res[i].final_nonprojectable = x.current_nonproj;
      res[i].total_pcg_iterations = x.total_pcg;
      res[i].device_ms = st.device_ms;
      res[i].kernel_launches = st.launches;
    }
    const uint32_t m = std::min(std::min(x.iteration, cap), d.max_records);
    if (its && m) {
      std::memcpy(its + i * cap, rec.data() + (size_t)slot[i] * d.max_records,
                  m * sizeof(vlba_iteration));
      // Iteration k of every problem ran in the batch's iteration k.
      if (pt)
        for (uint32_t k = 0; k < m && k < pt->lin.size(); ++k) {
          vlba_iteration& r = its[i * cap + k];
          r.linearize_ms = pt->lin[k];
          r.assemble_ms = pt->assemble[k];
          r.pcg_ms = pt->pcg[k];
          r.update_ms = pt->update[k];
        }
    }
  }
}

int pick_tb(const vlba_problem* const*, uint32_t) {
  return 8;  // the PCG streams 8 x 8-block tiles, one warp per tile
}

template <typename F>
int guarded(Context* c, F&& f) {
  try {
    if (c) c->error.clear();
    f();
    return VLBA_OK;
  } catch (const Status& s) {
    if (c) c->error = s.what();
    return s.code;
  } catch (const CudaError& e) {
    if (c) c->error = e.what();
    return e.code == cudaErrorMemoryAllocation ? VLBA_ERR_OUT_OF_MEMORY : VLBA_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    if (c) c->error = "host allocation failed";
    return VLBA_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    if (c) c->error = e.what();
    return VLBA_ERR_INVALID_ARGUMENT;
  }
}

// Validation of n problems, on host threads when they hold many observations.
std::vector<Validation> validate_all(const vlba_problem* const* probs,
                                     const vlba_config* const* cfgs, uint32_t n) {
  std::vector<Validation> v(n);
  uint64_t obs = 0;
  for (uint32_t i = 0; i < n; ++i) obs += probs[i] ? probs[i]->num_observations : 0;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned T = (unsigned)std::min<uint64_t>({hw, n, obs / 500000 + 1});
  std::atomic<uint32_t> next{0};
  auto work = [&] {
    for (uint32_t i; (i = next.fetch_add(1)) < n;) v[i] = validate_problem(probs[i], cfgs[i]);
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < T; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  return v;
}

// Problems of at least this many observations have their Schur terms built
// on the device (below it the host build is quick and avoids the round trip).
constexpr uint64_t kDeviceTermsMinObs = 200000;
// Rows the device builders take (their shared memory holds 12 bytes per row).
constexpr uint32_t kDeviceTermsMaxRows = 16384;
// Dynamic shared memory one block may use on sm_100.
constexpr size_t kMaxDynamicSmem = 227u * 1024u;

// The block structure of the plan's single problem from the device: uploads
// what the row counts read (point-major order, per-slot lists), counts and
// packs each row's columns, and returns them; false (the host builds the
// terms) for a point seen twice by one slot or a system the device builders
// do not take.
bool device_row_blocks(Context* c, const Plan& P, uint32_t nvar, RowBlocks* out) {
  if (nvar < 2 || nvar > kDeviceTermsMaxRows) return false;
  cudaStream_t s = c->stream;
  const size_t ntri = (size_t)nvar * (nvar - 1) / 2;
  auto up16 = [](size_t b) { return (b + 15) & ~size_t(15); };
  const size_t b_coff = up16(4 * P.cam_off.size()), b_cobs = up16(4 * P.cam_obs.size()),
               b_opt = up16(4 * P.obs_point.size()), b_oslot = up16(4 * P.obs_slot.size()),
               b_pvar = up16(P.point_var.size()), b_poff = up16(4 * P.pt_off.size());
  c->rows_in.ensure(b_coff + b_cobs + b_opt + b_oslot + b_pvar + b_poff);
  char* in = c->rows_in.as<char>();
  const size_t b_tri = up16(8 * ntri), b_nblk = up16(4 * (size_t)nvar),
               b_rblk = up16(4 * ((size_t)nvar + 1)), b_list = up16(4 * ntri);
  c->rows_out.ensure(16 + b_tri + b_nblk + b_rblk + 2 * b_list);
  char* o = c->rows_out.as<char>();
  RowsDev r{};
  r.nvar = nvar;
  size_t at = 0;
  int slot = 0;
  Stager st(c);  // through the pinned staging buffers
  auto put = [&](const void* src, size_t bytes, size_t room) {
    char* dst = in + at;
    c->rows_in_at[slot++] = at;
    st.add(dst, src, bytes);
    at += room;
    return dst;
  };
  r.cam_off = reinterpret_cast<const uint32_t*>(put(P.cam_off.data(), 4 * P.cam_off.size(), b_coff));
  r.cam_obs = reinterpret_cast<const uint32_t*>(put(P.cam_obs.data(), 4 * P.cam_obs.size(), b_cobs));
  r.obs_point = reinterpret_cast<const uint32_t*>(put(P.obs_point.data(), 4 * P.obs_point.size(), b_opt));
  r.obs_slot = reinterpret_cast<const uint32_t*>(put(P.obs_slot.data(), 4 * P.obs_slot.size(), b_oslot));
  r.point_var = reinterpret_cast<const uint8_t*>(put(P.point_var.data(), P.point_var.size(), b_pvar));
  r.pt_off = reinterpret_cast<const uint32_t*>(put(P.pt_off.data(), 4 * P.pt_off.size(), b_poff));
  st.flush(s);
  r.flags = reinterpret_cast<uint32_t*>(o);
  r.tri = reinterpret_cast<uint2*>(o + 16);
  r.row_nblk = reinterpret_cast<uint32_t*>(o + 16 + b_tri);
  r.row_blk = reinterpret_cast<uint32_t*>(o + 16 + b_tri + b_nblk);
  r.col = reinterpret_cast<uint32_t*>(o + 16 + b_tri + b_nblk + b_rblk);
  r.count = reinterpret_cast<uint32_t*>(o + 16 + b_tri + b_nblk + b_rblk + b_list);
  VLBA_CUDA(cudaMemsetAsync(r.flags, 0, 4, s));
  check_launch(launch_rows_count(r, s), "Schur term counts");
  uint32_t flags = 0;
  out->row_off.resize((size_t)nvar + 1);
  VLBA_CUDA(cudaMemcpyAsync(&flags, r.flags, 4, cudaMemcpyDeviceToHost, s));
  VLBA_CUDA(cudaMemcpyAsync(out->row_off.data(), r.row_blk, 4 * ((size_t)nvar + 1),
                            cudaMemcpyDeviceToHost, s));
  VLBA_CUDA(cudaStreamSynchronize(s));
  if (flags & 1u) return false;
  const size_t nb = out->row_off[nvar];
  if (nb > ntri) throw std::runtime_error("device Schur term counts out of range");
  // The placement keeps per-row state for the longest row's blocks in
  // shared memory; a system whose rows do not fit is laid out on the host.
  uint32_t max_row_blocks = 0;
  for (uint32_t i = 0; i < nvar; ++i)
    max_row_blocks = std::max(max_row_blocks, out->row_off[i + 1] - out->row_off[i]);
  if (rows_place_smem(nvar, max_row_blocks, 1) > kMaxDynamicSmem) return false;
  out->col.resize(nb);
  out->count.resize(nb);
  VLBA_CUDA(cudaMemcpyAsync(out->col.data(), r.col, 4 * nb, cudaMemcpyDeviceToHost, s));
  VLBA_CUDA(cudaMemcpyAsync(out->count.data(), r.count, 4 * nb, cudaMemcpyDeviceToHost, s));
  VLBA_CUDA(cudaStreamSynchronize(s));
  return true;
}

void do_upload(Context* c, const vlba_problem* const* probs, const vlba_config* const* cfgs,
               uint32_t n, uint32_t max_records, double* upload_ms) {
  const auto t0 = std::chrono::steady_clock::now();
  // VLBA_TRACE_UPLOAD: host time of the upload's phases, to stderr (the
  // analogue of the reference's VISLOC_BA_TRACE_PHASE_TIMING, lm.rs:345).
  const bool trace = std::getenv("VLBA_TRACE_UPLOAD") != nullptr;
  auto ms_since = [](std::chrono::steady_clock::time_point a) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
  };
  c->batch_slot.clear();
  const std::vector<Validation> vs = validate_all(probs, cfgs, n);
  for (uint32_t i = 0; i < n; ++i)
    if (vs[i].status != VLBA_OK)
      throw Status(vs[i].status, "problem " + std::to_string(i) + " failed validation",
                   vs[i].error_index);
  const double t_validate = ms_since(t0);
  set_device(c);
  c->reduced_generation = ~0ull;  // the host plan no longer matches the reduced layout
  // One large problem: its Schur terms (the plan's largest part) are found
  // and written on the device; the host lays out the rest.
  double t_rows = 0.0;
  const RowBlocksFn device_rows = [c, &t_rows, &ms_since](const Plan& P, uint32_t nvar,
                                                          RowBlocks* out) {
    const auto r0 = std::chrono::steady_clock::now();
    const bool ok = device_row_blocks(c, P, nvar, out);
    t_rows = ms_since(r0);
    return ok;
  };
  const bool large = n == 1 && probs[0]->num_observations >= kDeviceTermsMinObs;
  const auto tb0 = std::chrono::steady_clock::now();
  {
    // A large problem's plan arrays are page-locked when first allocated
    // (a context's plan keeps them for the next upload), so they are copied
    // to the device without staging.
    std::unique_ptr<PinScope> pin(large ? new PinScope() : nullptr);
    build_plan(probs, cfgs, n, (uint32_t)pick_tb(probs, n), &c->plan, 0,
               large ? &device_rows : nullptr);
  }
  const double t_build = ms_since(tb0);
  // The plan check runs on its own thread while the arrays are copied, and
  // ends before the first kernel reads them.
  const auto tu0 = std::chrono::steady_clock::now();
  std::string bad;
  double t_check = 0.0, t_wait = 0.0;
  std::thread checker([&] {
    const auto tc0 = std::chrono::steady_clock::now();
    bad = check_plan(c->plan);
    t_check = ms_since(tc0);
  });
  struct Join {
    std::thread& t;
    ~Join() {
      if (t.joinable()) t.join();
    }
  } join{checker};
  const std::function<void()> checked = [&] {
    if (checker.joinable()) {
      const auto w0 = std::chrono::steady_clock::now();
      checker.join();
      t_wait = ms_since(w0);
    }
    if (!bad.empty()) throw Status(VLBA_ERR_INVALID_ARGUMENT, bad);
  };
  upload_plan(c, max_records, checked);
  checked();
  if (trace)
    std::fprintf(stderr,
                 "vlba upload: validate %.2f ms, plan %.2f ms (device row counts %.2f ms), "
                 "copy, check and device terms %.2f ms (arrays issued %.2f ms, of it staged copies "
                 "%.2f ms; check %.2f ms beside them, %.2f ms waited; device terms %.2f ms)\n",
                 t_validate, t_build, t_rows, ms_since(tu0), c->up_copy_ms, c->up_flush_ms, t_check,
                 t_wait, c->up_terms_ms);
  c->num_poses.clear();
  c->num_points.clear();
  for (uint32_t i = 0; i < n; ++i) {
    c->num_poses.push_back(probs[i]->num_poses);
    c->num_points.push_back(probs[i]->num_landmarks);
  }
  const auto t1 = std::chrono::steady_clock::now();
  if (upload_ms) *upload_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  // Host -> device bytes of this upload: the plan's arrays.
  const Plan& P = c->plan;
  // (With terms built on the device, the arrays its row counts read went
  // over once, before the plan's other arrays, and count among them.)
  c->last_upload_bytes = P.upload_bytes();
}

// Write the current state of every uploaded problem back into `problems`
// (slot[i]: problem of the plan for output i, -1 skips it).
void download_all(Context* c, const std::vector<int>& slot, vlba_problem* const* problems) {
  const Dev& d = c->dev;
  const Plan& P = c->plan;
  check_launch(launch_state_to_front(d, c->stream), "state gather");
  for (size_t i = 0; i < slot.size(); ++i) {
    const int k = slot[i];
    if (k < 0 || !problems[i]) continue;
    if (P.prob_pose_begin[k + 1] - P.prob_pose_begin[k] != problems[i]->num_poses ||
        P.prob_point_begin[k + 1] - P.prob_point_begin[k] != problems[i]->num_landmarks)
      throw Status(VLBA_ERR_INVALID_ARGUMENT, "download: problem sizes differ from the upload");
  }
  // The state lands in the pinned staging buffer when it fits (else in
  // pageable vectors); then each problem's part is copied out.
  const size_t nq = P.pose_q.size(), nt = P.pose_t.size(), nx = P.points.size();
  const size_t bytes = 8 * (nq + nt + nx);
  std::vector<double> host;
  double* q = nullptr;
  if (c->stage[0] && bytes <= c->stage_cap) {
    VLBA_CUDA(cudaEventSynchronize(c->stage_ev[0]));
    q = reinterpret_cast<double*>(c->stage[0]);
  } else {
    host.resize(nq + nt + nx);
    q = host.data();
  }
  double* t = q + nq;
  double* x = t + nt;
  VLBA_CUDA(cudaMemcpyAsync(q, d.pose_q[0], nq * 8, cudaMemcpyDeviceToHost, c->stream));
  VLBA_CUDA(cudaMemcpyAsync(t, d.pose_t[0], nt * 8, cudaMemcpyDeviceToHost, c->stream));
  VLBA_CUDA(cudaMemcpyAsync(x, d.points[0], nx * 8, cudaMemcpyDeviceToHost, c->stream));
  VLBA_CUDA(cudaStreamSynchronize(c->stream));
  auto out = [&](size_t i) {
    const int k = slot[i];
    if (k < 0 || !problems[i]) return;
    vlba_problem* p = problems[i];
    const uint32_t pose0 = P.prob_pose_begin[k], pt0 = P.prob_point_begin[k];
    const size_t np = P.prob_pose_begin[k + 1] - pose0, nl = P.prob_point_begin[k + 1] - pt0;
    std::memcpy(p->pose_q, q + 4 * (size_t)pose0, np * 32);
    std::memcpy(p->pose_t, t + 3 * (size_t)pose0, np * 24);
    std::memcpy(p->landmarks, x + 3 * (size_t)pt0, nl * 24);
  };
  if (slot.size() == 1) {
    const int k = slot[0];
    if (k >= 0 && problems[0]) {
      vlba_problem* p = problems[0];
      const uint32_t pose0 = P.prob_pose_begin[k], pt0 = P.prob_point_begin[k];
      par_memcpy(p->pose_q, q + 4 * (size_t)pose0, (size_t)p->num_poses * 32);
      par_memcpy(p->pose_t, t + 3 * (size_t)pose0, (size_t)p->num_poses * 24);
      par_memcpy(p->landmarks, x + 3 * (size_t)pt0, (size_t)p->num_landmarks * 24);
    }
    return;
  }
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned T = (unsigned)std::min<size_t>({std::min(hw, 16u), slot.size(), bytes / (2u << 20) + 1});
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (size_t i; (i = next.fetch_add(1)) < slot.size();) out(i);
  };
  std::vector<std::thread> pool;
  for (unsigned w = 1; w < T; ++w) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

}  // namespace

Context* make_context(int device) {
  std::unique_ptr<Context> c(new Context());
  c->device = device;
  int count = 0;
  VLBA_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) throw std::runtime_error("no such device");
  VLBA_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  VLBA_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) throw std::runtime_error("requires an sm_100 (Blackwell) device");
  c->sm_count = prop.multiProcessorCount;
  c->l2_bytes = (size_t)prop.l2CacheSize;
  c->pcg_grid_hint = 4 * prop.multiProcessorCount;
  if (const char* f = std::getenv("VLBA_L2_RESIDENT_FRACTION")) c->l2_fraction = std::atof(f);
  VLBA_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  VLBA_CUDA(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
  VLBA_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
  VLBA_CUDA(cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming));
  for (auto& e : c->ev) VLBA_CUDA(cudaEventCreate(&e));
  return c.release();
}

void free_context(Context* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  drop_graph(c);
  c->arena.release();
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (int i = 0; i < 2; ++i) {
    if (c->stage_ev[i]) cudaEventDestroy(c->stage_ev[i]);
    if (c->stage[i]) cudaFreeHost(c->stage[i]);
  }
  if (c->gnc_sq) cudaFree(c->gnc_sq);
  c->elim.reset();
  if (c->fork) cudaEventDestroy(c->fork);
  if (c->join) cudaEventDestroy(c->join);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // namespace vlba

using vlba::Context;

extern "C" {

uint32_t visloc_ba_cuda_abi_version(void) { return VLBA_ABI_VERSION; }

void visloc_ba_cuda_default_config(vlba_config* out) {
  if (!out) return;
  std::memset(out, 0, sizeof *out);
  out->max_iterations = 20;
  out->has_initial_lambda = 1;
  out->initial_lambda = 1e-4;
  out->lambda_increase_factor = 10.0;
  out->lambda_decrease_factor = 0.1;
  out->max_lambda = 1e12;
  out->min_lambda = 1e-9;
  out->step_tolerance = 1e-7;
  out->cost_tolerance = 1e-9;
  out->has_relative_cost_tolerance = 0;
  out->relative_cost_tolerance = 0.0;
  out->robust_kernel = VLBA_KERNEL_NONE;
  out->robust_parameter = 0.0;
  out->max_pcg_iterations = 100;
  out->pcg_relative_tolerance = 1e-4;
  out->flags = 0;
}

void* visloc_ba_cuda_create(int device) {
  try {
    return vlba::make_context(device);
  } catch (...) {
    return nullptr;
  }
}

void visloc_ba_cuda_destroy(void* ctx) { vlba::free_context(static_cast<Context*>(ctx)); }

const char* visloc_ba_cuda_last_error(void* ctx) {
  auto* c = static_cast<Context*>(ctx);
  return c ? c->error.c_str() : "null context";
}

int visloc_ba_cuda_check(const vlba_problem* problem, const vlba_config* config,
                         uint64_t* error_index) {
  const vlba::Validation v = vlba::validate_problem(problem, config);
  if (error_index) *error_index = v.error_index;
  return v.status;
}

int visloc_ba_cuda_upload(void* ctx, const vlba_problem* problem, const vlba_config* config) {
  auto* c = static_cast<Context*>(ctx);
  if (!c) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    const vlba_problem* probs[1] = {problem};
    const vlba_config* cfgs[1] = {config};
    vlba::do_upload(c, probs, cfgs, 1, config ? config->max_iterations : 0, nullptr);
    c->flags = config ? config->flags : 0;
  });
}

int visloc_ba_cuda_solve_uploaded(void* ctx, const vlba_config* config, vlba_result* result,
                                  vlba_iteration* iterations, uint32_t iterations_capacity) {
  auto* c = static_cast<Context*>(ctx);
  if (!c) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    if (!c->uploaded) throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "nothing uploaded");
    vlba::set_device(c);
    if (config) {
      vlba::LmParams lp = vlba::make_params(config);
      if (lp.max_iterations > c->dev.max_records)
        throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "max_iterations exceeds the uploaded capacity");
      VLBA_CUDA(cudaMemcpyAsync(const_cast<vlba::LmParams*>(c->dev.params), &lp, sizeof lp,
                                cudaMemcpyHostToDevice, c->stream));
      c->plan.params[0] = lp;
    }
    vlba::reset_state(c);
    const bool profile = (config ? config->flags : c->flags) & VLBA_FLAG_PROFILE;
    vlba::PhaseTimes pt;
    const vlba::RunStats st = vlba::run_lm(c, profile, &pt);
    if (result) std::memset(result, 0, sizeof *result);
    vlba::fill_result(c, 0, result, iterations, iterations_capacity, profile ? &pt : nullptr);
    if (result) {
      result->device_ms = st.device_ms;
      result->kernel_launches = st.launches;
    }
  });
}

int visloc_ba_cuda_download(void* ctx, vlba_problem* problem) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !problem) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    if (!c->uploaded) throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "nothing uploaded");
    vlba::set_device(c);
    vlba::download_problem(c, 0, problem);
  });
}

int visloc_ba_cuda_optimize(void* ctx, vlba_problem* problem, const vlba_config* config,
                            vlba_result* result, vlba_iteration* iterations,
                            uint32_t iterations_capacity) {
  auto* c = static_cast<Context*>(ctx);
  if (!c) return VLBA_ERR_INVALID_ARGUMENT;
  if (result) std::memset(result, 0, sizeof *result);
  double upload_ms = 0.0;
  int st = vlba::guarded(c, [&] {
    const vlba_problem* probs[1] = {problem};
    const vlba_config* cfgs[1] = {config};
    vlba::do_upload(c, probs, cfgs, 1, config ? config->max_iterations : 0, &upload_ms);
    c->flags = config ? config->flags : 0;
  });
  if (st != VLBA_OK) {
    if (result && (st == VLBA_ERR_MISSING_POSE || st == VLBA_ERR_MISSING_LANDMARK ||
                   st == VLBA_ERR_INVALID_OBSERVATION_WEIGHT)) {
      uint64_t idx = 0;
      visloc_ba_cuda_check(problem, config, &idx);
      result->error_index = idx;
    }
    return st;
  }
  st = visloc_ba_cuda_solve_uploaded(ctx, nullptr, result, iterations, iterations_capacity);
  if (st != VLBA_OK) return st;
  if (result) {
    result->upload_ms = upload_ms;
    result->upload_bytes = c->last_upload_bytes;
  }
  return visloc_ba_cuda_download(ctx, problem);
}

int visloc_ba_cuda_batch_upload(void* ctx, uint32_t n, const vlba_problem* const* problems,
                                const vlba_config* const* configs, int* statuses) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || (n && (!problems || !configs))) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    std::vector<const vlba_problem*> ps;
    std::vector<const vlba_config*> cs;
    std::vector<int> slot(n, -1);
    uint32_t max_rec = 0, flags = 0;
    int first_bad = VLBA_ERR_INVALID_ARGUMENT;
    const std::vector<vlba::Validation> vs = vlba::validate_all(problems, configs, n);
    for (uint32_t i = 0; i < n; ++i) {
      const vlba::Validation& v = vs[i];
      if (statuses) statuses[i] = v.status;
      if (v.status != VLBA_OK) {
        if (ps.empty() && first_bad == VLBA_ERR_INVALID_ARGUMENT) first_bad = v.status;
        continue;
      }
      slot[i] = (int)ps.size();
      ps.push_back(problems[i]);
      cs.push_back(configs[i]);
      max_rec = std::max(max_rec, configs[i]->max_iterations);
      flags |= configs[i]->flags;
    }
    if (ps.empty()) throw vlba::Status(first_bad, "no problem of the batch passed validation");
    vlba::do_upload(c, ps.data(), cs.data(), (uint32_t)ps.size(), max_rec, nullptr);
    c->flags = flags;
    c->batch_slot = std::move(slot);
  });
}

int visloc_ba_cuda_batch_solve_uploaded(void* ctx, vlba_result* results,
                                        vlba_iteration* iterations,
                                        uint32_t iterations_capacity) {
  auto* c = static_cast<Context*>(ctx);
  if (!c) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    if (!c->uploaded || c->batch_slot.empty())
      throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "no batch uploaded");
    vlba::set_device(c);
    vlba::reset_state(c);
    const bool profile = c->flags & VLBA_FLAG_PROFILE;
    vlba::PhaseTimes pt;
    const vlba::RunStats st = vlba::run_lm(c, profile, &pt);
    vlba::fill_results_bulk(c, c->batch_slot, results, iterations, iterations_capacity, st,
                            profile ? &pt : nullptr);
  });
}

int visloc_ba_cuda_batch_download(void* ctx, uint32_t n, vlba_problem* const* problems) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || (n && !problems)) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    if (!c->uploaded || c->batch_slot.size() != n)
      throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "download: not the uploaded batch");
    vlba::set_device(c);
    vlba::download_all(c, c->batch_slot, problems);
  });
}

int visloc_ba_cuda_batch_optimize(void* ctx, uint32_t n, vlba_problem* const* problems,
                                  const vlba_config* const* configs, int* statuses,
                                  vlba_result* results, vlba_iteration* iterations,
                                  uint32_t iterations_capacity) {
  int st = visloc_ba_cuda_batch_upload(ctx, n, problems, configs, statuses);
  if (st != VLBA_OK) return st;
  st = visloc_ba_cuda_batch_solve_uploaded(ctx, results, iterations, iterations_capacity);
  if (st != VLBA_OK) return st;
  return visloc_ba_cuda_batch_download(ctx, n, problems);
}

int visloc_ba_cuda_plan(const vlba_problem* problem, const vlba_config* config,
                        double pcg_iterations, vlba_plan_info* info) {
  return vlba::guarded(nullptr, [&] {
    const vlba::Validation v = vlba::validate_problem(problem, config);
    if (v.status != VLBA_OK) throw vlba::Status(v.status, "validation", v.error_index);
    const vlba_problem* probs[1] = {problem};
    const vlba_config* cfgs[1] = {config};
    vlba::Plan plan;
    vlba::build_plan(probs, cfgs, 1, (uint32_t)vlba::pick_tb(probs, 1), &plan);
    const std::string bad = vlba::check_plan(plan);
    if (!bad.empty()) throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, bad);
    if (info) {
      std::memset(info, 0, sizeof *info);
      info->variable_cameras = plan.real_var_cams;
      info->variable_landmarks = plan.var_points;
      info->variable_observations = plan.var_obs;
      info->camera_pairs = plan.camera_pairs;
      info->schur_terms = plan.num_pairs;
      info->tile_size = plan.tb;
      info->tile_rows = plan.num_tile_rows;
      info->tiles = (uint32_t)plan.tile_ij.size();
      info->assembly_lanes = plan.group;
      info->device_bytes = plan.device_bytes();
      info->upload_bytes = plan.upload_bytes();
      double b_pcg = 0.0;
      info->bytes_per_iteration = vlba::algorithmic_bytes(plan, pcg_iterations, &b_pcg);
      info->bytes_per_pcg_iteration = b_pcg;
    }
  });
}

void visloc_ba_cuda_default_gnc_config(vlba_gnc_config* gnc) {
  if (!gnc) return;
  std::memset(gnc, 0, sizeof *gnc);  // GncConfig::default() (gnc.rs:100-110)
  gnc->kernel = VLBA_GNC_GEMAN_MCCLURE;
  gnc->c = 1.0;
  gnc->anneal_factor = 1.4;
  gnc->max_outer = 100;
  gnc->inner_iterations = 5;
}

int visloc_ba_cuda_optimize_gnc(void* ctx, vlba_problem* problem, const vlba_config* config,
                                const vlba_gnc_config* gnc, vlba_gnc_result* result,
                                double* observation_weights) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !problem || !config || !gnc) return VLBA_ERR_INVALID_ARGUMENT;
  if (result) std::memset(result, 0, sizeof *result);
  return vlba::guarded(c, [&] {
    using vlba::Status;
    if (problem->obs_weight)
      throw Status(VLBA_ERR_INVALID_ARGUMENT, "GNC sets the observation weights: obs_weight must be NULL");
    if (gnc->kernel > VLBA_GNC_TRUNCATED_LEAST_SQUARES)
      throw Status(VLBA_ERR_INVALID_ARGUMENT, "unknown GNC kernel");
    const uint64_t n = problem->num_observations;
    // The inner solve: the config's LM with no M-estimator (the GNC weights
    // are the only robustification) and inner_iterations iterations
    // (lm.rs:64-68).
    vlba_config inner = *config;
    inner.robust_kernel = VLBA_KERNEL_NONE;
    inner.robust_parameter = 0.0;
    inner.max_iterations = std::max(1u, gnc->inner_iterations);
    inner.flags &= ~VLBA_FLAG_PROFILE;
    std::vector<double> weights(n, 1.0);
    vlba_problem up = *problem;
    up.obs_weight = weights.data();  // a weight array on the device, rewritten per level
    const vlba_problem* probs[1] = {&up};
    const vlba_config* cfgs[1] = {&inner};
    vlba::do_upload(c, probs, cfgs, 1, inner.max_iterations, nullptr);
    c->flags = inner.flags;
    vlba::Dev& d = c->dev;
    const vlba::Plan& P = c->plan;
    cudaStream_t s = c->stream;
    if (c->gnc_cap < n) {
      if (c->gnc_sq) cudaFree(c->gnc_sq);
      c->gnc_sq = nullptr;
      c->gnc_cap = 0;
      VLBA_CUDA(cudaMalloc(&c->gnc_sq, std::max<uint64_t>(n, 1) * sizeof(double)));
      c->gnc_cap = n;
    }
    // Squared residuals in plan order at the current state (also left in
    // state buffer 0).
    vlba::reset_state(c);  // the uploaded state into buffer 0, control words cleared
    std::vector<double> sq(n), w(n, 1.0);
    auto residuals = [&] {
      vlba::check_launch(vlba::launch_state_to_front(d, s), "state gather");
      vlba::check_launch(vlba::launch_sq_residuals(d, c->gnc_sq, s), "residuals");
      VLBA_CUDA(cudaMemcpyAsync(sq.data(), c->gnc_sq, n * sizeof(double), cudaMemcpyDeviceToHost, s));
      VLBA_CUDA(cudaStreamSynchronize(s));
    };
    residuals();
    double initial_cost = 0.0, s_max = 0.0;
    for (double v : sq)
      if (std::isfinite(v)) {
        initial_cost += v;
        s_max = std::max(s_max, v);
      }
    // Inlier scale: the configured c, or the MAD estimate floored at it
    // (lm.rs:46-56).
    double scale = gnc->c;
    if (gnc->has_auto_scale) {
      double est = 0.0;
      if (vlba::estimate_scale_mad(sq, gnc->auto_scale, &est)) scale = std::max(est, gnc->c);
    }
    double inlier_scale = scale;
    vlba::GncState state = vlba::GncState::start(gnc->kernel, scale, gnc->anneal_factor, s_max);
    uint32_t outer = 0;
    bool converged = false;
    uint64_t lm_iterations = 0;
    double device_ms = 0.0;
    for (uint32_t level = 0; level < std::max(1u, gnc->max_outer); ++level) {
      ++outer;
      const bool terminal = state.terminal();
      residuals();
      if (gnc->auto_scale_readapt && gnc->has_auto_scale) {
        double est = 0.0;
        if (vlba::estimate_scale_mad(sq, gnc->auto_scale, &est)) {
          const double cc = std::max(est, gnc->c);
          state.set_inlier_scale(cc);
          inlier_scale = cc;
        }
      }
      for (uint64_t k = 0; k < n; ++k) w[k] = std::isfinite(sq[k]) ? state.weight(sq[k]) : 1.0;
      VLBA_CUDA(cudaMemcpyAsync(const_cast<double*>(d.obs_w), w.data(), n * sizeof(double),
                                cudaMemcpyHostToDevice, s));
      // The level starts from the previous level's state.
      VLBA_CUDA(cudaMemcpyAsync(const_cast<double*>(d.init_pose_q), d.pose_q[0], P.pose_q.size() * 8,
                                cudaMemcpyDeviceToDevice, s));
      VLBA_CUDA(cudaMemcpyAsync(const_cast<double*>(d.init_pose_t), d.pose_t[0], P.pose_t.size() * 8,
                                cudaMemcpyDeviceToDevice, s));
      VLBA_CUDA(cudaMemcpyAsync(const_cast<double*>(d.init_points), d.points[0], P.points.size() * 8,
                                cudaMemcpyDeviceToDevice, s));
      vlba::reset_state(c);
      const vlba::RunStats rs = vlba::run_lm(c, false, nullptr);
      device_ms += rs.device_ms;
      vlba::Ctrl ctrl;
      VLBA_CUDA(cudaMemcpy(&ctrl, d.ctrl, sizeof ctrl, cudaMemcpyDeviceToHost));
      lm_iterations += ctrl.iteration;
      if (terminal) {
        converged = true;
        break;
      }
      state.anneal();
    }
    // Final weights at the recovered estimate, NaN where an observation
    // cannot be evaluated; the weighted and the inlier-only (w >= 0.5) costs
    // (lm.rs:99-130).
    residuals();
    double final_cost = 0.0, inlier_cost = 0.0;
    for (uint64_t k = 0; k < n; ++k) {
      if (!std::isfinite(sq[k])) {
        w[k] = std::nan("");
        continue;
      }
      w[k] = state.weight(sq[k]);
      final_cost += w[k] * sq[k];
      if (w[k] >= 0.5) inlier_cost += sq[k];
    }
    vlba::download_problem(c, 0, problem);
    if (observation_weights)
      for (uint64_t k = 0; k < n; ++k) observation_weights[P.obs_src[k]] = w[k];
    if (result) {
      result->initial_cost = initial_cost;
      result->final_cost = final_cost;
      result->inlier_cost = inlier_cost;
      result->inlier_scale = inlier_scale;
      result->observation_count = n;
      result->outer_iterations = outer;
      result->converged = converged ? 1u : 0u;
      result->lm_iterations = lm_iterations;
      result->device_ms = device_ms;
    }
  });
}

namespace vlba {
namespace {
// Upload one problem and linearise it at its state with damping `lambda`
// (init + linearize + point prep + assembly).
void prepare_system(Context* c, const vlba_problem* problem, const vlba_config* config,
                    double lambda) {
  vlba_config cfg = *config;
  cfg.max_iterations = 1;
  const vlba_problem* probs[1] = {problem};
  const vlba_config* cfgs[1] = {&cfg};
  do_upload(c, probs, cfgs, 1, 1, nullptr);
  reset_state(c);
  Dev& d = c->dev;
  cudaStream_t s = c->stream;
  check_launch(launch_pose_table(d, s), "pose table");
  check_launch(launch_cost(d, false, s), "cost");
  check_launch(launch_decide(d, true, s), "init");
  VLBA_CUDA(cudaMemcpyAsync(&d.ctrl[0].lambda, &lambda, sizeof lambda, cudaMemcpyHostToDevice, s));
  check_launch(launch_linearize(d, s), "linearize");
  check_launch(launch_point_prep(d, s), "point prep");
  check_launch(launch_offdiag(d, s), "off-diagonal blocks");
  check_launch(launch_cam_diag(d, s), "camera blocks");
}
}  // namespace
}  // namespace vlba

int visloc_ba_cuda_linear_step(void* ctx, const vlba_problem* problem, const vlba_config* config,
                               double lambda, double* dp, double* dl, uint32_t* pcg_iterations,
                               double* pcg_relative_residual) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !problem || !config) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    vlba::prepare_system(c, problem, config, lambda);
    vlba::Dev& d = c->dev;
    cudaStream_t s = c->stream;
    vlba::check_launch(vlba::launch_pcg_setup(d, s), "pcg setup");
    vlba::check_launch(vlba::launch_pcg(d, c->pcg_grid, s), "pcg");
    if (d.trace) vlba::dump_trace(c);
    vlba::check_launch(vlba::launch_pose_update(d, s), "pose update");
    vlba::check_launch(vlba::launch_cost(d, true, s), "back-substitution");
    const vlba::Plan& P = c->plan;
    std::vector<float> x((size_t)P.num_var_cams * 6);
    if (!x.empty())
      VLBA_CUDA(cudaMemcpyAsync(x.data(), d.x, x.size() * 4, cudaMemcpyDeviceToHost, s));
    std::vector<double> pts0(P.points.size()), pts1(P.points.size());
    VLBA_CUDA(cudaMemcpyAsync(pts0.data(), d.points[0], pts0.size() * 8, cudaMemcpyDeviceToHost, s));
    VLBA_CUDA(cudaMemcpyAsync(pts1.data(), d.points[1], pts1.size() * 8, cudaMemcpyDeviceToHost, s));
    vlba::PcgState pg;
    VLBA_CUDA(cudaMemcpyAsync(&pg, d.pcg, sizeof pg, cudaMemcpyDeviceToHost, s));
    unsigned int err = 0;
    VLBA_CUDA(cudaMemcpyAsync(&err, d.error, 4, cudaMemcpyDeviceToHost, s));
    VLBA_CUDA(cudaStreamSynchronize(s));
    if (err) throw vlba::Status(VLBA_ERR_TIMEOUT, "a bounded device wait gave up");
    if (dp) {
      size_t n = 0;
      for (size_t i = 0; i < P.pose_slot.size(); ++i)
        if (P.pose_slot[i] != vlba::kNone) {
          for (int a = 0; a < 6; ++a) dp[6 * n + a] = x[6 * (size_t)P.pose_slot[i] + a];
          ++n;
        }
    }
    if (dl) {
      size_t n = 0;
      for (size_t j = 0; j < P.point_var.size(); ++j)
        if (P.point_var[j]) {
          for (int a = 0; a < 3; ++a) dl[3 * n + a] = pts1[3 * j + a] - pts0[3 * j + a];
          ++n;
        }
    }
    if (pcg_iterations) *pcg_iterations = pg.iters;
    if (pcg_relative_residual) *pcg_relative_residual = pg.bnorm > 0 ? pg.rnorm / pg.bnorm : 0.0;
  });
}

int visloc_ba_cuda_reduced_system(void* ctx, const vlba_problem* problem,
                                  const vlba_config* config, double lambda, double* s_dense,
                                  double* rhs) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !problem || !config) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    vlba::prepare_system(c, problem, config, lambda);
    vlba::Dev& d = c->dev;
    const vlba::Plan& P = c->plan;
    const size_t tile_floats = (size_t)P.tb * P.tb * vlba::kBlock;
    std::vector<float> tiles(P.tile_ij.size() * tile_floats), r((size_t)P.num_var_cams * 6);
    VLBA_CUDA(cudaMemcpyAsync(tiles.data(), d.tiles, tiles.size() * 4, cudaMemcpyDeviceToHost, c->stream));
    if (!r.empty())
      VLBA_CUDA(cudaMemcpyAsync(r.data(), d.rhs, r.size() * 4, cudaMemcpyDeviceToHost, c->stream));
    VLBA_CUDA(cudaStreamSynchronize(c->stream));
    // Variable slot -> dense index (slots are the variable poses in order).
    const size_t nc = P.real_var_cams, dim = 6 * nc;
    if (s_dense) {
      std::fill(s_dense, s_dense + dim * dim, 0.0);
      for (size_t t = 0; t < P.tile_ij.size(); ++t) {
        const uint32_t I = P.tile_ij[t] >> 16, J = P.tile_ij[t] & 0xFFFFu;
        for (uint32_t li = 0; li < P.tb; ++li)
          for (uint32_t lj = 0; lj < P.tb; ++lj) {
            const size_t i = (size_t)I * P.tb + li, j = (size_t)J * P.tb + lj;
            if (i >= nc || j >= nc) continue;
            const float* blk = &tiles[t * tile_floats + (li * P.tb + lj) * vlba::kBlock];
            for (int a = 0; a < 6; ++a)
              for (int b = 0; b < 6; ++b) {
                s_dense[(6 * i + a) * dim + 6 * j + b] = blk[a * 6 + b];
                if (I != J) s_dense[(6 * j + b) * dim + 6 * i + a] = blk[a * 6 + b];
              }
          }
      }
    }
    if (rhs)
      for (size_t e = 0; e < dim; ++e) rhs[e] = r[e];
  });
}

int visloc_ba_cuda_cost(void* ctx, const vlba_problem* problem, const vlba_config* config,
                        double* cost, uint64_t* nonprojectable) {
  auto* c = static_cast<Context*>(ctx);
  if (!c) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    vlba_config cfg = *config;
    cfg.max_iterations = 0;
    // The cost does not depend on what a solve would refine.
    cfg.refine_intrinsics = cfg.refine_distortion = 0;
    cfg.refine_tangential_distortion = cfg.shared_focal = 0;
    const vlba_problem* probs[1] = {problem};
    const vlba_config* cfgs[1] = {&cfg};
    const vlba::Validation v = vlba::validate_problem(problem, &cfg);
    if (v.status != VLBA_OK && v.status != VLBA_ERR_ALL_POSES_FIXED)
      throw vlba::Status(v.status, "validation", v.error_index);
    vlba::set_device(c);
    c->reduced_generation = ~0ull;
    vlba::build_plan(probs, cfgs, 1, 8, &c->plan);
    const std::string bad = vlba::check_plan(c->plan);
    if (!bad.empty()) throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, bad);
    vlba::upload_plan(c, 1);
    vlba::reset_state(c);
    vlba::Dev& d = c->dev;
    vlba::check_launch(vlba::launch_pose_table(d, c->stream), "pose table");
    vlba::check_launch(vlba::launch_cost(d, false, c->stream), "cost");
    vlba::check_launch(vlba::launch_decide(d, true, c->stream), "cost reduce");
    vlba::Ctrl ctrl;
    VLBA_CUDA(cudaMemcpyAsync(&ctrl, d.ctrl, sizeof ctrl, cudaMemcpyDeviceToHost, c->stream));
    VLBA_CUDA(cudaStreamSynchronize(c->stream));
    if (cost) *cost = ctrl.initial_cost;
    if (nonprojectable) *nonprojectable = ctrl.initial_nonproj;
  });
}

}  // extern "C"

// ------------------------------------------------------------------ server
// A request loop on one GPU: tickets are planned on host threads as they
// arrive, then admitted into batches by worker slots as slots and device
// memory free up.  Each slot owns a context (its own stream and a slab of
// device memory sized at start), so the batches of different slots overlap
// on the device; the persistent PCG kernels of the slots take turns (PcgGate).
// A large request (many observations) runs as a batch of its own, so small
// requests are not held behind it.  Every problem keeps its own LM state and
// fixed-order sums, so its result is the same in any batch.
namespace vlba {
namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Ticket {
  uint64_t id = 0;
  vlba_problem* problem = nullptr;
  vlba_config config{};
  Plan plan;
  size_t bytes = 0;
  uint64_t obs = 0;
  int status = VLBA_ERR_BUSY;
  uint64_t error_index = 0;
  std::string error;
  vlba_result result{};
  std::vector<vlba_iteration> iters;
  double t_submit = 0.0, t_start = 0.0, t_done = 0.0;
  uint32_t batch = 0, slot = 0;
  bool done = false;
};

struct Server {
  int device = 0;
  uint32_t max_batch = 64;
  size_t slot_bytes = 0;
  uint64_t large_obs = 100000;
  uint32_t plan_threads = 1;  // host threads per planner for one large plan
  std::vector<Context*> slots;
  PcgGate gate;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Ticket*> to_plan, ready;
  std::unordered_map<uint64_t, std::unique_ptr<Ticket>> tickets;
  uint64_t next_id = 1;
  uint32_t planning = 0;  // tickets taken by a planner, not yet ready or done
  bool stop = false;
  std::vector<std::thread> threads;
  std::string error;
};

// Device bytes a ticket's upload takes from a slot's slab (the plan's arrays
// plus its iteration records and the slab's alignment padding).
size_t ticket_bytes(const Plan& P, uint32_t records) {
  return P.device_bytes() + (size_t)records * sizeof(vlba_iteration) + 64 * 256 + (1u << 20);
}

void plan_ticket(Server* S, Ticket* t) {
  const Validation v = validate_problem(t->problem, &t->config);
  if (v.status != VLBA_OK) {
    t->status = v.status;
    t->error_index = v.error_index;
    t->error = "validation";
    return;
  }
  try {
    const vlba_problem* ps[1] = {t->problem};
    const vlba_config* cs[1] = {&t->config};
    build_plan(ps, cs, 1, (uint32_t)pick_tb(ps, 1), &t->plan, S->plan_threads);
    const std::string bad = check_plan(t->plan);
    if (!bad.empty()) throw Status(VLBA_ERR_INVALID_ARGUMENT, bad);
    t->bytes = ticket_bytes(t->plan, t->config.max_iterations);
    t->obs = t->problem->num_observations;
    if (t->bytes > S->slot_bytes)
      throw Status(VLBA_ERR_OUT_OF_MEMORY, "request larger than a serving slot's memory");
    t->status = VLBA_ERR_BUSY;
  } catch (const Status& e) {
    t->status = e.code;
    t->error = e.what();
  } catch (const std::exception& e) {
    t->status = VLBA_ERR_INVALID_ARGUMENT;
    t->error = e.what();
  }
}

void planner_loop(Server* S) {
  for (;;) {
    Ticket* t = nullptr;
    {
      std::unique_lock<std::mutex> lock(S->mu);
      S->cv.wait(lock, [&] { return S->stop || !S->to_plan.empty(); });
      if (S->to_plan.empty()) return;  // stopping
      t = S->to_plan.front();
      S->to_plan.pop_front();
      ++S->planning;
    }
    plan_ticket(S, t);
    std::lock_guard<std::mutex> lock(S->mu);
    --S->planning;
    if (t->status == VLBA_ERR_BUSY) {
      S->ready.push_back(t);
    } else {
      t->done = true;
      t->t_done = now_ms();
    }
    S->cv.notify_all();
  }
}

// Takes the next batch from the ready queue (caller holds the lock): a large
// request alone when it is first in line, else small requests in arrival
// order up to the slot's memory and the batch cap (large ones wait for the
// next slot).
std::vector<Ticket*> take_batch(Server* S) {
  std::vector<Ticket*> batch;
  size_t bytes = 0;
  for (auto it = S->ready.begin(); it != S->ready.end() && batch.size() < S->max_batch;) {
    Ticket* t = *it;
    if (t->obs >= S->large_obs) {
      if (batch.empty()) {
        batch.push_back(t);
        S->ready.erase(it);
        break;
      }
      ++it;
      continue;
    }
    if (bytes + t->bytes > S->slot_bytes) break;
    bytes += t->bytes;
    batch.push_back(t);
    it = S->ready.erase(it);
  }
  return batch;
}

void run_batch(Server* S, uint32_t k, const std::vector<Ticket*>& batch) {
  Context* c = S->slots[k];
  const double t0 = now_ms();
  for (Ticket* t : batch) {
    t->t_start = t0;
    t->batch = (uint32_t)batch.size();
    t->slot = k;
  }
  try {
    set_device(c);
    std::vector<const Plan*> parts;
    uint32_t records = 1, flags = 0;
    for (Ticket* t : batch) {
      parts.push_back(&t->plan);
      records = std::max(records, t->config.max_iterations);
      flags |= t->config.flags;
    }
    c->reduced_generation = ~0ull;
    if (parts.size() == 1) c->plan = std::move(batch[0]->plan);
    else merge_plans(parts, &c->plan);
    upload_plan(c, records);
    c->flags = flags & ~(uint32_t)(VLBA_FLAG_GRAPH | VLBA_FLAG_PROFILE);
    reset_state(c);
    PhaseTimes pt;
    const RunStats st = run_lm(c, false, &pt);
    std::vector<int> slot(batch.size());
    std::vector<vlba_result> res(batch.size());
    std::vector<vlba_iteration> its(batch.size() * (size_t)records);
    for (size_t i = 0; i < batch.size(); ++i) slot[i] = (int)i;
    fill_results_bulk(c, slot, res.data(), its.data(), records, st, nullptr);
    std::vector<vlba_problem*> probs;
    for (Ticket* t : batch) probs.push_back(t->problem);
    download_all(c, slot, probs.data());
    for (size_t i = 0; i < batch.size(); ++i) {
      Ticket* t = batch[i];
      t->result = res[i];
      const uint32_t m = std::min(res[i].num_iterations, records);
      t->iters.assign(its.begin() + i * records, its.begin() + i * records + m);
      t->status = VLBA_OK;
    }
  } catch (const Status& e) {
    for (Ticket* t : batch) {
      t->status = e.code;
      t->error = e.what();
    }
  } catch (const CudaError& e) {
    for (Ticket* t : batch) {
      t->status = e.code == cudaErrorMemoryAllocation ? VLBA_ERR_OUT_OF_MEMORY : VLBA_ERR_CUDA;
      t->error = e.what();
    }
  } catch (const std::exception& e) {
    for (Ticket* t : batch) {
      t->status = VLBA_ERR_INVALID_ARGUMENT;
      t->error = e.what();
    }
  }
  for (Ticket* t : batch) t->plan = Plan();  // the host plan is no longer needed
  std::lock_guard<std::mutex> lock(S->mu);
  const double t1 = now_ms();
  for (Ticket* t : batch) {
    t->done = true;
    t->t_done = t1;
  }
  S->cv.notify_all();
}

void worker_loop(Server* S, uint32_t k) {
  cudaSetDevice(S->device);
  for (;;) {
    std::vector<Ticket*> batch;
    {
      std::unique_lock<std::mutex> lock(S->mu);
      // Stop only once every submitted ticket has been planned and taken.
      S->cv.wait(lock, [&] {
        return !S->ready.empty() || (S->stop && S->to_plan.empty() && S->planning == 0);
      });
      if (S->ready.empty()) return;
      batch = take_batch(S);
    }
    if (!batch.empty()) run_batch(S, k, batch);
  }
}

void stop_server(Server* S) {
  {
    std::lock_guard<std::mutex> lock(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  for (auto& t : S->threads)
    if (t.joinable()) t.join();
  for (Context* c : S->slots) free_context(c);
  S->slots.clear();
  if (S->gate.last) cudaEventDestroy(S->gate.last);
  S->gate.last = nullptr;
}

}  // namespace
}  // namespace vlba

extern "C" {

void* visloc_ba_cuda_server_create(int device, uint32_t slots, uint64_t memory_bytes,
                                   uint32_t max_batch) {
  auto* S = new (std::nothrow) vlba::Server();
  if (!S) return nullptr;
  try {
    S->device = device;
    if (slots == 0) slots = 3;
    if (max_batch) S->max_batch = max_batch;
    VLBA_CUDA(cudaSetDevice(device));
    if (memory_bytes == 0) {
      size_t free_b = 0, total_b = 0;
      VLBA_CUDA(cudaMemGetInfo(&free_b, &total_b));
      memory_bytes = free_b / 2;
    }
    S->slot_bytes = (size_t)(memory_bytes / slots);
    VLBA_CUDA(cudaEventCreateWithFlags(&S->gate.last, cudaEventDisableTiming));
    for (uint32_t k = 0; k < slots; ++k) {
      vlba::Context* c = vlba::make_context(device);
      S->slots.push_back(c);
      c->arena.use_slab(S->slot_bytes);
      c->gate = &S->gate;
      vlba::reserve_stage(c, vlba::kStageMax);  // at full size before the first request
    }
    const uint32_t planners =
        std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2));
    S->plan_threads = std::max(1u, std::thread::hardware_concurrency() / planners);
    for (uint32_t i = 0; i < planners; ++i) S->threads.emplace_back(vlba::planner_loop, S);
    for (uint32_t k = 0; k < slots; ++k) S->threads.emplace_back(vlba::worker_loop, S, k);
  } catch (...) {
    vlba::stop_server(S);
    delete S;
    return nullptr;
  }
  return S;
}

void visloc_ba_cuda_server_destroy(void* server) {
  auto* S = static_cast<vlba::Server*>(server);
  if (!S) return;
  vlba::stop_server(S);
  delete S;
}

int visloc_ba_cuda_server_submit(void* server, vlba_problem* problem, const vlba_config* config,
                                 uint64_t* ticket) {
  auto* S = static_cast<vlba::Server*>(server);
  if (!S || !problem || !config || !ticket) return VLBA_ERR_INVALID_ARGUMENT;
  auto t = std::make_unique<vlba::Ticket>();
  t->problem = problem;
  t->config = *config;
  t->t_submit = vlba::now_ms();
  std::lock_guard<std::mutex> lock(S->mu);
  if (S->stop) return VLBA_ERR_INVALID_ARGUMENT;
  t->id = S->next_id++;
  *ticket = t->id;
  S->to_plan.push_back(t.get());
  S->tickets.emplace(t->id, std::move(t));
  S->cv.notify_all();
  return VLBA_OK;
}

int visloc_ba_cuda_server_wait(void* server, uint64_t ticket, double timeout_ms,
                               vlba_result* result, vlba_iteration* iterations,
                               uint32_t iterations_capacity, vlba_ticket_info* info) {
  auto* S = static_cast<vlba::Server*>(server);
  if (!S) return VLBA_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(S->mu);
  auto it = S->tickets.find(ticket);
  if (it == S->tickets.end()) return VLBA_ERR_INVALID_ARGUMENT;
  vlba::Ticket* t = it->second.get();
  auto ready = [&] { return t->done; };
  if (timeout_ms < 0) S->cv.wait(lock, ready);
  else if (!S->cv.wait_for(lock, std::chrono::duration<double, std::milli>(timeout_ms), ready))
    return VLBA_ERR_BUSY;
  if (result) {
    *result = t->result;
    result->error_index = t->error_index;
  }
  if (iterations && iterations_capacity) {
    const size_t m = std::min<size_t>(iterations_capacity, t->iters.size());
    std::memcpy(iterations, t->iters.data(), m * sizeof(vlba_iteration));
  }
  if (info) {
    std::memset(info, 0, sizeof *info);
    info->latency_ms = t->t_done - t->t_submit;
    info->queue_ms = (t->t_start > 0.0 ? t->t_start : t->t_done) - t->t_submit;
    info->solve_ms = t->t_start > 0.0 ? t->t_done - t->t_start : 0.0;
    info->batch_size = t->batch;
    info->slot = t->slot;
  }
  const int st = t->status;
  if (st != VLBA_OK) S->error = t->error;
  S->tickets.erase(it);
  return st;
}

}  // extern "C"

namespace vlba {

bool reduced_system_ok(const vlba_reduced_system* sys) {
  return sys && sys->diag && sys->rhs && sys->num_nodes != 0 &&
         (!sys->num_edges || sys->edges) && sys->tol >= 0.0;
}

// Plans and uploads a reduced system given in the reference's layout and
// fills S's tiles, the block-Jacobi inverses and the rhs on the device; with
// no off-diagonal blocks (offdiag null), from the blocks of the context's
// last elimination of the same edges.
void reduced_setup(Context* c, const vlba_reduced_system* sys) {
  const bool resident = sys->num_edges && !sys->offdiag;
  if (resident) {
    const ElimState* E = c->elim.get();
    if (!E || !E->blocks_valid || E->n != sys->num_nodes || E->num_edges != sys->num_edges ||
        std::memcmp(E->edges.data(), sys->edges, 8 * sys->num_edges) != 0)
      throw Status(VLBA_DECLINED, "no off-diagonal blocks given and none formed for these edges");
  }
  vlba_config cfg;
  visloc_ba_cuda_default_config(&cfg);
  cfg.max_pcg_iterations = sys->max_iterations;
  cfg.pcg_relative_tolerance = sys->tol;
  const LmParams lp = make_params(&cfg);
  const size_t n = sys->num_nodes, ne = sys->num_edges;
  cudaStream_t s = c->stream;
  // The layout (tiles, block destinations, PCG lists) depends on the edges
  // only: rebuilt when they change or another upload replaced it.
  const bool same = c->reduced_generation == c->plan_generation && c->reduced_nodes == n &&
                    c->reduced_edges.size() == 2 * ne &&
                    (ne == 0 || std::memcmp(c->reduced_edges.data(), sys->edges, 8 * ne) == 0);
  if (!same) {
    // Edges out of order or repeated: the reference's solver declines them
    // (its product needs each node's edges contiguous), and so does this one.
    for (uint64_t e = 0; e < ne; ++e) {
      const uint32_t a = sys->edges[2 * e], b = sys->edges[2 * e + 1];
      if (!(a < b && b < n))
        throw Status(VLBA_ERR_INVALID_ARGUMENT, "edge " + std::to_string(e) +
                                                    " is not (a, b) with a < b < nodes");
      if (e && ((uint64_t)sys->edges[2 * e - 2] << 32 | sys->edges[2 * e - 1]) >=
                   ((uint64_t)a << 32 | b))
        throw Status(VLBA_DECLINED, "edges are not sorted and distinct at " + std::to_string(e));
    }
    c->reduced_generation = ~0ull;
    build_reduced_plan(sys->num_nodes, sys->edges, sys->num_edges, 8, lp, &c->plan);
    const std::string bad = check_plan(c->plan);
    if (!bad.empty()) throw Status(VLBA_ERR_INVALID_ARGUMENT, bad);
    upload_plan(c, 1);
    c->reduced_edges.assign(sys->edges, sys->edges + 2 * ne);
    c->reduced_nodes = (uint32_t)n;
    c->reduced_generation = c->plan_generation;
  } else {
    c->plan.params[0] = lp;  // this call's tolerance and iteration cap
    VLBA_CUDA(cudaMemcpyAsync(const_cast<LmParams*>(c->dev.params), &c->plan.params[0],
                              sizeof(LmParams), cudaMemcpyHostToDevice, s));
  }
  // The caller's arrays, staged for the fill kernel through pinned memory.
  const size_t b_diag = 288 * n, b_rhs = 48 * n, b_off = resident ? 0 : 144 * ne;
  c->reduced_in.ensure(b_diag + b_rhs + b_off);
  char* in = c->reduced_in.as<char>();
  VLBA_CUDA(cudaEventRecord(c->ev[0], s));
  {
    Stager st(c);
    st.add(in, sys->diag, b_diag);
    st.add(in + b_diag, sys->rhs, b_rhs);
    if (b_off) st.add(in + b_diag + b_rhs, sys->offdiag, b_off);
    st.flush(s);
  }
  reset_state(c);
  check_launch(launch_reduced_fill(c->dev, (uint32_t)n, ne, reinterpret_cast<const double*>(in),
                                   b_off ? reinterpret_cast<const float*>(in + b_diag + b_rhs)
                                         : nullptr,
                                   resident ? c->elim->blocks.as<const double>() : nullptr,
                                   reinterpret_cast<const double*>(in + b_diag), s),
               "reduced fill");
  VLBA_CUDA(cudaEventRecord(c->ev[1], s));
  VLBA_CUDA(cudaStreamSynchronize(s));
  float ms = 0.0f;
  VLBA_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
  c->reduced_ms.fill_ms = ms;
}

// Device time from ev[2] (recorded at the PCG loop's start) to now.
void record_pcg_ms(Context* c) {
  VLBA_CUDA(cudaEventRecord(c->ev[3], c->stream));
  VLBA_CUDA(cudaEventSynchronize(c->ev[3]));
  float ms = 0.0f;
  VLBA_CUDA(cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]));
  c->reduced_ms.pcg_ms = ms;
}

void download_step(Context* c, size_t n, double* x) {
  std::vector<float> xf(6 * n);
  VLBA_CUDA(cudaMemcpyAsync(xf.data(), c->dev.x, xf.size() * 4, cudaMemcpyDeviceToHost, c->stream));
  VLBA_CUDA(cudaStreamSynchronize(c->stream));
  for (size_t i = 0; i < xf.size(); ++i) x[i] = xf[i];
}

constexpr uint32_t kMaxRunNodes = 1024;
constexpr uint32_t kMaxAggregates = 2048;

// The preconditioner's shape against the system's node count.
std::string check_preconditioner(const vlba_reduced_preconditioner* pre, uint32_t n) {
  if (!pre) return "";
  if (pre->num_clusters) {
    if (!pre->cluster_first || !pre->cluster_size || !pre->cluster_inverse)
      return "cluster arrays missing";
    uint64_t next = 0;
    for (uint32_t k = 0; k < pre->num_clusters; ++k) {
      const uint64_t f = pre->cluster_first[k], m = pre->cluster_size[k];
      if (m == 0 || m > kMaxRunNodes)
        return "run " + std::to_string(k) + " has " + std::to_string(m) + " nodes (1 to 1024)";
      if (f < next || f + m > n)
        return "run " + std::to_string(k) + " overlaps another or leaves the system";
      next = f + m;
    }
  }
  if (pre->coarse_nodes) {
    if (pre->coarse_group == 0 || pre->coarse_nodes > n || !pre->coarse_inverse)
      return "coarse level: group 0, too many nodes or no inverse";
    if ((pre->coarse_nodes + (uint64_t)pre->coarse_group - 1) / pre->coarse_group > kMaxAggregates)
      return "coarse level: more than 2048 aggregates";
  }
  return "";
}

// Iterations per CUDA graph launch of the preconditioned loop (the host
// checks the done flag between launches).
constexpr int kRpChunk = 8;

void reduced_solve_preconditioned(Context* c, const vlba_reduced_system* sys,
                                  const vlba_reduced_preconditioner* pre, double* x,
                                  uint32_t* iterations, double* relative_residual) {
  const size_t n = sys->num_nodes;
  cudaStream_t s = c->stream;
  Dev& d = c->dev;
  RpData rp{};
  // One device block: the scalars, the run tables and inverses, the coarse
  // inverse (row-major) and its two vectors.
  const uint32_t nc = pre ? pre->num_clusters : 0;
  std::vector<uint64_t> cl_off(nc);
  uint64_t cl_floats = 0;
  uint32_t max_rows = 0;
  for (uint32_t k = 0; k < nc; ++k) {
    const uint64_t rows = 6ull * pre->cluster_size[k];
    cl_off[k] = cl_floats;
    cl_floats += rows * rows;
    max_rows = std::max<uint32_t>(max_rows, (uint32_t)rows);
  }
  const uint32_t m = (pre && pre->coarse_nodes)
                         ? (pre->coarse_nodes + pre->coarse_group - 1) / pre->coarse_group
                         : 0;
  const uint64_t cm = 6ull * m;
  auto up16 = [](uint64_t b) { return (b + 15) & ~uint64_t(15); };
  const uint64_t o_first = up16(sizeof(RpScalars)), o_size = o_first + up16(4ull * nc),
                 o_off = o_size + up16(4ull * nc), o_mat = o_off + up16(8ull * nc),
                 o_cinv = o_mat + up16(4 * cl_floats), o_rc = o_cinv + up16(4 * cm * cm),
                 o_yc = o_rc + up16(4 * cm), total = o_yc + up16(4 * cm);
  c->reduced_pre.ensure(total);
  char* base = c->reduced_pre.as<char>();
  {
    std::vector<float> mat(cl_floats), cinv(cm * cm);
    if (nc) {
      std::atomic<uint32_t> next{0};
      auto work = [&] {
        for (uint32_t k; (k = next.fetch_add(1)) < nc;) {
          const uint64_t cnt = 36ull * pre->cluster_size[k] * pre->cluster_size[k];
          const double* src = pre->cluster_inverse + cl_off[k];
          for (uint64_t e = 0; e < cnt; ++e) mat[cl_off[k] + e] = (float)src[e];
        }
      };
      const unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 32u));
      std::vector<std::thread> pool;
      for (unsigned t = 1; t < std::min<unsigned>(nt, nc); ++t) pool.emplace_back(work);
      work();
      for (auto& t : pool) t.join();
      VLBA_CUDA(cudaMemcpyAsync(base + o_first, pre->cluster_first, 4ull * nc, cudaMemcpyHostToDevice, s));
      VLBA_CUDA(cudaMemcpyAsync(base + o_size, pre->cluster_size, 4ull * nc, cudaMemcpyHostToDevice, s));
      VLBA_CUDA(cudaMemcpyAsync(base + o_off, cl_off.data(), 8ull * nc, cudaMemcpyHostToDevice, s));
      VLBA_CUDA(cudaMemcpyAsync(base + o_mat, mat.data(), 4 * cl_floats, cudaMemcpyHostToDevice, s));
    }
    if (m) {
      for (uint64_t r = 0; r < cm; ++r)
        for (uint64_t col = 0; col < cm; ++col)
          cinv[r * cm + col] = (float)pre->coarse_inverse[col * cm + r];
      VLBA_CUDA(cudaMemcpyAsync(base + o_cinv, cinv.data(), 4 * cm * cm, cudaMemcpyHostToDevice, s));
    }
    VLBA_CUDA(cudaMemsetAsync(base, 0, sizeof(RpScalars), s));
    VLBA_CUDA(cudaStreamSynchronize(s));  // the host copies above are freed next
  }
  rp.sc = reinterpret_cast<RpScalars*>(base);
  rp.dots = d.dots;
  rp.num_clusters = nc;
  rp.max_cluster_rows = max_rows;
  rp.cl_first = reinterpret_cast<const uint32_t*>(base + o_first);
  rp.cl_size = reinterpret_cast<const uint32_t*>(base + o_size);
  rp.cl_off = reinterpret_cast<const uint64_t*>(base + o_off);
  rp.cl_mat = reinterpret_cast<const float*>(base + o_mat);
  rp.coarse_m = m;
  rp.coarse_group = m ? pre->coarse_group : 1;
  rp.coarse_nodes = m ? pre->coarse_nodes : 0;
  rp.coarse_inv = reinterpret_cast<const float*>(base + o_cinv);
  rp.rc = reinterpret_cast<float*>(base + o_rc);
  rp.yc = reinterpret_cast<float*>(base + o_yc);
  rp.max_iterations = sys->max_iterations;
  rp.tol = sys->tol;

  VLBA_CUDA(cudaEventRecord(c->ev[2], s));
  check_launch(launch_rp_init(d, rp, s), "preconditioned solve init");
  // kRpChunk iterations as one graph, launched until the device says done.
  struct Graph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~Graph() {
      if (e) cudaGraphExecDestroy(e);
      if (g) cudaGraphDestroy(g);
    }
  } gr;
  VLBA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaError_t le = cudaSuccess;
  for (int k = 0; k < kRpChunk && le == cudaSuccess; ++k) le = launch_rp_iteration(d, rp, s);
  const cudaError_t ce = cudaStreamEndCapture(s, &gr.g);
  check_launch(le, "preconditioned solve iteration");
  VLBA_CUDA(ce);
  VLBA_CUDA(cudaGraphInstantiate(&gr.e, gr.g, 0));
  RpScalars sc{};
  for (uint64_t launched = 0;; launched += kRpChunk) {
    VLBA_CUDA(cudaMemcpyAsync(&sc, rp.sc, sizeof sc, cudaMemcpyDeviceToHost, s));
    VLBA_CUDA(cudaStreamSynchronize(s));
    if (sc.done || launched >= sys->max_iterations) break;
    VLBA_CUDA(cudaGraphLaunch(gr.e, s));
  }
  record_pcg_ms(c);
  if (sc.failed)
    throw Status(VLBA_DECLINED, "p.q not positive and finite at iteration " +
                                    std::to_string(sc.iters + 1) + ": the CPU solver takes the system");
  download_step(c, n, x);
  if (iterations) *iterations = sc.iters;
  if (relative_residual) *relative_residual = sc.bnorm > 0 ? sc.rnorm / sc.bnorm : 0.0;
}

// ReducedSolveAccelerator::eliminate on the device.  Returns false (and
// sets nothing) when a returned block is not finite.
bool reduced_eliminate(Context* c, const vlba_point_elimination* el, double* run_blocks,
                       double* coarse_sums) {
  cudaStream_t s = c->stream;
  const uint32_t n = el->num_nodes, P = el->num_points;
  const uint64_t ne = el->num_edges, nobs = el->point_off[P];
  if (!c->elim) c->elim = std::make_unique<ElimState>();
  ElimState& E = *c->elim;
  E.blocks_valid = false;
  if (E.structure_id != el->structure_id || E.n != n || E.num_points != P ||
      E.num_edges != ne || E.num_obs != nobs) {
    E.structure_id = 0;
    E.hcp_valid = false;
    ElimIndex X;
    const std::string bad =
        build_elimination_index(n, el->edges, ne, P, el->point_off, el->point_nodes, &X);
    if (!bad.empty()) throw Status(VLBA_ERR_INVALID_ARGUMENT, bad);
    // The structure on the device; its pair index built there: counts per
    // edge, their prefix here, then the pairs at each edge's cursor.
    E.row_off.ensure(4 * X.row_off.size());
    E.edge_t.ensure(4 * ne);
    E.slot_off.ensure(4 * X.slot_off.size());
    E.slot_obs.ensure(4 * nobs);
    E.obs_point.ensure(4 * nobs);
    E.point_off32.ensure(4 * X.point_off.size());
    E.point_nodes.ensure(4 * nobs);
    E.pair_off.ensure(4 * (ne + 1));
    E.cursor.ensure(4 * ne);
    E.flag.ensure(4);
    {
      Stager st(c);
      st.add(E.row_off.p, X.row_off.data(), 4 * X.row_off.size());
      st.add(E.edge_t.p, X.edge_t.data(), 4 * ne);
      st.add(E.slot_off.p, X.slot_off.data(), 4 * X.slot_off.size());
      st.add(E.slot_obs.p, X.slot_obs.data(), 4 * nobs);
      st.add(E.obs_point.p, X.obs_point.data(), 4 * nobs);
      st.add(E.point_off32.p, X.point_off.data(), 4 * X.point_off.size());
      st.add(E.point_nodes.p, el->point_nodes, 4 * nobs);
      st.flush(s);
    }
    VLBA_CUDA(cudaMemsetAsync(E.cursor.p, 0, 4 * ne, s));
    VLBA_CUDA(cudaMemsetAsync(E.flag.p, 0, 4, s));
    ElimDev ix{};
    ix.n = n;
    ix.num_points = P;
    ix.num_edges = ne;
    ix.num_obs = nobs;
    ix.row_off = E.row_off.as<const uint32_t>();
    ix.edge_t = E.edge_t.as<const uint32_t>();
    ix.slot_off = E.slot_off.as<const uint32_t>();
    ix.slot_obs = E.slot_obs.as<const uint32_t>();
    ix.obs_point = E.obs_point.as<const uint32_t>();
    ix.point_off = E.point_off32.as<const uint32_t>();
    ix.point_nodes = E.point_nodes.as<const uint32_t>();
    ix.cursor = E.cursor.as<uint32_t>();
    ix.err = E.flag.as<unsigned int>();
    check_launch(launch_el_index(ix, false, s), "elimination index count");
    std::vector<uint32_t> cnt(ne + 1, 0);
    unsigned int ierr = 0;
    VLBA_CUDA(cudaMemcpyAsync(cnt.data(), E.cursor.p, 4 * ne, cudaMemcpyDeviceToHost, s));
    VLBA_CUDA(cudaMemcpyAsync(&ierr, E.flag.p, 4, cudaMemcpyDeviceToHost, s));
    VLBA_CUDA(cudaStreamSynchronize(s));
    if (ierr) throw Status(VLBA_ERR_INVALID_ARGUMENT, "two nodes of a point have no edge");
    uint64_t total = 0;
    for (uint64_t e = 0; e < ne; ++e) {
      const uint32_t k = cnt[e];
      cnt[e] = (uint32_t)total;
      total += k;
    }
    if (total >= (1ull << 32)) throw Status(VLBA_ERR_INVALID_ARGUMENT, "too many point pairs");
    cnt[ne] = (uint32_t)total;
    E.num_pairs = total;
    E.pairs.ensure(8 * total);
    VLBA_CUDA(cudaMemcpyAsync(E.pair_off.p, cnt.data(), 4 * (ne + 1), cudaMemcpyHostToDevice, s));
    VLBA_CUDA(cudaMemcpyAsync(E.cursor.p, cnt.data(), 4 * ne, cudaMemcpyHostToDevice, s));
    ix.pairs_out = E.pairs.as<uint2>();
    check_launch(launch_el_index(ix, true, s), "elimination index write");
    E.edges.assign(el->edges, el->edges + 2 * ne);
    E.hcp64.ensure(144 * nobs);
    E.hcp32.ensure(4 * kElRec * nobs);
    E.sk32.ensure(4 * kElRec * nobs);
    E.blocks.ensure(288 * ne);
    VLBA_CUDA(cudaStreamSynchronize(s));  // X's host arrays go next
    E.n = n;
    E.num_points = P;
    E.num_edges = ne;
    E.num_obs = nobs;
    E.structure_id = el->structure_id;
  }
  if (!E.hcp_valid || E.linearization_id != el->linearization_id) {
    Stager st(c);
    st.add(E.hcp64.p, el->hcp, 144 * nobs);
    st.flush(s);
    E.hcp_valid = true;
    E.linearization_id = el->linearization_id;
  }
  // Per call: the point inverses, the couplings (merged per edge in their
  // order), the run edges and the outputs.
  E.vinv64.ensure(72ull * P);
  VLBA_CUDA(cudaEventRecord(c->ev[4], s));
  Stager st(c);  // this call's uploads, through pinned memory
  st.add(E.vinv64.p, el->point_inverse, 72ull * P);
  if (el->point_used) {
    E.used.ensure(P);
    st.add(E.used.p, el->point_used, P);
  }
  std::vector<int32_t> extra_of;
  std::vector<double> extra;
  if (el->num_extra) {
    extra_of.assign(ne, -1);
    for (uint64_t i = 0; i < el->num_extra; ++i) {
      int32_t& x = extra_of[el->extra_edge[i]];
      if (x < 0) {
        x = (int32_t)(extra.size() / 36);
        extra.insert(extra.end(), el->extra_block + 36 * i, el->extra_block + 36 * i + 36);
      } else {
        for (int q = 0; q < 36; ++q) extra[36 * (size_t)x + q] += el->extra_block[36 * i + q];
      }
    }
    E.extra_of.ensure(4 * ne);
    E.extra64.ensure(8 * extra.size());
    st.add(E.extra_of.p, extra_of.data(), 4 * ne);
    st.add(E.extra64.p, extra.data(), 8 * extra.size());
  }
  const uint64_t nrun = el->num_run_edges;
  if (nrun) {
    E.run_edges.ensure(4 * nrun);
    E.run_out.ensure(288 * nrun);
    st.add(E.run_edges.p, el->run_edges, 4 * nrun);
  }
  st.flush(s);
  const uint32_t m = el->coarse_group && el->coarse_nodes
                         ? (el->coarse_nodes + el->coarse_group - 1) / el->coarse_group
                         : 0;
  const uint64_t nsum = 36ull * m * m;
  if (m) {
    E.coarse_out.ensure(8 * nsum);
    VLBA_CUDA(cudaMemsetAsync(E.coarse_out.p, 0, 8 * nsum, s));
  }
  ElimDev d{};
  d.n = n;
  d.num_points = P;
  d.num_edges = ne;
  d.num_obs = nobs;
  d.num_run = nrun;
  d.coarse_m = m;
  d.coarse_group = m ? el->coarse_group : 1;
  d.coarse_nodes = m ? el->coarse_nodes : 0;
  d.row_off = E.row_off.as<const uint32_t>();
  d.edge_t = E.edge_t.as<const uint32_t>();
  d.pair_off = E.pair_off.as<const uint32_t>();
  d.pairs = E.pairs.as<const uint2>();
  d.obs_point = E.obs_point.as<const uint32_t>();
  d.hcp64 = E.hcp64.as<const double>();
  d.vinv64 = E.vinv64.as<const double>();
  d.used = el->point_used ? E.used.as<const uint8_t>() : nullptr;
  d.hcp32 = E.hcp32.as<float>();
  d.sk32 = E.sk32.as<float>();
  d.extra_of = el->num_extra ? E.extra_of.as<const int32_t>() : nullptr;
  d.extra64 = el->num_extra ? E.extra64.as<const double>() : nullptr;
  d.blocks = E.blocks.as<double>();
  d.run_edges = E.run_edges.as<const uint32_t>();
  d.run_out = E.run_out.as<double>();
  d.coarse_out = E.coarse_out.as<double>();
  check_launch(launch_el_prepare(d, s), "elimination prepare");
  check_launch(launch_el_blocks(d, s), "elimination blocks");
  check_launch(launch_el_outputs(d, s), "elimination outputs");
  VLBA_CUDA(cudaEventRecord(c->ev[5], s));
  if (nrun)
    VLBA_CUDA(cudaMemcpyAsync(run_blocks, E.run_out.p, 288 * nrun, cudaMemcpyDeviceToHost, s));
  if (m && coarse_sums)
    VLBA_CUDA(cudaMemcpyAsync(coarse_sums, E.coarse_out.p, 8 * nsum, cudaMemcpyDeviceToHost, s));
  VLBA_CUDA(cudaStreamSynchronize(s));
  {
    float ms = 0.0f;
    VLBA_CUDA(cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]));
    c->reduced_ms.eliminate_ms = ms;
  }
  for (uint64_t i = 0; i < 36 * nrun; ++i)
    if (!std::isfinite(run_blocks[i])) return false;
  if (m && coarse_sums)
    for (uint64_t i = 0; i < nsum; ++i)
      if (!std::isfinite(coarse_sums[i])) return false;
  E.blocks_valid = true;
  return true;
}

}  // namespace vlba

extern "C" {

int visloc_ba_cuda_reduced_solve(void* ctx, const vlba_reduced_system* sys, double* x,
                                 uint32_t* iterations, double* relative_residual) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !x || !vlba::reduced_system_ok(sys)) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    vlba::set_device(c);
    vlba::reduced_setup(c, sys);
    cudaStream_t s = c->stream;
    vlba::Dev& d = c->dev;
    VLBA_CUDA(cudaEventRecord(c->ev[2], s));
    vlba::check_launch(vlba::launch_pcg_setup(d, s), "pcg setup");
    vlba::check_launch(vlba::launch_pcg(d, c->pcg_grid, s), "pcg");
    vlba::record_pcg_ms(c);
    vlba::PcgState pg;
    VLBA_CUDA(cudaMemcpyAsync(&pg, d.pcg, sizeof pg, cudaMemcpyDeviceToHost, s));
    unsigned int err = 0;
    VLBA_CUDA(cudaMemcpyAsync(&err, d.error, 4, cudaMemcpyDeviceToHost, s));
    VLBA_CUDA(cudaStreamSynchronize(s));
    if (err) throw vlba::Status(VLBA_ERR_TIMEOUT, "a bounded device wait gave up");
    vlba::download_step(c, sys->num_nodes, x);
    if (iterations) *iterations = pg.iters;
    if (relative_residual) *relative_residual = pg.bnorm > 0 ? pg.rnorm / pg.bnorm : 0.0;
  });
}

int visloc_ba_cuda_reduced_solve_preconditioned(void* ctx, const vlba_reduced_system* sys,
                                                const vlba_reduced_preconditioner* pre,
                                                double* x, uint32_t* iterations,
                                                double* relative_residual) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !x || !vlba::reduced_system_ok(sys)) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    const std::string bad = vlba::check_preconditioner(pre, sys->num_nodes);
    if (!bad.empty()) throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, bad);
    vlba::set_device(c);
    vlba::reduced_setup(c, sys);
    vlba::reduced_solve_preconditioned(c, sys, pre, x, iterations, relative_residual);
  });
}

int visloc_ba_cuda_reduced_eliminate(void* ctx, const vlba_point_elimination* el,
                                     double* run_blocks, double* coarse_sums) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !el || el->structure_id == 0 || el->num_nodes == 0 || !el->point_off ||
      (el->num_edges && !el->edges) || (el->num_points && !el->point_inverse) ||
      (el->num_extra && (!el->extra_edge || !el->extra_block)) ||
      (el->num_run_edges && (!el->run_edges || !run_blocks)))
    return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    const uint64_t nobs = el->point_off[el->num_points];
    if (nobs && (!el->point_nodes || !el->hcp))
      throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "point_nodes or hcp missing");
    for (uint64_t i = 0; i < el->num_extra; ++i)
      if (el->extra_edge[i] >= el->num_edges)
        throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "extra coupling " + std::to_string(i) +
                                                          " names no edge");
    for (uint64_t i = 0; i < el->num_run_edges; ++i)
      if (el->run_edges[i] >= el->num_edges)
        throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "run edge " + std::to_string(i) +
                                                          " names no edge");
    if (el->coarse_group &&
        (el->coarse_nodes > el->num_nodes || !coarse_sums ||
         (el->coarse_nodes + (uint64_t)el->coarse_group - 1) / el->coarse_group > 2048))
      throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT,
                         "coarse level: more nodes than the system, no output or over 2048 "
                         "aggregates");
    vlba::set_device(c);
    if (!vlba::reduced_eliminate(c, el, run_blocks, coarse_sums))
      throw vlba::Status(VLBA_DECLINED, "an eliminated block is not finite");
  });
}

int visloc_ba_cuda_reduced_timing(void* ctx, vlba_reduced_timing* out) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !out) return VLBA_ERR_INVALID_ARGUMENT;
  *out = c->reduced_ms;
  return VLBA_OK;
}

int visloc_ba_cuda_wait_probe(void* ctx, double limit_ms, double* waited_ms) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !(limit_ms >= 0.0) || limit_ms > 10000.0) return VLBA_ERR_INVALID_ARGUMENT;
  unsigned int err = 0;
  const int st = vlba::guarded(c, [&] {
    vlba::set_device(c);
    struct Words {
      void* p = nullptr;
      ~Words() {
        if (p) cudaFree(p);
      }
    } w;
    VLBA_CUDA(cudaMalloc(&w.p, 16));
    VLBA_CUDA(cudaMemsetAsync(w.p, 0, 16, c->stream));
    auto* flag = static_cast<unsigned int*>(w.p);
    auto* waited = reinterpret_cast<unsigned long long*>(static_cast<char*>(w.p) + 8);
    vlba::check_launch(vlba::launch_wait_probe(flag, (unsigned long long)(limit_ms * 1e6),
                                               flag + 1, waited, c->stream),
                       "wait probe");
    unsigned long long ns = 0;
    VLBA_CUDA(cudaMemcpyAsync(&err, flag + 1, 4, cudaMemcpyDeviceToHost, c->stream));
    VLBA_CUDA(cudaMemcpyAsync(&ns, waited, 8, cudaMemcpyDeviceToHost, c->stream));
    VLBA_CUDA(cudaStreamSynchronize(c->stream));
    if (waited_ms) *waited_ms = ns / 1e6;
  });
  if (st != VLBA_OK) return st;
  if (err) {
    c->error = "the wait gave up as bounded (a flag that nothing sets)";
    return VLBA_ERR_TIMEOUT;
  }
  return VLBA_OK;
}

int visloc_ba_cuda_autotune(void* ctx, vlba_launch_shape* chosen) {
  auto* c = static_cast<Context*>(ctx);
  if (!c) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    if (!c->uploaded) throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "nothing uploaded");
    vlba::set_device(c);
    {  // a new measurement, not the cached shape
      std::lock_guard<std::mutex> lock(vlba::g_tune_mu);
      vlba::g_tune_cache.erase(vlba::shape_key(c->plan));
    }
    const vlba::LaunchShape sh = vlba::autotune(c);
    if (chosen) {
      std::memset(chosen, 0, sizeof *chosen);
      chosen->pcg_blocks = c->pcg_grid;
      chosen->l2_resident_fraction = sh.l2_fraction;
      chosen->pcg_iteration_us = sh.pcg_iteration_us;
    }
  });
}

int visloc_ba_cuda_set_launch_shape(void* ctx, const vlba_launch_shape* shape) {
  auto* c = static_cast<Context*>(ctx);
  if (!c || !shape) return VLBA_ERR_INVALID_ARGUMENT;
  return vlba::guarded(c, [&] {
    if (!c->uploaded) throw vlba::Status(VLBA_ERR_INVALID_ARGUMENT, "nothing uploaded");
    vlba::LaunchShape sh;
    sh.pcg_grid = shape->pcg_blocks;
    sh.l2_fraction = shape->l2_resident_fraction;
    vlba::apply_shape(c, sh);
    c->tuned = true;
  });
}

const char* visloc_ba_cuda_server_last_error(void* server) {
  auto* S = static_cast<vlba::Server*>(server);
  return S ? S->error.c_str() : "null server";
}

}  // extern "C"
