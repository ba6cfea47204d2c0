// vlba_reduced.cu -- preconditioned CG on an uploaded reduced camera system
// with the reference's run inverses and additive coarse level
// (ReducedCameraSystem::clusters / coarse, pipelines/slam/src/ba_accel.rs:
// 50-72; the iteration of crates/ba-gpu/src/shaders/reduced_pcg.wgsl):
//
//   z = M r:  z_run = inverse of the run's block of S times r_run over each
//             run of consecutive nodes, the 6x6 block-Jacobi inverse for
//             nodes in no run, plus (coarse level) P (P^T S P)^-1 P^T r with
//             P summing each aggregate of `coarse_group` leading nodes.
//
// The system is the uploaded plan's tiles (the same S the persistent PCG
// kernel streams); the loop is a sequence of small kernels with every scalar
// on the device (no host round trip inside an iteration), each returning at
// once when the solve is over.  Vectors are FP32 as in the persistent PCG,
// dots FP64; every sum runs in a fixed order, so a solve is deterministic.
//
// Also here: the point elimination of ReducedSolveAccelerator::eliminate
// (ba_accel.rs:74-144) -- the structure's pair index (k_el_index), the
// FP32 camera-point blocks and their products with the point inverses
// (k_el_prepare), the per-edge FP64 block sums (k_el_blocks), and the run
// blocks and coarse aggregate-pair sums returned to the caller.
#include <cuda_runtime.h>

#include <algorithm>

#include "vlba_kernels.cuh"

namespace vlba {
namespace {

constexpr int kRow = 48;  // floats of a tile row (8 nodes x 6)

__device__ __forceinline__ bool rp_done(const RpData& r) {
  return *(volatile const uint32_t*)&r.sc->done != 0u;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Per tile row R, one warp: entries e = lane and lane + 32 (< 48).
#define RP_ROW_LOOP(d)                                                              \
  const uint32_t lane = threadIdx.x & 31u;                                          \
  const uint32_t R = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;                  \
  if (R >= (d).num_tile_rows) return;                                               \
  const size_t base = (size_t)R * kRow;                                             \
  const bool e1 = lane + 32u < (uint32_t)kRow;

// x = 0, r = b; the rows' |b|^2.
__global__ void k_rp_init_xr(Dev d, RpData rp) {
  RP_ROW_LOOP(d)
  double bb = 0.0;
  for (uint32_t e = lane; e < (uint32_t)kRow; e += 32) {
    const float b = d.rhs[base + e];
    d.x[base + e] = 0.0f;
    d.r[base + e] = b;
    bb += (double)b * (double)b;
  }
  (void)e1;
  bb = warp_sum_d(bb);
  if (lane == 0) rp.dots[2 * (size_t)d.num_tile_rows + R] = bb;
}

// 16-byte asynchronous global -> shared copies (LDGSTS), committed as groups.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int kTileFloats = 64 * kBlock;   // 8 x 8 blocks of 36 floats
constexpr int kMatvecWarps = 4;            // warps per block, each with a 2-tile ring
constexpr size_t kMatvecSmem = (size_t)kMatvecWarps * 2 * kTileFloats * sizeof(float);

// One warp per tile: the row-side partial S_IJ p_J and, off the diagonal,
// the column-side partial S_IJ^T p_I into the tile's partial slots (as the
// persistent PCG kernel does).  Each warp streams its tiles through a
// two-stage shared-memory ring: coalesced 16-byte copies of the next tile
// in flight while it multiplies the current one; lane l reads blocks l and
// l + 32 as float4 at a 144-byte stride, free of bank conflicts within each
// quarter warp.
__global__ void __launch_bounds__(kMatvecWarps * 32) k_rp_matvec(Dev d, RpData rp) {
  if (rp_done(rp)) return;
  extern __shared__ __align__(16) float rp_smem[];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  float* ring = rp_smem + (size_t)warp * 2 * kTileFloats;
  const uint32_t nw = gridDim.x * kMatvecWarps;
  const int li = (int)(lane >> 3), lj = (int)(lane & 7);
  auto issue = [&](uint32_t tile, int stage) {
    const float4* src = reinterpret_cast<const float4*>(d.tiles + (size_t)tile * kTileFloats);
    float* dst = ring + stage * kTileFloats;
#pragma unroll
    for (int k = 0; k < kTileFloats / 4 / 32; ++k)
      cp_async16(dst + 4 * (k * 32 + lane), src + k * 32 + lane);
    cp_async_commit();
  };
  uint32_t t = blockIdx.x * kMatvecWarps + warp;
  int st = 0;
  if (t < d.num_tiles) issue(t, 0);
  for (; t < d.num_tiles; t += nw) {
    const uint32_t tn = t + nw;
    if (tn < d.num_tiles) {
      issue(tn, st ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncwarp();  // every lane's copies of this tile have landed
    const uint4 meta = reinterpret_cast<const uint4*>(d.tile_meta)[t];
    const uint32_t I = meta.x >> 16, J = meta.x & 0xFFFFu;
    const float* tile = ring + st * kTileFloats;
    float pj[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) pj[c] = d.p[(size_t)J * kRow + lj * 6 + c];
    float row[2][6], col[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float4* blk = reinterpret_cast<const float4*>(tile + (size_t)(lane + 32 * h) * kBlock);
      float sv[36];
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        const float4 v = blk[q];
        sv[4 * q] = v.x;
        sv[4 * q + 1] = v.y;
        sv[4 * q + 2] = v.z;
        sv[4 * q + 3] = v.w;
      }
      float pi[6];
#pragma unroll
      for (int a = 0; a < 6; ++a) pi[a] = d.p[(size_t)I * kRow + (li + 4 * h) * 6 + a];
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        float acc = 0.0f;
#pragma unroll
        for (int c = 0; c < 6; ++c) acc += sv[a * 6 + c] * pj[c];
        row[h][a] = acc;
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        float acc = 0.0f;
#pragma unroll
        for (int a = 0; a < 6; ++a) acc += sv[a * 6 + c] * pi[a];
        col[c] += acc;
      }
    }
    __syncwarp();  // the stage is read: the next issue may overwrite it
#pragma unroll
    for (int off = 4; off > 0; off >>= 1)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int a = 0; a < 6; ++a) row[h][a] += __shfl_xor_sync(0xffffffffu, row[h][a], off);
    if (lj == 0) {
      float* part = d.partial + (size_t)meta.y * kRow;
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int a = 0; a < 6; ++a) part[(li + 4 * h) * 6 + a] = row[h][a];
    }
    if (I != J) {
#pragma unroll
      for (int off = 8; off < 32; off <<= 1)
#pragma unroll
        for (int c = 0; c < 6; ++c) col[c] += __shfl_xor_sync(0xffffffffu, col[c], off);
      if (li == 0) {
        float* part = d.partial + (size_t)meta.z * kRow;
#pragma unroll
        for (int c = 0; c < 6; ++c) part[lj * 6 + c] = col[c];
      }
    }
    st ^= 1;
  }
}

// ---- scalar steps
// The rows' dots of a step summed lane-strided by one warp, then by a
// butterfly (a fixed order), and the step's scalars; run by warp 0 of the
// last block of a row kernel to finish (rp_arrive).
enum RpStep { kRpInit = 0, kRpAlpha = 1, kRpCheck = 2, kRpBeta = 3 };
__device__ void rp_scalar_step(const Dev& d, const RpData& rp, int step) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t rows = d.num_tile_rows;
  const double* v = rp.dots + (size_t)(step == kRpAlpha ? 0 : step == kRpBeta ? 1 : 2) * rows;
  double s = 0.0;
  for (uint32_t r = lane; r < rows; r += 32) s += __ldcg(v + r);
  s = warp_sum_d(s);
  double rz = 0.0;
  if (step == kRpInit) {  // |b|^2 and the initial r.z
    for (uint32_t r = lane; r < rows; r += 32) rz += __ldcg(rp.dots + rows + r);
    rz = warp_sum_d(rz);
  }
  if (lane != 0) return;
  RpScalars& sc = *rp.sc;
  switch (step) {
    case kRpInit:
      sc.bnorm = sqrt(s);
      sc.rnorm = sc.bnorm;
      sc.rz = rz;
      sc.iters = 0u;
      if (!(sc.bnorm > 0.0) || rp.max_iterations == 0u) sc.done = 1u;
      break;
    case kRpAlpha:  // a non-positive or non-finite curvature fails the solve
      if (s > 0.0 && isfinite(s)) {
        sc.alpha = sc.rz / s;
      } else {
        sc.failed = 1u;
        sc.done = 1u;
      }
      break;
    case kRpCheck:
      sc.iters += 1u;
      sc.rnorm = sqrt(s);
      if (sc.rnorm <= rp.tol * sc.bnorm || sc.iters >= rp.max_iterations) sc.done = 1u;
      break;
    default:  // beta = r.z (new) / r.z (old)
      sc.beta = s / sc.rz;
      sc.rz = s;
      break;
  }
}

// Every block of a row kernel arrives once its rows' dots are written and
// fenced; the last block to arrive (the one that sees the count reach the
// grid size) resets the count and runs the scalar step.  No block waits for
// another.  Every thread of the block must call it.
__device__ void rp_arrive(const Dev& d, const RpData& rp, int step) {
  __shared__ unsigned int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(&rp.sc->arrive, 1u);
    last = prev == gridDim.x - 1 ? 1u : 0u;
    if (last) rp.sc->arrive = 0u;  // every block has arrived
  }
  __syncthreads();
  if (last && threadIdx.x < 32) {
    __threadfence();
    rp_scalar_step(d, rp, step);
  }
}

// Tile row R of the calling warp (rows past the end take no part but arrive).
__device__ __forceinline__ uint32_t rp_row() {
  return (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}

// q_R = the sum of the row's partial slots; the row's p.q; then alpha.  One
// block per tile row: kRowGroups groups of the row's 48 entries, group g
// adding slots g, g + kRowGroups, ... in order (coalesced across the entries),
// then the groups in order -- a fixed order, with enough threads in flight for
// rows of many slots.
constexpr int kRowGroups = 5;
__global__ void __launch_bounds__(kRow * kRowGroups) k_rp_rowsum(Dev d, RpData rp) {
  if (rp_done(rp)) return;
  __shared__ float part[kRowGroups][kRow];
  __shared__ double pqs[kRow];
  const uint32_t R = blockIdx.x;
  const uint32_t c = threadIdx.x % kRow, g = threadIdx.x / kRow;
  const uint32_t m0 = d.tr_list_off[R], m1 = d.tr_list_off[R + 1];
  float acc = 0.0f;
  for (uint32_t m = m0 + g; m < m1; m += kRowGroups) acc += d.partial[(size_t)m * kRow + c];
  part[g][c] = acc;
  __syncthreads();
  if (threadIdx.x < (uint32_t)kRow) {
    float q = 0.0f;
#pragma unroll
    for (int k = 0; k < kRowGroups; ++k) q += part[k][c];
    const size_t base = (size_t)R * kRow;
    d.q[base + c] = q;
    pqs[c] = (double)d.p[base + c] * (double)q;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double pq = 0.0;
    for (int e = 0; e < kRow; ++e) pq += pqs[e];
    rp.dots[R] = pq;
    __threadfence();
  }
  rp_arrive(d, rp, kRpAlpha);
}

// x += alpha p, r -= alpha q; z = the 6x6 block-Jacobi inverse times r for
// the row's nodes (runs overwrite theirs next); the rows' |r|^2; then the
// stopping rule.
__global__ void k_rp_update_xr(Dev d, RpData rp) {
  if (rp_done(rp)) return;
  const uint32_t lane = threadIdx.x & 31u, R = rp_row();
  if (R < d.num_tile_rows) {
    const size_t base = (size_t)R * kRow;
    const float af = (float)rp.sc->alpha;
    double rr = 0.0;
    for (uint32_t e = lane; e < (uint32_t)kRow; e += 32) {
      d.x[base + e] += af * d.p[base + e];
      const float rv = d.r[base + e] - af * d.q[base + e];
      d.r[base + e] = rv;
      rr += (double)rv * (double)rv;
    }
    __syncwarp();  // the row's new r is visible to the whole warp
    for (uint32_t e = lane; e < (uint32_t)kRow; e += 32) {
      const size_t node = (base + e) / 6, a = (base + e) % 6;
      const float* m = d.minv + 36 * node + a * 6;
      float z = 0.0f;
#pragma unroll
      for (int b = 0; b < 6; ++b) z += m[b] * d.r[6 * node + b];
      d.z[base + e] = z;
    }
    rr = warp_sum_d(rr);
    if (lane == 0) {
      rp.dots[2 * (size_t)d.num_tile_rows + R] = rr;
      __threadfence();
    }
  }
  rp_arrive(d, rp, kRpCheck);
}

// z = the 6x6 block-Jacobi inverse times r, every node (the initial z).
__global__ void k_rp_jacobi(Dev d, RpData rp) {
  if (rp_done(rp)) return;
  const size_t n = (size_t)d.num_var_cams * 6;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t node = i / 6, a = i % 6;
    const float* m = d.minv + 36 * node + a * 6;
    float z = 0.0f;
#pragma unroll
    for (int b = 0; b < 6; ++b) z += m[b] * d.r[6 * node + b];
    d.z[i] = z;
  }
}

constexpr int kClusterThreads = 1024;

// One block per run: z_run = inverse (column-major, FP32) times r_run, the
// run's residual staged in shared memory.  A run of at most 512 rows splits
// each row's sum over `parts` threads (contiguous column ranges, so reads
// stay coalesced across the rows) and adds the parts in order.
__global__ void __launch_bounds__(kClusterThreads) k_rp_cluster(Dev d, RpData rp) {
  if (rp_done(rp)) return;
  extern __shared__ float seg[];  // [rows] r, then [parts x rows] partial sums
  for (uint32_t c = blockIdx.x; c < rp.num_clusters; c += gridDim.x) {
    const uint32_t rows = 6u * rp.cl_size[c];
    const uint32_t parts = rows <= 512u ? min(8u, blockDim.x / rows) : 1u;
    const size_t base = 6 * (size_t)rp.cl_first[c];
    const float* mat = rp.cl_mat + rp.cl_off[c];
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < rows; i += blockDim.x) seg[i] = d.r[base + i];
    __syncthreads();
    if (parts > 1) {
      float* part = seg + rows;
      if (threadIdx.x < parts * rows) {
        const uint32_t row = threadIdx.x % rows, pi = threadIdx.x / rows;
        const uint32_t k0 = rows * pi / parts, k1 = rows * (pi + 1) / parts;
        float acc = 0.0f;
        for (uint32_t k = k0; k < k1; ++k) acc += mat[(size_t)k * rows + row] * seg[k];
        part[pi * rows + row] = acc;
      }
      __syncthreads();
      for (uint32_t row = threadIdx.x; row < rows; row += blockDim.x) {
        float z = 0.0f;
        for (uint32_t pi = 0; pi < parts; ++pi) z += part[pi * rows + row];
        d.z[base + row] = z;
      }
    } else {
      for (uint32_t row = threadIdx.x; row < rows; row += blockDim.x) {
        float acc = 0.0f;
        for (uint32_t k = 0; k < rows; ++k) acc += mat[(size_t)k * rows + row] * seg[k];
        d.z[base + row] = acc;
      }
    }
  }
}

// rc = P^T r: per aggregate and component, the sum over its nodes in order.
__global__ void k_rp_restrict(Dev d, RpData rp) {
  if (rp_done(rp)) return;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 6u * rp.coarse_m) return;
  const uint32_t g = j / 6u, k = j % 6u;
  const uint32_t end = min((g + 1u) * rp.coarse_group, rp.coarse_nodes);
  float acc = 0.0f;
  for (uint32_t i = g * rp.coarse_group; i < end; ++i) acc += d.r[6 * (size_t)i + k];
  rp.rc[j] = acc;
}

// yc = (P^T S P)^-1 rc (row-major), one block per row in a fixed-order
// block sum.
__global__ void __launch_bounds__(256) k_rp_coarse_apply(Dev d, RpData rp) {
  if (rp_done(rp)) return;
  __shared__ float red[256];
  const uint32_t m = 6u * rp.coarse_m;
  for (uint32_t t = blockIdx.x; t < m; t += gridDim.x) {
    float acc = 0.0f;
    for (uint32_t c = threadIdx.x; c < m; c += blockDim.x)
      acc += rp.coarse_inv[(size_t)t * m + c] * rp.rc[c];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) rp.yc[t] = red[0];
    __syncthreads();
  }
}

// z += P yc over the aggregated nodes; the rows' r.z; then beta (or, for
// the initial z, |b| and the first r.z).
__global__ void k_rp_prolong_rz(Dev d, RpData rp, int step) {
  if (rp_done(rp)) return;
  const uint32_t lane = threadIdx.x & 31u, R = rp_row();
  if (R < d.num_tile_rows) {
    const size_t base = (size_t)R * kRow;
    double rz = 0.0;
    for (uint32_t e = lane; e < (uint32_t)kRow; e += 32) {
      const size_t i = base + e;
      float z = d.z[i];
      const size_t node = i / 6;
      if (rp.coarse_m && node < rp.coarse_nodes) {
        z += rp.yc[6 * (node / rp.coarse_group) + i % 6];
        d.z[i] = z;
      }
      rz += (double)d.r[i] * (double)z;
    }
    rz = warp_sum_d(rz);
    if (lane == 0) {
      rp.dots[(size_t)d.num_tile_rows + R] = rz;
      __threadfence();
    }
  }
  rp_arrive(d, rp, step);
}

// p = z (first) or z + beta p.
__global__ void k_rp_update_p(Dev d, RpData rp, int first) {
  if (rp_done(rp)) return;
  const size_t n = (size_t)d.num_var_cams * 6;
  const float bf = first ? 0.0f : (float)rp.sc->beta;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    d.p[i] = first ? d.z[i] : d.z[i] + bf * d.p[i];
}

// ---------------------------------------------------------------- elimination
// The pair index of a structure: one warp per node s walks the node's blocks
// x in point order, the lanes over the later blocks y of x's point (nodes
// ascend within a point, so these are its partners t > s); each pair (x, y)
// belongs to edge (s, t), found by binary search in s's edges.  Counting
// (atomics: the totals do not depend on order), then writing at the edge's
// cursor: the partners of one x are distinct edges, and only s's warp
// touches s's edges, so each edge's pairs land in point order with no race.
template <bool WRITE>
__global__ void __launch_bounds__(256) k_el_index(ElimDev E) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t nw = gridDim.x * blockDim.x / 32u;
  for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) / 32u; s < E.n; s += nw) {
    const uint32_t e0 = E.row_off[s], e1 = E.row_off[s + 1];
    for (uint32_t q = E.slot_off[s]; q < E.slot_off[s + 1]; ++q) {
      const uint32_t x = E.slot_obs[q];
      const uint32_t y1 = E.point_off[E.obs_point[x] + 1];
      for (uint32_t y = x + 1 + lane; y < y1; y += 32) {
        const uint32_t t = E.point_nodes[y];
        uint32_t lo = e0, hi = e1;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) / 2;
          if (E.edge_t[mid] < t) lo = mid + 1;
          else hi = mid;
        }
        if (lo == e1 || E.edge_t[lo] != t) {
          atomicOr(E.err, 1u);
          continue;
        }
        if (WRITE) {
          const uint32_t pos = E.cursor[lo];
          E.cursor[lo] = pos + 1;
          E.pairs_out[pos] = make_uint2(x, y);
        } else {
          atomicAdd(E.cursor + lo, 1u);
        }
      }
      __syncwarp();  // this x's cursor updates before the next x's reads
    }
  }
}

// Per camera-point block o of point p: an FP32 copy of hcp and sk = hcp V_p^-1
// (formed in FP64; zero for a point left out, whose pairs then add zero).
// One thread per entry q = 6 i + r of the 6x3 outputs, so that consecutive
// threads read and write consecutive addresses (the three hcp entries an
// output needs come from the same 144-byte block, through L1).  The FP32
// copies are kElRec floats apart (80 bytes: five 16-byte loads a block).
__global__ void k_el_prepare(ElimDev E) {
  const uint64_t n = 18 * E.num_obs;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t o = j / 18;
    const int q = (int)(j - 18 * o), i = q / 6, r = q - 6 * i;
    const uint32_t p = E.obs_point[o];
    const double* h = E.hcp64 + 18 * o;
    const double* v = E.vinv64 + 9 * (size_t)p;
    const bool used = !E.used || E.used[p];
    const double sk = h[r] * v[3 * i] + h[6 + r] * v[3 * i + 1] + h[12 + r] * v[3 * i + 2];
    E.sk32[kElRec * o + q] = used ? (float)sk : 0.0f;
    E.hcp32[kElRec * o + q] = (float)h[q];
  }
}

// One warp per edge (s, t), lane l taking the edge's pairs l, l + 32, ...
// (ascending point order): each pair's 6x3 blocks hcp_t and sk_s arrive as
// five 16-byte loads each, their product hcp_t sk_s^T in FP32 is added to the
// lane's FP64 6x6 accumulator, and the lanes' accumulators are summed by a
// butterfly (a fixed order: the blocks do not depend on scheduling); then
// block = extra - sum, column-major (row r of t, column c of s).
__global__ void __launch_bounds__(128) k_el_blocks(ElimDev E) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t nw = (uint64_t)gridDim.x * blockDim.x / 32u;
  for (uint64_t e = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32u; e < E.num_edges;
       e += nw) {
    const uint32_t a = E.pair_off[e], b = E.pair_off[e + 1];
    double acc[36];
#pragma unroll
    for (int q = 0; q < 36; ++q) acc[q] = 0.0;
#pragma unroll 2
    for (uint32_t i = a + lane; i < b; i += 32) {
      const uint2 pr = __ldg(E.pairs + i);
      const float4* ht4 = reinterpret_cast<const float4*>(E.hcp32 + kElRec * (size_t)pr.y);
      const float4* ss4 = reinterpret_cast<const float4*>(E.sk32 + kElRec * (size_t)pr.x);
      float h[kElRec], g[kElRec];  // entries 18 and 19 are padding
#pragma unroll
      for (int k = 0; k < kElRec / 4; ++k) {
        const float4 u = __ldg(ht4 + k), v = __ldg(ss4 + k);
        h[4 * k] = u.x;
        h[4 * k + 1] = u.y;
        h[4 * k + 2] = u.z;
        h[4 * k + 3] = u.w;
        g[4 * k] = v.x;
        g[4 * k + 1] = v.y;
        g[4 * k + 2] = v.z;
        g[4 * k + 3] = v.w;
      }
      // h[6 i + r] = hcp_t[r][i], g[6 i + c] = sk_s[c][i].
#pragma unroll
      for (int c = 0; c < 6; ++c)
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          float v = h[r] * g[c];
          v = fmaf(h[6 + r], g[6 + c], v);
          v = fmaf(h[12 + r], g[12 + c], v);
          acc[6 * c + r] += (double)v;
        }
    }
    // Butterfly over the lanes: every lane ends with the same 36 sums.
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int q = 0; q < 36; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    const int x = E.extra_of ? E.extra_of[e] : -1;
    double* out = E.blocks + 36 * e;
    // Lane l writes entry l and (lanes 0-3) entry 32 + l.
    double mine = acc[0], mine2 = acc[32];
#pragma unroll
    for (int q = 1; q < 32; ++q)
      if ((int)lane == q) mine = acc[q];
#pragma unroll
    for (int q = 33; q < 36; ++q)
      if ((int)lane == q - 32) mine2 = acc[q];
    out[lane] = (x >= 0 ? E.extra64[36 * (size_t)x + lane] : 0.0) - mine;
    if (lane < 4u) out[32 + lane] = (x >= 0 ? E.extra64[36 * (size_t)x + 32 + lane] : 0.0) - mine2;
  }
}

// The blocks of the run edges, copied out.
__global__ void k_el_gather(ElimDev E) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 36 * E.num_run;
       i += (uint64_t)gridDim.x * blockDim.x)
    E.run_out[i] = E.blocks[36 * (size_t)E.run_edges[i / 36] + i % 36];
}

// coarse_out[g m + h] (g <= h): the sum of the blocks of edges (a, b), a in
// aggregate g, b in aggregate h, both below coarse_nodes, in node then edge
// order.  One warp per aggregate pair (g, h), g <= h, lanes over the 36
// entries.
__global__ void __launch_bounds__(256) k_el_coarse(ElimDev E) {
  const uint32_t m = E.coarse_m, grp = E.coarse_group;
  const uint32_t lane = threadIdx.x & 31u;
  const bool two = lane < 4u;
  const uint64_t npairs = (uint64_t)m * m;
  const uint64_t nw = (uint64_t)gridDim.x * blockDim.x / 32u;
  for (uint64_t gh = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32u; gh < npairs;
       gh += nw) {
    const uint32_t g = (uint32_t)(gh / m), h = (uint32_t)(gh % m);
    if (h < g) continue;
    const uint32_t a1 = min((g + 1) * grp, E.coarse_nodes);
    const uint32_t t0 = h * grp, t1 = min((h + 1) * grp, E.coarse_nodes);
    double acc0 = 0.0, acc1 = 0.0;
    for (uint32_t a = g * grp; a < a1; ++a) {
      uint32_t lo = E.row_off[a], hi = E.row_off[a + 1];
      const uint32_t end = hi;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (E.edge_t[mid] < t0) lo = mid + 1;
        else hi = mid;
      }
      for (uint32_t e = lo; e < end && E.edge_t[e] < t1; ++e) {
        acc0 += E.blocks[36 * (size_t)e + lane];
        if (two) acc1 += E.blocks[36 * (size_t)e + 32 + lane];
      }
    }
    double* out = E.coarse_out + 36 * gh;
    out[lane] = acc0;
    if (two) out[32 + lane] = acc1;
  }
}

int rows_grid(const Dev& d) { return (int)((d.num_tile_rows + 7) / 8); }
int flat_grid(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

// z = M r beyond block-Jacobi: the runs, then the coarse level (restrict and
// apply; its prolongation is in k_rp_prolong_rz).
void precondition_rest(const Dev& d, const RpData& rp, cudaStream_t s) {
  if (rp.num_clusters)
    k_rp_cluster<<<std::min<uint32_t>(rp.num_clusters, 148 * 2), kClusterThreads,
                   (rp.max_cluster_rows + kClusterThreads) * sizeof(float), s>>>(d, rp);
  if (rp.coarse_m) {
    k_rp_restrict<<<(6 * rp.coarse_m + 255) / 256, 256, 0, s>>>(d, rp);
    k_rp_coarse_apply<<<std::min<uint32_t>(6 * rp.coarse_m, 148 * 8), 256, 0, s>>>(d, rp);
  }
}

}  // namespace

cudaError_t launch_rp_init(const Dev& d, const RpData& rp, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(k_rp_matvec, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kMatvecSmem);
  if (e != cudaSuccess) return e;
  k_rp_init_xr<<<rows_grid(d), 256, 0, s>>>(d, rp);
  k_rp_jacobi<<<flat_grid((size_t)d.num_var_cams * 6), 256, 0, s>>>(d, rp);
  precondition_rest(d, rp, s);
  k_rp_prolong_rz<<<rows_grid(d), 256, 0, s>>>(d, rp, kRpInit);
  k_rp_update_p<<<flat_grid((size_t)d.num_var_cams * 6), 256, 0, s>>>(d, rp, 1);
  return cudaGetLastError();
}

// One iteration: the product, q and alpha, the x and r update with the
// block-Jacobi z and the stopping rule, the runs and the coarse level, r.z
// and beta, the p update -- six to eight launches.
cudaError_t launch_rp_iteration(const Dev& d, const RpData& rp, cudaStream_t s) {
  // Three blocks per SM (their rings take 3 x 72 KB of shared memory).
  const int tiles_grid =
      (int)std::min<uint32_t>((d.num_tiles + kMatvecWarps - 1) / kMatvecWarps, 148 * 3);
  k_rp_matvec<<<std::max(1, tiles_grid), kMatvecWarps * 32, kMatvecSmem, s>>>(d, rp);
  k_rp_rowsum<<<d.num_tile_rows, kRow * kRowGroups, 0, s>>>(d, rp);
  k_rp_update_xr<<<rows_grid(d), 256, 0, s>>>(d, rp);
  precondition_rest(d, rp, s);
  k_rp_prolong_rz<<<rows_grid(d), 256, 0, s>>>(d, rp, kRpBeta);
  k_rp_update_p<<<flat_grid((size_t)d.num_var_cams * 6), 256, 0, s>>>(d, rp, 0);
  return cudaGetLastError();
}

cudaError_t launch_el_index(const ElimDev& e, bool write, cudaStream_t s) {
  const int g = (int)std::min<uint32_t>((e.n + 7) / 8, 148 * 16);
  if (write) k_el_index<true><<<std::max(1, g), 256, 0, s>>>(e);
  else k_el_index<false><<<std::max(1, g), 256, 0, s>>>(e);
  return cudaGetLastError();
}

cudaError_t launch_el_prepare(const ElimDev& e, cudaStream_t s) {
  if (e.num_obs) k_el_prepare<<<flat_grid(18 * e.num_obs), 256, 0, s>>>(e);
  return cudaGetLastError();
}

cudaError_t launch_el_blocks(const ElimDev& e, cudaStream_t s) {
  if (e.num_edges)  // four warps a block: three blocks per SM at the kernel's registers
    k_el_blocks<<<(int)std::min<uint64_t>((e.num_edges + 3) / 4, 148 * 96), 128, 0, s>>>(e);
  return cudaGetLastError();
}

cudaError_t launch_el_outputs(const ElimDev& e, cudaStream_t s) {
  if (e.num_run) k_el_gather<<<flat_grid(36 * e.num_run), 256, 0, s>>>(e);
  if (e.coarse_m)
    k_el_coarse<<<(int)std::min<uint64_t>(((uint64_t)e.coarse_m * e.coarse_m + 7) / 8, 148 * 16),
                  256, 0, s>>>(e);
  return cudaGetLastError();
}

}  // namespace vlba
