// vlba_pairs.cu -- the Schur terms of one problem's reduced system built on
// the device at upload (the largest part of the plan: one 8-byte term per
// pair of a variable point's observations by two variable cameras).
//
// The host plan (vlba_plan.cpp) lists the terms per block (camera pair
// (i, j), i > j, blocks row-major, columns ascending), each block's terms in
// ascending point order; the off-diagonal assembly sums them in that order,
// so the order fixes every block's rounding.  Here:
//
//   k_rows_count  one block per camera row i: walks the row camera's
//                 observations (ascending point order) and, for each, the
//                 other observations of its point; counts the terms of each
//                 column j < i in shared memory, then writes the row's
//                 nonzero columns and counts in ascending column order.
//                 A point seen twice by one camera (same-camera terms) sets
//                 a flag: those plans are built on the host.
//   k_rows_pack   the rows' lists, packed by the prefix of their lengths.
//   k_rows_place  one warp per camera row: the row's observations in groups
//                 of 32 consecutive ones (32 distinct points, ascending);
//                 for each of the row's blocks (found from the column by a
//                 shared map), the lanes that have a term there take
//                 consecutive places in lane order (a shared bit mask per
//                 block and the lane's rank in it), so each block receives
//                 its terms in ascending point order -- the host's order
//                 (with each term's point beside it);
//                 the column's lowest lane then advances its cursor and
//                 clears its mask.
//                 Every place is checked against its block's range; a term
//                 outside it, or a block left short, sets the error flag
//                 and writes nothing outside the array.
//
// The host lays out the blocks, tiles and destinations from the counts
// (exactly as for terms it builds itself) between the two passes.
#include <cuda_runtime.h>

#include <cstdint>

#include "vlba_kernels.cuh"

namespace vlba {
namespace {

__global__ void __launch_bounds__(256) k_rows_count(RowsDev r) {
  extern __shared__ uint32_t cnt[];  // [nvar]
  __shared__ uint32_t s_part[256];
  for (uint32_t i = blockIdx.x; i < r.nvar; i += gridDim.x) {
    for (uint32_t j = threadIdx.x; j < r.nvar; j += blockDim.x) cnt[j] = 0u;
    __syncthreads();
    for (uint32_t q = r.cam_off[i] + threadIdx.x; q < r.cam_off[i + 1]; q += blockDim.x) {
      const uint32_t a = r.cam_obs[q];
      const uint32_t p = r.obs_point[a];
      if (!r.point_var[p]) continue;
      for (uint32_t b = r.pt_off[p]; b < r.pt_off[p + 1]; ++b) {
        if (b == a) continue;
        const uint32_t sb = r.obs_slot[b];
        if (sb == kNone) continue;
        if (sb == i) {
          atomicOr(r.flags, 1u);  // same-camera terms: the host builds this plan
        } else if (sb < i) {
          atomicAdd(&cnt[sb], 1u);
        }
      }
    }
    __syncthreads();
    // Compaction in ascending column: thread t owns columns [t c, (t+1) c).
    const uint32_t per = (i + blockDim.x - 1) / blockDim.x;
    const uint32_t j0 = min(i, threadIdx.x * per), j1 = min(i, j0 + per);
    uint32_t mine = 0;
    for (uint32_t j = j0; j < j1; ++j) mine += cnt[j] != 0u;
    s_part[threadIdx.x] = mine;
    __syncthreads();
    // Exclusive prefix over the 256 thread counts (serial in thread 0's
    // order is enough: 256 adds).
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (uint32_t t = 0; t < blockDim.x; ++t) {
        const uint32_t v = s_part[t];
        s_part[t] = run;
        run += v;
      }
      r.row_nblk[i] = run;
    }
    __syncthreads();
    uint2* out = r.tri + (size_t)i * (i - (i > 0 ? 1u : 0u)) / 2;  // row i holds <= i entries
    uint32_t k = s_part[threadIdx.x];
    for (uint32_t j = j0; j < j1; ++j)
      if (cnt[j] != 0u) out[k++] = make_uint2(j, cnt[j]);
    __syncthreads();
  }
}

// Exclusive prefix of the rows' block counts (one block): row_blk[i], and
// row_blk[nvar] the total.
__global__ void __launch_bounds__(1024) k_rows_scan(RowsDev r) {
  __shared__ uint32_t s_part[1024];
  const uint32_t per = (r.nvar + blockDim.x - 1) / blockDim.x;
  const uint32_t i0 = min(r.nvar, threadIdx.x * per), i1 = min(r.nvar, i0 + per);
  uint32_t sum = 0;
  for (uint32_t i = i0; i < i1; ++i) sum += r.row_nblk[i];
  s_part[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (uint32_t t = 0; t < blockDim.x; ++t) {
      const uint32_t v = s_part[t];
      s_part[t] = run;
      run += v;
    }
    r.row_blk[r.nvar] = run;
  }
  __syncthreads();
  uint32_t run = s_part[threadIdx.x];
  for (uint32_t i = i0; i < i1; ++i) {
    r.row_blk[i] = run;
    run += r.row_nblk[i];
  }
}

__global__ void __launch_bounds__(256) k_rows_pack(RowsDev r) {
  for (uint32_t i = blockIdx.x; i < r.nvar; i += gridDim.x) {
    const uint2* src = r.tri + (size_t)i * (i - (i > 0 ? 1u : 0u)) / 2;
    const uint32_t base = r.row_blk[i], n = r.row_nblk[i];
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
      const uint2 v = src[k];
      r.col[base + k] = v.x;
      r.count[base + k] = v.y;
    }
  }
}

// W warps per row, each taking a contiguous segment of the row's
// observation list (whole groups of 32).  Shared memory per block: a map
// from column slot to the row's block (0xFFFF: no block of this row), then
// per warp and block of the row a cursor, a limit and the lane mask of the
// current group -- sized by the longest row's block count.  A first pass
// counts each warp's terms per block; the counts, added in warp order from
// the block's start, give each warp's first place in the block, and the next
// warp's first place is its limit.  The segments are consecutive in point
// order, so each block still receives its terms in ascending point order.
constexpr uint16_t kNoBlock = 0xFFFFu;

template <int W>
__global__ void __launch_bounds__(32 * W) k_rows_place(RowsDev r, const uint32_t* blk_off,
                                                       const uint32_t* row_blk,
                                                       const uint32_t* blk_col,
                                                       uint32_t max_row_blocks, uint2* pairs,
                                                       uint32_t* pair_pt) {
  extern __shared__ uint32_t sm[];
  __shared__ int s_bad;
  uint16_t* colmap = reinterpret_cast<uint16_t*>(sm);       // [nvar]
  uint32_t* cur = sm + (r.nvar + 1) / 2;                     // [W][max_row_blocks]
  uint32_t* lim = cur + (size_t)W * max_row_blocks;          // [W][max_row_blocks]
  uint32_t* msk = lim + (size_t)W * max_row_blocks;          // [W][max_row_blocks]
  const uint32_t lane = threadIdx.x % 32, w = threadIdx.x / 32;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t* const mcur = cur + (size_t)w * max_row_blocks;
  uint32_t* const mlim = lim + (size_t)w * max_row_blocks;
  uint32_t* const mmsk = msk + (size_t)w * max_row_blocks;
  for (uint32_t j = threadIdx.x; j < r.nvar; j += 32 * W) colmap[j] = kNoBlock;
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x; i < r.nvar; i += gridDim.x) {
    const uint32_t rb0 = row_blk[i], rb1 = row_blk[i + 1];
    bool bad = rb1 - rb0 > max_row_blocks;
    const uint32_t nb = bad ? 0u : rb1 - rb0;
    for (uint32_t q = threadIdx.x; q < nb; q += 32 * W) {
      const uint32_t col = blk_col[rb0 + q];
      if (col < i) colmap[col] = (uint16_t)q;
      else bad = true;
    }
    for (uint32_t q = threadIdx.x; q < (uint32_t)W * nb; q += 32 * W) {
      const uint32_t ww = q / nb, qq = q % nb;
      cur[(size_t)ww * max_row_blocks + qq] = 0u;
      msk[(size_t)ww * max_row_blocks + qq] = 0u;
    }
    __syncthreads();
    // This warp's segment: groups [g0, g1) of the row's list.
    const uint32_t q0 = r.cam_off[i], q1 = r.cam_off[i + 1];
    const uint32_t ngroups = (q1 - q0 + 31) / 32;
    const uint32_t g0 = ngroups * w / W, g1 = ngroups * (w + 1) / W;
    // Each lane's observation and its point's range in a group.
    auto lane_obs = [&](uint32_t g, uint32_t* a, uint32_t* b0, uint32_t* b1, uint32_t* pp) {
      const uint32_t q = q0 + 32 * g + lane;
      *a = kNone;
      *b0 = *b1 = 0u;
      *pp = 0u;
      if (q < q1) {
        *a = r.cam_obs[q];
        const uint32_t p = r.obs_point[*a];
        *pp = p;
        if (r.point_var[p]) {
          *b0 = r.pt_off[p];
          *b1 = r.pt_off[p + 1];
        }
      }
    };
    // Pass 1: this warp's terms per block.
    for (uint32_t g = g0; g < g1; ++g) {
      uint32_t a, b0, b1, pp;
      lane_obs(g, &a, &b0, &b1, &pp);
      for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t sb = r.obs_slot[b];
        if (b == a || sb == kNone || sb >= i) continue;
        const uint32_t lb = colmap[sb];
        if (lb == kNoBlock) bad = true;  // a term outside the row's blocks
        else atomicAdd(&mcur[lb], 1u);
      }
    }
    __syncthreads();
    // Each warp's first place and limit per block, warps in order.
    for (uint32_t q = threadIdx.x; q < nb; q += 32 * W) {
      uint32_t run = blk_off[rb0 + q];
      for (int ww = 0; ww < W; ++ww) {
        const uint32_t c = cur[(size_t)ww * max_row_blocks + q];
        cur[(size_t)ww * max_row_blocks + q] = run;
        run += c;
        lim[(size_t)ww * max_row_blocks + q] = run;
      }
      if (run != blk_off[rb0 + q + 1]) bad = true;  // the block's size
    }
    __syncthreads();
    // Pass 2: the lanes of a block in lane order from this warp's cursor.
    for (uint32_t g = g0; g < g1; ++g) {
      uint32_t a, b0, b1, pp;
      lane_obs(g, &a, &b0, &b1, &pp);
      for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t sb = r.obs_slot[b];
        if (b == a || sb == kNone || sb >= i) continue;
        const uint32_t lb = colmap[sb];
        if (lb != kNoBlock) atomicOr(&mmsk[lb], 1u << lane);
      }
      __syncwarp();
      for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t sb = r.obs_slot[b];
        if (b == a || sb == kNone || sb >= i) continue;
        const uint32_t lb = colmap[sb];
        if (lb == kNoBlock) continue;
        const uint32_t at = mcur[lb] + __popc(mmsk[lb] & lt);
        if (at >= mlim[lb]) {
          bad = true;
        } else {
          pairs[at] = make_uint2(a, b);
          pair_pt[at] = pp;
        }
      }
      __syncwarp();
      // The block's lowest lane advances its cursor and clears its mask
      // (another lane of the block then reads the full mask or zero, and
      // does nothing either way).
      for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t sb = r.obs_slot[b];
        if (b == a || sb == kNone || sb >= i) continue;
        const uint32_t lb = colmap[sb];
        if (lb == kNoBlock) continue;
        const uint32_t m = static_cast<volatile uint32_t*>(mmsk)[lb];
        if (m != 0u && (uint32_t)(__ffs(m) - 1) == lane) {
          mcur[lb] += __popc(m);
          atomicExch(&mmsk[lb], 0u);
        }
      }
      __syncwarp();
    }
    __syncthreads();
    // Every warp's share of every block filled exactly; the map back to
    // empty.
    for (uint32_t q = threadIdx.x; q < (uint32_t)W * nb; q += 32 * W) {
      const uint32_t ww = q / nb, qq = q % nb;
      if (cur[(size_t)ww * max_row_blocks + qq] != lim[(size_t)ww * max_row_blocks + qq]) bad = true;
    }
    for (uint32_t q = threadIdx.x; q < nb; q += 32 * W) {
      const uint32_t col = blk_col[rb0 + q];
      if (col < i) colmap[col] = kNoBlock;
    }
    if (bad) s_bad = 1;
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_bad) atomicOr(r.flags, 2u);
}

}  // namespace

size_t rows_count_smem(uint32_t nvar) { return (size_t)nvar * 4; }
size_t rows_place_smem(uint32_t nvar, uint32_t max_row_blocks, int warps) {
  return (size_t)(nvar + 1) / 2 * 4 + (size_t)max_row_blocks * 12 * warps;
}

cudaError_t launch_rows_count(const RowsDev& r, cudaStream_t s) {
  const size_t sm = rows_count_smem(r.nvar);
  cudaError_t e = cudaFuncSetAttribute(k_rows_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sm);
  if (e != cudaSuccess) return e;
  const int g = (int)(r.nvar < 148u * 8u ? r.nvar : 148u * 8u);
  k_rows_count<<<g, 256, sm, s>>>(r);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_rows_scan<<<1, 1024, 0, s>>>(r);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_rows_pack<<<g, 256, 0, s>>>(r);
  return cudaGetLastError();
}

cudaError_t launch_rows_place(const RowsDev& r, const uint32_t* blk_off, const uint32_t* row_blk,
                              const uint32_t* blk_col, uint32_t max_row_blocks, uint2* pairs,
                              uint32_t* pair_pt, cudaStream_t s) {
  // Four warps per row where their state fits in shared memory, else one.
  constexpr size_t kMaxSmem = 227u * 1024u;
  const int g = (int)(r.nvar < 148u * 16u ? r.nvar : 148u * 16u);
  size_t sm = rows_place_smem(r.nvar, max_row_blocks, 4);
  cudaError_t e;
  if (sm <= kMaxSmem) {
    e = cudaFuncSetAttribute(k_rows_place<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_rows_place<4><<<g, 128, sm, s>>>(r, blk_off, row_blk, blk_col, max_row_blocks, pairs, pair_pt);
    return cudaGetLastError();
  }
  sm = rows_place_smem(r.nvar, max_row_blocks, 1);
  e = cudaFuncSetAttribute(k_rows_place<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k_rows_place<1><<<g, 32, sm, s>>>(r, blk_off, row_blk, blk_col, max_row_blocks, pairs, pair_pt);
  return cudaGetLastError();
}

}  // namespace vlba
