// vlba_noalloc.cu -- robust cost of a device-resident problem without any
// device allocation (visloc_ba_cuda_cost_noalloc).
//
// Some callers cannot allocate device memory at the point where they need a
// cost: a tracking thread with a per-frame deadline, where cudaMalloc and
// cudaFree may synchronise the whole device and stall every stream on it; or
// a host process whose device memory is handed out by another allocator that
// owns the whole budget (a framework's caching allocator, a fixed arena).
// Their problem arrays already live in device memory.  This entry point
// evaluates the same FP64 robust cost and non-projectable count as
// visloc_ba_cuda_cost on those arrays, in one kernel on the caller's stream,
// using a fixed scratch array that is part of the loaded module instead of
// allocated memory.
//
// Scratch: kScratchBytes (1 MiB + 256 B) in g_noalloc_scratch, present on
// every GPU that loads this library until the process exits.  It holds a
// ticket word and one partial per chunk of 256 observations, which bounds a
// call to kMaxChunks * 256 = 16,777,216 observations.  Every call on a device
// shares that device's array and finds the previous call's contents in it:
// two calls whose kernels overlap in time on the same GPU (on two streams, or
// from two threads) race on it and return wrong sums, so serialise them.
//
// Device pointers: host code never passes g_noalloc_scratch itself to a
// kernel -- in host code the name is a host-side stand-in, not a device
// address.  The device address is looked up with cudaGetSymbolAddress
// (scratch_address below) on the first call made with that device current,
// and looked up again when the device's current context is no longer the
// one the address was taken in (after cudaDeviceReset the module is loaded
// anew and the array may move); make such a call before any stream capture.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "vlba_device_math.cuh"
#include "vlba_plan.h"

namespace vlba {
namespace {

constexpr uint32_t kChunk = 256;                  // observations per partial
constexpr uint32_t kMaxChunks = 65536;
constexpr uint64_t kMaxObservations = (uint64_t)kMaxChunks * kChunk;
constexpr size_t kHeaderBytes = 256;              // ticket word, padded
constexpr size_t kScratchBytes = kHeaderBytes + (size_t)kMaxChunks * 16;
constexpr int kMaxCameras = 16;
constexpr int kMaxDevices = 64;

// Layout: [0, 4) ticket (must be zero when a call's kernel starts; every call
// clears it on its stream first), then per chunk {double cost, uint32
// non-projectable, uint32 invalid} at kHeaderBytes.  Chunk partials are
// written before they are read in every call, so they need no clearing.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct ChunkPartial {
  double cost;
  uint32_t nonproj;
  uint32_t invalid;
};
static_assert(sizeof(ChunkPartial) == 16, "chunk partial layout");

struct NoallocArgs {
  uint64_t num_poses, num_landmarks, num_obs;
  const double* pose_q;
  const double* pose_t;
  const double* landmarks;
  const uint32_t* obs_pose;
  const uint32_t* obs_landmark;
  const double2* obs_xy;
  const uint32_t* obs_camera;  // null: cameras[0] for every observation
  const double* obs_weight;    // null: every weight 1
  const uint8_t* obs_kind;     // null: every observation monocular or rig
  const double* obs_stereo;
  const uint32_t* obs_right_camera;
  double stereo_baseline;
  uint32_t stereo_camera_ok;   // cameras[0] is PINHOLE or SIMPLE_PINHOLE
  uint32_t num_cameras;
  uint32_t robust_kernel;
  double robust_parameter;
  uint32_t num_chunks;
  double* out_cost;
  unsigned long long* out_counts;  // [0] non-projectable, [1] invalid indices
  DevCamera cameras[kMaxCameras];
};

// Fixed-shape tree sum over 256 threads (the same order on every call).
template <typename T>
__device__ __forceinline__ T tree_sum256(T v, T* red) {
  red[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  const T r = red[0];
  __syncthreads();
  return r;
}

// One thread per observation, 256 per chunk; each chunk's sums go to its
// partial slot, and the block that takes the last ticket adds the partials
// in chunk order.  The order of every sum is fixed by the observation order,
// not by the grid, so repeated calls give identical results.
__global__ void __launch_bounds__(256) k_cost_noalloc(const NoallocArgs a, unsigned char* scratch) {
  __shared__ double red_d[256];
  __shared__ unsigned long long red_u[256];
  __shared__ int s_last;
  unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch);
  ChunkPartial* part = reinterpret_cast<ChunkPartial*>(scratch + kHeaderBytes);
  for (uint32_t ch = blockIdx.x; ch < a.num_chunks; ch += gridDim.x) {
    const uint64_t o = (uint64_t)ch * kChunk + threadIdx.x;
    double cost = 0.0;
    unsigned long long bad = 0, invalid = 0;
    if (o < a.num_obs) {
      const uint32_t ip = a.obs_pose[o], il = a.obs_landmark[o];
      const uint32_t kind = a.obs_kind ? a.obs_kind[o] : kObsMono;
      const uint32_t ic = (kind == kObsMono && a.obs_camera) ? a.obs_camera[o] : 0u;
      const uint32_t rc = (kind == kObsGeneralStereo && a.obs_right_camera) ? a.obs_right_camera[o] : 0u;
      const double w = a.obs_weight ? a.obs_weight[o] : 1.0;
      const bool stereo_ok =
          kind == kObsMono ||
          (kind <= kObsGeneralStereo && a.stereo_camera_ok && rc < a.num_cameras &&
           (kind != kObsGeneralStereo || a.obs_right_camera) &&
           (kind != kObsStereo || (isfinite(a.stereo_baseline) && a.stereo_baseline > 0.0)));
      if (ip >= a.num_poses || il >= a.num_landmarks || ic >= a.num_cameras || !isfinite(w) ||
          w < 0.0 || !stereo_ok) {
        invalid = 1;
      } else {
        double q[4], rt[12], X[3], xs[3], pred[2];
#pragma unroll
        for (int c = 0; c < 4; ++c) q[c] = a.pose_q[4 * (size_t)ip + c];
        quat_to_matrix(q, rt);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          rt[9 + c] = a.pose_t[3 * (size_t)ip + c];
          X[c] = a.landmarks[3 * (size_t)il + c];
        }
        const DevCamera& cam = a.cameras[ic];
        to_sensor(rt, cam, X, xs);
        if (kind != kObsMono) {
          const double2 st = kind == kObsStereo
                                 ? make_double2(a.obs_stereo[2 * o], a.stereo_baseline)
                                 : make_double2(a.obs_stereo[2 * o], a.obs_stereo[2 * o + 1]);
          double r[4];
          const int m = stereo_rows(kind, cam, a.cameras[rc], a.obs_xy[o], st, xs, nullptr, r,
                                    nullptr);
          if (!m) {
            bad = 1;
          } else {
            double ss = 0.0;
            for (int i = 0; i < m; ++i) ss += r[i] * r[i];
            cost = robust_cost(a.robust_kernel, a.robust_parameter, ss);
            if (a.obs_weight) cost *= w;
          }
        } else if (!(xs[2] > 0.0) || !camera_project(cam, xs, pred)) {
          bad = 1;
        } else {
          const double2 xy = a.obs_xy[o];
          const double rx = pred[0] - xy.x, ry = pred[1] - xy.y;
          cost = robust_cost(a.robust_kernel, a.robust_parameter, rx * rx + ry * ry);
          if (a.obs_weight) cost *= w;
        }
      }
    }
    const double tc = tree_sum256<double>(cost, red_d);
    const unsigned long long tb = tree_sum256<unsigned long long>(bad | (invalid << 32), red_u);
    if (threadIdx.x == 0) part[ch] = ChunkPartial{tc, (uint32_t)tb, (uint32_t)(tb >> 32)};
  }
  // Last block in: every other block's partials are visible after its
  // release (threadfence before the ticket) and our acquire fence.
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    s_last = (t == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double cost = 0.0;
  unsigned long long bad = 0, invalid = 0;
  for (uint32_t ch = threadIdx.x; ch < a.num_chunks; ch += blockDim.x) {
    const volatile ChunkPartial* pc = part + ch;
    cost += pc->cost;
    bad += pc->nonproj;
    invalid += pc->invalid;
  }
  const double tc = tree_sum256<double>(cost, red_d);
  const unsigned long long tb = tree_sum256<unsigned long long>(bad, red_u);
  const unsigned long long ti = tree_sum256<unsigned long long>(invalid, red_u);
  if (threadIdx.x == 0) {
    *a.out_cost = tc;
    a.out_counts[0] = tb;
    a.out_counts[1] = ti;
    *ticket = 0u;  // the next call clears it on its stream too
  }
}

// Process-unique id of the calling thread's current context (cuCtxGetId),
// or 0 when there is none or the driver cannot tell.  The driver functions
// come through the runtime's entry-point query, so the library needs no
// link-time dependency on libcuda.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_noalloc_scratch on the current device: looked up on
// the first call with the device current and again whenever the current
// context differs from the one it was taken in (a cudaDeviceReset in
// between, or another context of the device made current).  nullptr and
// `err` set on failure.
unsigned char* scratch_address(int device, cudaError_t* err) {
  static std::mutex mu;
  static unsigned char* addr[kMaxDevices] = {};
  static unsigned long long context_of[kMaxDevices] = {};
  std::lock_guard<std::mutex> lock(mu);
  const unsigned long long ctx = current_context_id();
  if (!addr[device] || ctx == 0 || ctx != context_of[device]) {
    unsigned char* ptr = nullptr;
    *err = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
    if (*err != cudaSuccess) return nullptr;
    addr[device] = ptr;
    // The lookup makes the device's primary context current if none was.
    context_of[device] = current_context_id();
  }
  *err = cudaSuccess;
  return addr[device];
}

int fail(char* msg, size_t cap, int status, const char* fmt, unsigned long long v0 = 0,
         unsigned long long v1 = 0) {
  if (msg && cap) std::snprintf(msg, cap, fmt, v0, v1);
  return status;
}

}  // namespace
}  // namespace vlba

extern "C" {

int visloc_ba_cuda_cost_noalloc(const vlba_problem* problem, const vlba_config* config,
                                void* stream, double* cost, uint64_t* counts, char* error,
                                size_t error_capacity) {
  using namespace vlba;
  if (error && error_capacity) error[0] = '\0';
  if (!problem || !config || !cost || !counts)
    return fail(error, error_capacity, VLBA_ERR_INVALID_ARGUMENT,
                "null problem, config or output pointer");
  const vlba_problem& p = *problem;
  if (config->robust_kernel > VLBA_KERNEL_CAUCHY)
    return fail(error, error_capacity, VLBA_ERR_INVALID_ARGUMENT, "unknown robust kernel %llu",
                config->robust_kernel);
  if (p.num_cameras == 0 || !p.cameras)
    return fail(error, error_capacity, VLBA_ERR_UNSUPPORTED_CAMERA_MODEL, "no camera");
  if (p.num_cameras > (uint32_t)kMaxCameras)
    return fail(error, error_capacity, VLBA_ERR_INVALID_ARGUMENT,
                "%llu cameras: this entry point takes at most %llu", p.num_cameras, kMaxCameras);
  if (p.num_poses == 0) return fail(error, error_capacity, VLBA_ERR_NO_POSES, "no poses");
  if (p.num_observations == 0)
    return fail(error, error_capacity, VLBA_ERR_NO_OBSERVATIONS, "no observations");
  if (p.num_landmarks == 0) return fail(error, error_capacity, VLBA_ERR_NO_LANDMARKS, "no landmarks");
  if (p.num_observations > kMaxObservations)
    return fail(error, error_capacity, VLBA_ERR_INVALID_ARGUMENT,
                "%llu observations: the fixed scratch of this entry point holds at most %llu",
                p.num_observations, kMaxObservations);
  if (!p.pose_q || !p.pose_t || !p.landmarks || !p.obs_pose || !p.obs_landmark || !p.obs_xy)
    return fail(error, error_capacity, VLBA_ERR_INVALID_ARGUMENT, "null problem array");
  if (p.obs_kind && !p.obs_stereo)
    return fail(error, error_capacity, VLBA_ERR_INVALID_ARGUMENT, "obs_kind without obs_stereo");
  NoallocArgs a;
  std::memset(&a, 0, sizeof a);
  for (uint32_t c = 0; c < p.num_cameras; ++c) {
    const uint32_t m = p.cameras[c].model;
    if (m > VLBA_CAMERA_OPENCV)
      return fail(error, error_capacity, VLBA_DECLINED, "camera %llu: model outside the radial "
                  "pinhole family", c);
    if (!resolve_camera(p.cameras[c], &a.cameras[c]))
      return fail(error, error_capacity,
                  m == VLBA_CAMERA_OPENCV ? VLBA_DECLINED : VLBA_ERR_UNSUPPORTED_CAMERA_MODEL,
                  "camera %llu: unsupported parameters", c);
    if (!p.obs_camera) a.cameras[c].rig = 0;  // monocular: the pose is the camera
  }
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess || device < 0 || device >= kMaxDevices)
    return fail(error, error_capacity, VLBA_ERR_CUDA, "no current CUDA device");
  unsigned char* scratch = scratch_address(device, &e);
  if (!scratch) {
    if (error && error_capacity)
      std::snprintf(error, error_capacity, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    return VLBA_ERR_CUDA;
  }
  a.num_poses = p.num_poses;
  a.num_landmarks = p.num_landmarks;
  a.num_obs = p.num_observations;
  a.pose_q = p.pose_q;
  a.pose_t = p.pose_t;
  a.landmarks = p.landmarks;
  a.obs_pose = p.obs_pose;
  a.obs_landmark = p.obs_landmark;
  a.obs_xy = reinterpret_cast<const double2*>(p.obs_xy);
  a.obs_camera = p.obs_camera;
  a.obs_weight = p.obs_weight;
  a.obs_kind = p.obs_kind;
  a.obs_stereo = p.obs_stereo;
  a.obs_right_camera = p.obs_right_camera;
  a.stereo_baseline = p.stereo_baseline;
  a.stereo_camera_ok = (p.cameras[0].model == VLBA_CAMERA_PINHOLE ||
                        p.cameras[0].model == VLBA_CAMERA_SIMPLE_PINHOLE) ? 1u : 0u;
  a.num_cameras = p.num_cameras;
  a.robust_kernel = config->robust_kernel;
  a.robust_parameter = config->robust_parameter;
  a.num_chunks = (uint32_t)((p.num_observations + kChunk - 1) / kChunk);
  a.out_cost = cost;
  a.out_counts = reinterpret_cast<unsigned long long*>(counts);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const uint32_t grid = a.num_chunks < (uint32_t)(8 * sms) ? a.num_chunks : (uint32_t)(8 * sms);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s);  // the ticket starts at zero
  if (e == cudaSuccess) {
    k_cost_noalloc<<<grid, 256, 0, s>>>(a, scratch);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    if (error && error_capacity)
      std::snprintf(error, error_capacity, "cost kernel: %s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? VLBA_ERR_OUT_OF_MEMORY : VLBA_ERR_CUDA;
  }
  return VLBA_OK;
}

}  // extern "C"
