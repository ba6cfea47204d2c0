// vlba_plan.cpp -- see vlba_plan.h.
#include "vlba_plan.h"

#include <cuda_runtime.h>

#include <sys/mman.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <exception>
#include <stdexcept>
#include <map>
#include <mutex>
#include <thread>

namespace vlba {

namespace {
thread_local int t_pin_depth = 0;
std::mutex g_pin_mu;
std::map<uintptr_t, size_t> g_pinned;  // base -> bytes of page-locked allocations
}  // namespace

PinScope::PinScope() { ++t_pin_depth; }
PinScope::~PinScope() { --t_pin_depth; }
bool pin_requested() { return t_pin_depth > 0; }

void pin_allocation(void* p, size_t bytes) {
  if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) != cudaSuccess) {
    (void)cudaGetLastError();  // stays pageable: the upload stages it
    return;
  }
  std::lock_guard<std::mutex> lock(g_pin_mu);
  g_pinned[(uintptr_t)p] = bytes;
}

void unpin_allocation(void* p) {
  {
    std::lock_guard<std::mutex> lock(g_pin_mu);
    auto it = g_pinned.find((uintptr_t)p);
    if (it == g_pinned.end()) return;
    g_pinned.erase(it);
  }
  cudaHostUnregister(p);
  (void)cudaGetLastError();
}

bool pinned_range(const void* p, size_t bytes) {
  std::lock_guard<std::mutex> lock(g_pin_mu);
  if (g_pinned.empty()) return false;
  auto it = g_pinned.upper_bound((uintptr_t)p);
  if (it == g_pinned.begin()) return false;
  --it;
  return (uintptr_t)p + bytes <= it->first + it->second;
}

void advise_huge_pages(void* p, size_t bytes) {
  constexpr uintptr_t kHuge = 2u << 20;
  const uintptr_t a = ((uintptr_t)p + kHuge - 1) & ~(kHuge - 1);
  const uintptr_t e = ((uintptr_t)p + bytes) & ~(kHuge - 1);
  if (e > a) madvise(reinterpret_cast<void*>(a), e - a, MADV_HUGEPAGE);
}

namespace {

void quat_to_matrix(const double* q, double* m) {
  const double w = q[0], i = q[1], j = q[2], k = q[3];
  const double ww = w * w, ii = i * i, jj = j * j, kk = k * k;
  const double ij = i * j * 2.0, wk = w * k * 2.0, wj = w * j * 2.0;
  const double ik = i * k * 2.0, jk = j * k * 2.0, wi = w * i * 2.0;
  m[0] = ww + ii - jj - kk; m[1] = ij - wk;           m[2] = wj + ik;
  m[3] = wk + ij;           m[4] = ww - ii + jj - kk; m[5] = jk - wi;
  m[6] = ik - wj;           m[7] = wi + jk;           m[8] = ww - ii - jj + kk;
}

uint32_t round_up(uint32_t v, uint32_t m) { return (v + m - 1) / m * m; }

}  // namespace

bool resolve_camera(const vlba_camera& c, DevCamera* out) {
  const double* p = c.params;
  const uint32_t n = c.num_params;
  double fx, fy, cx, cy, k1 = 0.0, k2 = 0.0;
  bool has_radial = false;
  switch (c.model) {
    case VLBA_CAMERA_PINHOLE:
      if (n < 4 || n > 8) return false;
      fx = p[0]; fy = p[1]; cx = p[2]; cy = p[3];
      if (n >= 5) { has_radial = true; k1 = p[4]; k2 = n >= 6 ? p[5] : 0.0; }
      break;
    case VLBA_CAMERA_OPENCV:
      if (n < 4 || n > 8) return false;
      fx = p[0]; fy = p[1]; cx = p[2]; cy = p[3];
      if ((n >= 7 && p[6] != 0.0) || (n >= 8 && p[7] != 0.0)) return false;
      if (n >= 5) { has_radial = true; k1 = p[4]; k2 = n >= 6 ? p[5] : 0.0; }
      break;
    case VLBA_CAMERA_SIMPLE_PINHOLE:
      if (n < 3 || n > 8) return false;
      fx = fy = p[0]; cx = p[1]; cy = p[2];
      break;
    case VLBA_CAMERA_SIMPLE_RADIAL:
      if (n < 3 || n > 8) return false;
      fx = fy = p[0]; cx = p[1]; cy = p[2];
      if (n >= 4) { has_radial = true; k1 = p[3]; }
      break;
    case VLBA_CAMERA_RADIAL:
      if (n < 3 || n > 8) return false;
      fx = fy = p[0]; cx = p[1]; cy = p[2];
      if (n >= 4) { has_radial = true; k1 = p[3]; k2 = n >= 5 ? p[4] : 0.0; }
      break;
    default:
      return false;
  }
  std::memset(out, 0, sizeof *out);
  out->fx = fx; out->fy = fy; out->cx = cx; out->cy = cy;
  out->k1 = k1; out->k2 = k2;
  out->radial = (has_radial && (k1 != 0.0 || k2 != 0.0)) ? 1 : 0;
  quat_to_matrix(c.sensor_from_rig_q, out->R);
  for (int a = 0; a < 3; ++a) out->t[a] = c.sensor_from_rig_t[a];
  const bool identity = c.sensor_from_rig_q[0] == 1.0 && c.sensor_from_rig_q[1] == 0.0 &&
                        c.sensor_from_rig_q[2] == 0.0 && c.sensor_from_rig_q[3] == 0.0 &&
                        c.sensor_from_rig_t[0] == 0.0 && c.sensor_from_rig_t[1] == 0.0 &&
                        c.sensor_from_rig_t[2] == 0.0;
  out->rig = identity ? 0 : 1;
  return true;
}

LmParams make_params(const vlba_config* cfg) {
  LmParams lp;
  std::memset(&lp, 0, sizeof lp);
  lp.initial_lambda = cfg->initial_lambda;
  lp.lambda_increase_factor = cfg->lambda_increase_factor;
  lp.lambda_decrease_factor = cfg->lambda_decrease_factor;
  lp.max_lambda = cfg->max_lambda;
  lp.min_lambda = cfg->min_lambda;
  lp.step_tolerance = cfg->step_tolerance;
  lp.cost_tolerance = cfg->cost_tolerance;
  lp.relative_cost_tolerance = cfg->relative_cost_tolerance;
  lp.robust_parameter = cfg->robust_parameter;
  lp.pcg_relative_tolerance = cfg->pcg_relative_tolerance;
  lp.has_initial_lambda = cfg->has_initial_lambda ? 1u : 0u;
  lp.has_relative_cost_tolerance = cfg->has_relative_cost_tolerance ? 1u : 0u;
  lp.robust_kernel = cfg->robust_kernel;
  lp.max_iterations = cfg->max_iterations;
  lp.max_pcg_iterations = cfg->max_pcg_iterations;
  return lp;
}

namespace {

// Lowest index in [0, n) at which pred fails (n if none), on the host's
// threads for large n: each thread scans its own range in order and stops at
// its first failure, and the lowest of those is the serial scan's answer.
template <typename F>
uint64_t first_failing(uint64_t n, F&& pred) {
  const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const uint32_t T = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(hw, n >> 18));
  std::vector<uint64_t> first(T, n);
  auto body = [&](uint32_t t) {
    for (uint64_t i = n * t / T, e = n * (t + 1) / T; i < e; ++i)
      if (!pred(i)) {
        first[t] = i;
        return;
      }
  };
  std::vector<std::thread> pool;
  for (uint32_t t = 1; t < T; ++t) pool.emplace_back(body, t);
  body(0);
  for (auto& th : pool) th.join();
  return *std::min_element(first.begin(), first.end());
}

}  // namespace

Validation validate_problem(const vlba_problem* p, const vlba_config* cfg) {
  Validation v;
  if (!p || !cfg) { v.status = VLBA_ERR_INVALID_ARGUMENT; return v; }
  // Joint intrinsics refinement is the CPU solver's (optimize.rs:9-27):
  // declined before anything else, as GpuBundleAdjuster::check does first
  // (crates/ba-gpu/src/solver.rs:214-216).
  if (cfg->refine_intrinsics || cfg->refine_distortion || cfg->refine_tangential_distortion ||
      cfg->shared_focal) {
    v.status = VLBA_DECLINED;
    return v;
  }
  if (cfg->robust_kernel > VLBA_KERNEL_CAUCHY) { v.status = VLBA_ERR_INVALID_ARGUMENT; return v; }
  if (p->num_poses >= kNone || p->num_landmarks >= kNone || p->num_observations >= kNone) {
    v.status = VLBA_ERR_INVALID_ARGUMENT;
    return v;
  }
  if ((p->num_poses && (!p->pose_q || !p->pose_t)) || (p->num_landmarks && !p->landmarks) ||
      (p->num_observations && (!p->obs_pose || !p->obs_landmark || !p->obs_xy))) {
    v.status = VLBA_ERR_INVALID_ARGUMENT;
    return v;
  }
  // External observation weights before anything else, as
  // optimize_with_observation_weights checks them (optimize.rs:48, 628-650).
  if (p->obs_weight) {
    const uint64_t o = first_failing(p->num_observations, [&](uint64_t k) {
      return std::isfinite(p->obs_weight[k]) && p->obs_weight[k] >= 0.0;
    });
    if (o < p->num_observations) {
      v.status = VLBA_ERR_INVALID_OBSERVATION_WEIGHT;
      v.error_index = o;
      return v;
    }
  }
  // Camera model first (lm.rs:168 `intrinsics()?`); a model outside the
  // radial pinhole family is declined, so the caller runs its CPU solver.
  if (p->num_cameras == 0 || !p->cameras) { v.status = VLBA_ERR_UNSUPPORTED_CAMERA_MODEL; return v; }
  for (uint32_t c = 0; c < p->num_cameras; ++c) {
    DevCamera dc;
    const uint32_t m = p->cameras[c].model;
    if (m > VLBA_CAMERA_OPENCV) { v.status = VLBA_DECLINED; return v; }
    if (!resolve_camera(p->cameras[c], &dc)) {
      // Known model with a tangential term or malformed parameters.
      v.status = (m == VLBA_CAMERA_OPENCV) ? VLBA_DECLINED : VLBA_ERR_UNSUPPORTED_CAMERA_MODEL;
      return v;
    }
  }
  // Stereo observations: known kinds with their arrays, and a pinhole
  // BundleAdjustment::camera (check_stereo_camera_model, problem.rs:733-745).
  bool has_stereo = false, has_rectified = false, has_general = false;
  if (p->obs_kind)
    for (uint64_t o = 0; o < p->num_observations; ++o) {
      const uint32_t k = p->obs_kind[o];
      if (k > kObsGeneralStereo) {
        v.status = VLBA_ERR_INVALID_ARGUMENT;
        v.error_index = o;
        return v;
      }
      has_rectified = has_rectified || k == kObsStereo;
      has_general = has_general || k == kObsGeneralStereo;
    }
  has_stereo = has_rectified || has_general;
  if ((has_stereo && !p->obs_stereo) || (has_general && !p->obs_right_camera)) {
    v.status = VLBA_ERR_INVALID_ARGUMENT;
    return v;
  }
  if (has_stereo && p->cameras[0].model != VLBA_CAMERA_PINHOLE &&
      p->cameras[0].model != VLBA_CAMERA_SIMPLE_PINHOLE) {
    v.status = VLBA_ERR_UNSUPPORTED_CAMERA_MODEL;
    return v;
  }
  if (p->num_poses == 0) { v.status = VLBA_ERR_NO_POSES; return v; }
  if (p->num_observations == 0) { v.status = VLBA_ERR_NO_OBSERVATIONS; return v; }
  if (p->num_landmarks == 0) { v.status = VLBA_ERR_NO_LANDMARKS; return v; }
  // Pose and landmark references list by list, in the reference's order
  // (lm.rs:185-228): monocular, rectified stereo (after its baseline),
  // general stereo (with its right camera), rig.
  auto kind_of = [&](uint64_t o) -> uint32_t { return p->obs_kind ? p->obs_kind[o] : kObsMono; };
  auto refs_ok = [&](uint64_t o) {
    if (p->obs_pose[o] >= p->num_poses) {
      v.status = VLBA_ERR_MISSING_POSE;
      v.error_index = p->obs_pose[o];
      return false;
    }
    if (p->obs_landmark[o] >= p->num_landmarks) {
      v.status = VLBA_ERR_MISSING_LANDMARK;
      v.error_index = p->obs_landmark[o];
      return false;
    }
    return true;
  };
  const int lists[4] = {p->obs_camera ? -1 : (int)kObsMono, (int)kObsStereo, (int)kObsGeneralStereo,
                        p->obs_camera ? (int)kObsMono : -1};
  for (int li = 0; li < 4; ++li) {
    if (lists[li] < 0 || (lists[li] != (int)kObsMono && !has_stereo)) continue;
    if (lists[li] == (int)kObsStereo && has_rectified &&
        !(std::isfinite(p->stereo_baseline) && p->stereo_baseline > 0.0)) {
      v.status = VLBA_ERR_MISSING_STEREO_BASELINE;
      return v;
    }
    // The list's first observation with a bad reference, then its error as
    // the serial checks below order them.
    const uint64_t o = first_failing(p->num_observations, [&](uint64_t k) {
      if (kind_of(k) != (uint32_t)lists[li]) return true;
      return p->obs_pose[k] < p->num_poses && p->obs_landmark[k] < p->num_landmarks &&
             !(lists[li] == (int)kObsGeneralStereo && p->obs_right_camera[k] >= p->num_cameras) &&
             !(lists[li] == (int)kObsMono && p->obs_camera && p->obs_camera[k] >= p->num_cameras);
    });
    if (o < p->num_observations) {
      if (!refs_ok(o)) return v;
      v.status = VLBA_ERR_INVALID_ARGUMENT;
      v.error_index = o;
      return v;
    }
  }
  bool any_var = false;
  for (uint64_t i = 0; i < p->num_poses && !any_var; ++i)
    any_var = !(p->pose_fixed && p->pose_fixed[i]);
  for (uint64_t i = 0; i < p->num_landmarks && !any_var; ++i)
    any_var = !(p->landmark_fixed && p->landmark_fixed[i]);
  if (!any_var) { v.status = VLBA_ERR_ALL_POSES_FIXED; return v; }
  return v;
}

namespace {

void finish_tiles(Plan& P);

// Runs f(t) for t in [0, n) on n threads (t = 0 on the caller's thread),
// rethrowing the first exception.
template <typename F>
void run_threads(uint32_t n, F&& f) {
  std::exception_ptr err;
  std::atomic<bool> failed{false};
  auto body = [&](uint32_t t) {
    try {
      f(t);
    } catch (...) {
      if (!failed.exchange(true)) err = std::current_exception();
    }
  };
  std::vector<std::thread> pool;
  for (uint32_t t = 1; t < n; ++t) pool.emplace_back(body, t);
  body(0);
  for (auto& th : pool) th.join();
  if (err) std::rethrow_exception(err);
}

// Stable counting sort of the indices i in [0, n) by key(i) < m (kNone:
// left out) on T threads over contiguous index ranges: order[] receives
// value_base + i bucket after bucket, off[b] .. off[b + 1] bucket b's range.
// The output does not depend on T.
template <typename Key>
void counting_sort(uint32_t n, uint32_t m, uint32_t T, Key key, uint32_t value_base,
                   uint32_t* order, uint32_t* off) {
  std::vector<std::vector<uint32_t>> tc(T, std::vector<uint32_t>(m, 0));
  auto ilo = [&](uint32_t t) { return (uint32_t)((uint64_t)n * t / T); };
  auto blo = [&](uint32_t t) { return (uint32_t)((uint64_t)m * t / T); };
  run_threads(T, [&](uint32_t t) {
    uint32_t* c = tc[t].data();
    for (uint32_t i = ilo(t); i < ilo(t + 1); ++i) {
      const uint32_t b = key(i);
      if (b != kNone) ++c[b];
    }
  });
  // Bucket totals per chunk of buckets, then each (bucket, range) start.
  std::vector<uint64_t> csum(T + 1, 0);
  run_threads(T, [&](uint32_t t) {
    uint64_t s = 0;
    for (uint32_t b = blo(t); b < blo(t + 1); ++b)
      for (uint32_t u = 0; u < T; ++u) s += tc[u][b];
    csum[t + 1] = s;
  });
  for (uint32_t t = 0; t < T; ++t) csum[t + 1] += csum[t];
  run_threads(T, [&](uint32_t t) {
    uint32_t run = (uint32_t)csum[t];
    for (uint32_t b = blo(t); b < blo(t + 1); ++b) {
      off[b] = run;
      for (uint32_t u = 0; u < T; ++u) {
        const uint32_t c = tc[u][b];
        tc[u][b] = run;
        run += c;
      }
    }
  });
  off[m] = (uint32_t)csum[T];
  run_threads(T, [&](uint32_t t) {
    uint32_t* c = tc[t].data();
    for (uint32_t i = ilo(t); i < ilo(t + 1); ++i) {
      const uint32_t b = key(i);
      if (b != kNone) order[c[b]++] = value_base + i;
    }
  });
}

void build_plan_serial(const vlba_problem* const* problems, const vlba_config* const* configs,
                       uint32_t n, uint32_t tb, Plan* plan, uint32_t max_threads,
                       const RowBlocksFn* device_rows) {
  Plan& P = *plan;
  {
    // A plan rebuilt in place keeps the memory of its largest arrays (their
    // pages stay mapped, so the rebuild takes no page faults on them); their
    // contents go.
    Plan old = std::move(P);
    P = Plan();
    auto keep = [](auto& dst, auto& src) {
      dst.swap(src);
      dst.clear();
    };
    keep(P.pairs, old.pairs);
    keep(P.dup_pairs, old.dup_pairs);
    keep(P.scratch, old.scratch);
    keep(P.points, old.points);
    keep(P.obs_point, old.obs_point);
    keep(P.obs_pose, old.obs_pose);
    keep(P.obs_cam, old.obs_cam);
    keep(P.obs_slot, old.obs_slot);
    keep(P.obs_xy, old.obs_xy);
    keep(P.obs_w, old.obs_w);
    keep(P.obs_src, old.obs_src);
    keep(P.obs_kind, old.obs_kind);
    keep(P.obs_st, old.obs_st);
    keep(P.obs_rcam, old.obs_rcam);
    keep(P.cam_obs, old.cam_obs);
  }
  P.tb = tb;
  P.num_problems = n;
  uint64_t tot_poses = 0, tot_points = 0, tot_obs = 0, tot_cams = 0;
  for (uint32_t i = 0; i < n; ++i) {
    tot_poses += problems[i]->num_poses;
    tot_points += problems[i]->num_landmarks;
    tot_obs += problems[i]->num_observations;
    tot_cams += problems[i]->num_cameras;
  }
  if (tot_poses >= kNone || tot_points >= kNone || tot_obs >= kNone)
    throw std::runtime_error("batch exceeds 2^32 poses, points or observations");
  P.pose_q.resize(4 * tot_poses);
  P.pose_t.resize(3 * tot_poses);
  P.points.resize(3 * tot_points);
  P.pose_slot.assign(tot_poses, kNone);
  P.point_var.assign(tot_points, 0);
  P.pose_prob.resize(tot_poses);
  P.point_prob.resize(tot_points);
  P.pt_off.assign(tot_points + 1, 0);
  P.obs_pose.resize(tot_obs);
  P.obs_cam.resize(tot_obs);
  P.obs_slot.resize(tot_obs);
  P.obs_xy.resize(2 * tot_obs);
  P.obs_point.resize(tot_obs);
  P.obs_src.resize(tot_obs);
  bool weighted = false;
  for (uint32_t i = 0; i < n; ++i) weighted = weighted || problems[i]->obs_weight != nullptr;
  if (weighted) P.obs_w.resize(tot_obs);
  bool stereo = false;
  for (uint32_t i = 0; i < n; ++i) stereo = stereo || problems[i]->obs_kind != nullptr;
  if (stereo) {
    P.obs_kind.resize(tot_obs);
    P.obs_st.resize(2 * tot_obs);
    P.obs_rcam.resize(tot_obs);
  }
  P.cameras.reserve(tot_cams);
  P.prob_pose_begin.push_back(0);
  P.prob_point_begin.push_back(0);
  P.prob_obs_begin.push_back(0);
  P.prob_tr_begin.push_back(0);
  P.prob_chunk_begin.push_back(0);
  P.prob_camera_begin.push_back(0);
  P.chunk_point_begin.push_back(0);
  P.cam_off.push_back(0);
  P.dup_off.push_back(0);
  P.blk_off.push_back(0);
  P.tr_list_off.push_back(0);

  const uint32_t tile_floats = tb * tb * kBlock;
  uint32_t pose_base = 0, point_base = 0, obs_base = 0, slot_base = 0, tr_base = 0;
  uint32_t tile_count = 0;

  for (uint32_t pi = 0; pi < n; ++pi) {
    const vlba_problem* p = problems[pi];
    P.params.push_back(make_params(configs[pi]));
    const uint32_t np = (uint32_t)p->num_poses, nl = (uint32_t)p->num_landmarks,
                   no = (uint32_t)p->num_observations;
    const uint32_t cam_base = (uint32_t)P.cameras.size();
    for (uint32_t c = 0; c < p->num_cameras; ++c) {
      DevCamera dc;
      if (!resolve_camera(p->cameras[c], &dc)) throw std::runtime_error("camera model");
      if (!p->obs_camera) dc.rig = 0;  // monocular: the pose is the camera
      P.cameras.push_back(dc);
    }
    // Poses and variable slots, in index (= ascending id) order (lm.rs:234-249).
    uint32_t nvar = 0;
    for (uint32_t i = 0; i < np; ++i) {
      const uint32_t g = pose_base + i;
      for (int a = 0; a < 4; ++a) P.pose_q[4 * (size_t)g + a] = p->pose_q[4 * (size_t)i + a];
      for (int a = 0; a < 3; ++a) P.pose_t[3 * (size_t)g + a] = p->pose_t[3 * (size_t)i + a];
      P.pose_prob[g] = pi;
      if (!(p->pose_fixed && p->pose_fixed[i])) P.pose_slot[g] = slot_base + nvar++;
    }
    P.real_var_cams += nvar;
    const uint32_t nslots = round_up(nvar, tb);
    for (uint32_t s = 0; s < nslots; ++s) P.slot_prob.push_back(pi);
    {
      const uint32_t Tp = std::max(1u, std::min<uint32_t>(max_threads, nl / 100000));
      std::vector<uint64_t> nvp(Tp, 0);
      run_threads(Tp, [&](uint32_t t) {
        double* const pts = P.points.data();
        uint32_t* const pprob = P.point_prob.data();
        uint8_t* const pvar = P.point_var.data();
        uint64_t nv = 0;
        for (uint32_t j = (uint32_t)((uint64_t)nl * t / Tp); j < (uint32_t)((uint64_t)nl * (t + 1) / Tp); ++j) {
          const uint32_t g = point_base + j;
          for (int a = 0; a < 3; ++a) pts[3 * (size_t)g + a] = p->landmarks[3 * (size_t)j + a];
          pprob[g] = pi;
          const bool var = !(p->landmark_fixed && p->landmark_fixed[j]);
          pvar[g] = var ? 1 : 0;
          nv += var;
        }
        nvp[t] = nv;
      });
      for (uint32_t t = 0; t < Tp; ++t) P.var_points += nvp[t];
    }
    // Point-major observation order: stable counting sort by landmark.
    // Observation-level passes run on up to max_threads threads (the
    // per-thread landmark counts bound to 2^25 words).
    const uint32_t To = std::max(1u, std::min<uint32_t>(max_threads, no / 200000));
    const uint32_t Ts = std::max(1u, std::min<uint32_t>(To, (uint32_t)((32u << 20) / (nl + 1u))));
    std::vector<uint32_t> cnt(nl + 1, 0);
    std::unique_ptr<uint32_t[]> order;  // uninitialised, never page-locked
    // Observations listed by landmark already (point-major exports): the
    // stable sort is the identity, and landmark j starts where the landmark
    // index first reaches j.
    std::vector<uint8_t> unsorted(To, 0);
    const uint32_t* const ol = p->obs_landmark;
    run_threads(To, [&](uint32_t t) {
      const uint32_t a = std::max(1u, (uint32_t)((uint64_t)no * t / To)),
                     e = (uint32_t)((uint64_t)no * (t + 1) / To);
      for (uint32_t o = a; o < e; ++o)
        if (ol[o - 1] > ol[o]) {
          unsorted[t] = 1;
          return;
        }
    });
    const bool identity = std::find(unsorted.begin(), unsorted.end(), 1) == unsorted.end();
    if (identity) {
      run_threads(To, [&](uint32_t t) {
        const uint32_t a = (uint32_t)((uint64_t)no * t / To), e = (uint32_t)((uint64_t)no * (t + 1) / To);
        for (uint32_t o = a; o < e; ++o)
          for (uint32_t j = o ? ol[o - 1] + 1 : 0u; j <= ol[o]; ++j) cnt[j] = o;
        if (t == To - 1)
          for (uint32_t j = no ? ol[no - 1] + 1 : 0u; j <= nl; ++j) cnt[j] = no;
      });
    } else {
      order.reset(new uint32_t[no]);
      counting_sort(no, nl, Ts, [p](uint32_t o) { return p->obs_landmark[o]; }, 0u, order.get(),
                    cnt.data());
    }
    // Observations with a variable point and a variable pose, per thread.
    std::vector<uint64_t> nvo(To, 0);
    run_threads(To, [&](uint32_t t) {
      for (uint32_t j = (uint32_t)((uint64_t)nl * t / To); j < (uint32_t)((uint64_t)nl * (t + 1) / To); ++j) {
        P.pt_off[point_base + j + 1] = obs_base + cnt[j + 1];
        for (uint32_t k = cnt[j]; k < cnt[j + 1]; ++k) P.obs_point[obs_base + k] = point_base + j;
      }
      // The arrays through local pointers (the compiler cannot keep a
      // vector's data pointer in a register across the stores).
      uint32_t* const opose = P.obs_pose.data();
      uint32_t* const ocam = P.obs_cam.data();
      uint32_t* const oslot = P.obs_slot.data();
      double* const oxy = P.obs_xy.data();
      uint32_t* const osrc = P.obs_src.data();
      const uint32_t* const pslot = P.pose_slot.data();
      const uint8_t* const pvar = P.point_var.data();
      uint64_t nv = 0;
      for (uint32_t k = (uint32_t)((uint64_t)no * t / To); k < (uint32_t)((uint64_t)no * (t + 1) / To); ++k) {
        const uint32_t o = identity ? k : order[k];
        const uint32_t g = obs_base + k;
        const uint32_t pose = pose_base + p->obs_pose[o];
        opose[g] = pose;
        const uint32_t kind = p->obs_kind ? p->obs_kind[o] : kObsMono;
        // Stereo observations project through BundleAdjustment::camera.
        ocam[g] = cam_base + (kind == kObsMono && p->obs_camera ? p->obs_camera[o] : 0u);
        if (stereo) {
          P.obs_kind[g] = (uint8_t)kind;
          double s0 = 0.0, s1 = 0.0;
          if (kind == kObsStereo) {
            s0 = p->obs_stereo[2 * (size_t)o];
            s1 = p->stereo_baseline;
          } else if (kind == kObsGeneralStereo) {
            s0 = p->obs_stereo[2 * (size_t)o];
            s1 = p->obs_stereo[2 * (size_t)o + 1];
          }
          P.obs_st[2 * (size_t)g] = s0;
          P.obs_st[2 * (size_t)g + 1] = s1;
          P.obs_rcam[g] = cam_base + (kind == kObsGeneralStereo ? p->obs_right_camera[o] : 0u);
        }
        const uint32_t slot = pslot[pose];
        oslot[g] = slot;
        nv += slot != kNone && pvar[point_base + p->obs_landmark[o]];
        oxy[2 * (size_t)g] = p->obs_xy[2 * (size_t)o];
        oxy[2 * (size_t)g + 1] = p->obs_xy[2 * (size_t)o + 1];
        if (weighted) P.obs_w[g] = p->obs_weight ? p->obs_weight[o] : 1.0;
        osrc[g] = o;
      }
      nvo[t] = nv;
    });
    // Per-slot observation lists (ascending point-major index).
    std::vector<uint32_t> c2(nslots + 1, 0);
    const uint32_t list_base = (uint32_t)P.cam_obs.size();
    P.cam_obs.resize(list_base + (size_t)no);
    counting_sort(no, nslots, To, [&](uint32_t k) {
      const uint32_t s = P.obs_slot[obs_base + k];
      return s == kNone ? kNone : s - slot_base;
    }, obs_base, P.cam_obs.data() + list_base, c2.data());
    P.cam_obs.resize(list_base + (size_t)c2[nslots]);
    for (uint32_t s = 0; s < nslots; ++s) P.cam_off.push_back(list_base + c2[s + 1]);
    const uint64_t pair_base = P.pairs.size();
    std::vector<uint64_t> row_at(nvar + 1, pair_base);
    // The block structure from the device when it can take this problem
    // (one problem, no point seen twice by one slot): the terms are then
    // written there, in the order of the host build below.
    RowBlocks rb;
    const bool device_terms = n == 1 && device_rows && *device_rows &&
                              (*device_rows)(P, nvar, &rb) && rb.row_off.size() == nvar + 1u;
    // Each row's blocks (columns ascending) and their term counts, flat:
    // row i's are [blk_row[i], blk_row[i + 1]) of blk_cols / blk_cnts.
    std::vector<uint32_t> blk_row, blk_cols, blk_cnts;
    if (device_terms) {
      for (uint32_t t = 0; t < To; ++t) P.var_obs += nvo[t];
      blk_row = std::move(rb.row_off);
      blk_cols = std::move(rb.col);
      blk_cnts = std::move(rb.count);
      if (blk_row[0] != 0 || blk_cols.size() != blk_row[nvar] || blk_cnts.size() != blk_row[nvar])
        throw std::runtime_error("device row blocks out of range");
      // Each row's columns below it, ascending, with terms; its term total.
      std::vector<uint64_t> row_terms(nvar, 0);
      run_threads(To, [&](uint32_t t) {
        for (uint32_t i = (uint32_t)((uint64_t)nvar * t / To); i < (uint32_t)((uint64_t)nvar * (t + 1) / To); ++i) {
          if (blk_row[i] > blk_row[i + 1]) throw std::runtime_error("device row blocks out of order");
          uint64_t sum = 0;
          for (uint32_t q = blk_row[i]; q < blk_row[i + 1]; ++q) {
            if (blk_cols[q] >= i || blk_cnts[q] == 0 || (q > blk_row[i] && blk_cols[q] <= blk_cols[q - 1]))
              throw std::runtime_error("device row blocks out of order");
            sum += blk_cnts[q];
          }
          row_terms[i] = sum;
        }
      });
      for (uint32_t i = 0; i < nvar; ++i) row_at[i + 1] = row_at[i] + row_terms[i];
      if (row_at[nvar] >= kNone) throw std::runtime_error("more than 2^32 Schur terms");
      for (uint32_t s = 0; s < nslots; ++s) P.dup_off.push_back((uint32_t)P.dup_pairs.size());
      P.pairs_on_device = true;
      P.num_pairs = row_at[nvar];
      P.row_blk.assign(blk_row.begin(), blk_row.end());
      P.row_blk.resize((size_t)nslots + 1, blk_row[nvar]);
      P.blk_col.assign(blk_cols.begin(), blk_cols.end());
    } else {
      // Camera pairs sharing a variable point: blocks (i, j), j < i (local
      // slots), each holding its terms (x, y) -- x the observation in slot i,
      // y the one in slot j -- in point order and, within a point, in the order
      // of the loop "for a, for b < a" over the point's observations.  Points
      // with enough work are split into T contiguous ranges, one per thread,
      // in three passes that keep that order whatever T is: (A) count each
      // row's terms per range; (B) scatter them row-major, ranges in order,
      // with each term's column beside it; (C) per row, a stable counting sort
      // by column.  A point's observations in one slot give that slot's
      // same-camera terms, both orders.
      uint32_t T = 1;
      std::vector<uint32_t> range{0, nl};
      if (max_threads > 1) {
        std::vector<double> work(nl + 1, 0.0);
        for (uint32_t j = 0; j < nl; ++j) {
          const double t = (double)(cnt[j + 1] - cnt[j]);
          work[j + 1] = work[j] + t * t;
        }
        if (work[nl] > 2e6)
          T = std::max(1u, std::min<uint32_t>({max_threads, nvar, (uint32_t)(work[nl] / 2e5)}));
        range.assign(T + 1, nl);
        range[0] = 0;
        for (uint32_t t = 1, j = 0; t < T; ++t) {
          const double goal = work[nl] * t / T;
          while (j < nl && work[j + 1] < goal) ++j;
          range[t] = j;
        }
      }
      // f(la, lb, a, b) for every pair a > b of variable-slot observations of a
      // variable point in range t (local slots, local observation indices).
      // The arrays are read through local pointers (the compiler cannot keep a
      // vector's data pointer in a register across the callers' stores).
      const uint8_t* const pvar = P.point_var.data() + point_base;
      const uint32_t* const oslot = P.obs_slot.data() + obs_base;
      const uint32_t* const pcnt = cnt.data();
      auto each_pair = [&](uint32_t t, auto&& f, uint64_t* var) {
        uint64_t nv = 0;
        for (uint32_t j = range[t], je = range[t + 1]; j < je; ++j) {
          if (!pvar[j]) continue;
          const uint32_t k0 = pcnt[j], k1 = pcnt[j + 1];
          for (uint32_t a = k0; a < k1; ++a) {
            const uint32_t sa = oslot[a];
            if (sa == kNone) continue;
            ++nv;
            for (uint32_t b = k0; b < a; ++b) {
              const uint32_t sb = oslot[b];
              if (sb != kNone) f(sa - slot_base, sb - slot_base, a, b);
            }
          }
        }
        if (var) *var += nv;
      };
      // (A) per range: terms of each row, same-camera terms of each slot.
      std::vector<std::vector<uint64_t>> tcnt(T, std::vector<uint64_t>(2 * (size_t)nvar, 0));
      std::vector<uint64_t> tvar(T, 0);
      run_threads(T, [&](uint32_t t) {
        uint64_t* c = tcnt[t].data();
        each_pair(t, [c, nvar](uint32_t la, uint32_t lb, uint32_t, uint32_t) {
          if (la != lb) ++c[std::max(la, lb)];
          else c[nvar + la] += 2;
        }, &tvar[t]);
      });
      for (uint32_t t = 0; t < T; ++t) P.var_obs += tvar[t];
      // Row and slot ranges; per range, its start inside each (the counts
      // become positions).
      const uint64_t dup_base = P.dup_pairs.size();
      std::vector<uint64_t> dup_at(nslots + 1, dup_base);
      for (uint32_t i = 0; i < nvar; ++i) {
        uint64_t at = row_at[i], d = dup_at[i];
        for (uint32_t t = 0; t < T; ++t) {
          const uint64_t c = tcnt[t][i], e = tcnt[t][nvar + i];
          tcnt[t][i] = at;
          tcnt[t][nvar + i] = d;
          at += c;
          d += e;
        }
        row_at[i + 1] = at;
        dup_at[i + 1] = d;
      }
      for (uint32_t s = nvar; s < nslots; ++s) dup_at[s + 1] = dup_at[s];
      if (row_at[nvar] >= kNone) throw std::runtime_error("more than 2^32 Schur terms");
      if (dup_at[nslots] >= kNone) throw std::runtime_error("more than 2^32 same-camera terms");
      P.pairs.resize(row_at[nvar]);
      P.dup_pairs.resize(dup_at[nslots]);
      for (uint32_t s = 0; s < nslots; ++s) P.dup_off.push_back((uint32_t)dup_at[s + 1]);
      // (B) scatter, each term's column beside it.
      auto& term_col = P.scratch;
      term_col.resize(row_at[nvar] - pair_base);
      run_threads(T, [&](uint32_t t) {
        uint64_t* pos = tcnt[t].data();
        uint64_t* dpos = pos + nvar;
        PairIdx* const pairs = P.pairs.data();
        PairIdx* const dups = P.dup_pairs.data();
        uint32_t* const tcol = term_col.data();
        each_pair(t, [=](uint32_t la, uint32_t lb, uint32_t a, uint32_t b) {
          const uint32_t ga = obs_base + a, gb = obs_base + b;
          if (la > lb) {
            const uint64_t w = pos[la]++;
            tcol[w - pair_base] = lb;
            pairs[w] = PairIdx{ga, gb};
          } else if (lb > la) {
            const uint64_t w = pos[lb]++;
            tcol[w - pair_base] = la;
            pairs[w] = PairIdx{gb, ga};
          } else {
            dups[dpos[la]++] = PairIdx{ga, gb};
            dups[dpos[la]++] = PairIdx{gb, ga};
          }
        }, nullptr);
      });
      // (C) per row, a stable counting sort of its terms by column; the row's
      // blocks are its distinct columns, ascending.
      std::vector<std::vector<uint32_t>> row_col(nvar), row_count(nvar);
      {
        std::atomic<uint32_t> next{0};
        run_threads(T, [&](uint32_t) {
          std::vector<uint32_t> mark(nvar, 0), touched;
          std::vector<uint64_t> at(nvar, 0);
          std::vector<PairIdx> buf;
          const uint32_t* const tcol = term_col.data();
          PairIdx* const pairs = P.pairs.data();
          uint32_t* const mk = mark.data();
          for (uint32_t i; (i = next.fetch_add(1)) < nvar;) {
            const uint64_t lo = row_at[i], hi = row_at[i + 1];
            touched.clear();
            for (uint64_t k = lo; k < hi; ++k)
              if (mk[tcol[k - pair_base]]++ == 0) touched.push_back(tcol[k - pair_base]);
            std::sort(touched.begin(), touched.end());
            row_col[i] = touched;
            row_count[i].resize(touched.size());
            uint64_t run = lo;
            for (size_t b = 0; b < touched.size(); ++b) {
              row_count[i][b] = mark[touched[b]];
              at[touched[b]] = run;
              run += mark[touched[b]];
              mark[touched[b]] = 0;
            }
            if (touched.size() > 1) {
              buf.assign(pairs + lo, pairs + hi);
              uint64_t* const at_ = at.data();
              for (uint64_t k = lo; k < hi; ++k) pairs[at_[tcol[k - pair_base]]++] = buf[k - lo];
            }
          }
        });
      }
      term_col.clear();
      blk_row.assign(nvar + 1, 0u);
      for (uint32_t i = 0; i < nvar; ++i) blk_row[i + 1] = blk_row[i] + (uint32_t)row_col[i].size();
      blk_cols.reserve(blk_row[nvar]);
      blk_cnts.reserve(blk_row[nvar]);
      for (uint32_t i = 0; i < nvar; ++i) {
        blk_cols.insert(blk_cols.end(), row_col[i].begin(), row_col[i].end());
        blk_cnts.insert(blk_cnts.end(), row_count[i].begin(), row_count[i].end());
      }
    }

    // Blocks in row-major order; per-tile existence.  Rows run on the host's
    // threads in whole tile rows (a tile row's existence flags are its own).
    const uint32_t ntr = nslots / tb;
    std::vector<uint8_t> tile_has((size_t)ntr * ntr, 0);
    const uint32_t blk_base = (uint32_t)P.blk_dst.size();
    const uint32_t nblk = blk_row[nvar];
    const uint32_t Tr = std::max(1u, std::min<uint32_t>(To, ntr));
    auto tile_rows = [&](uint32_t t, auto&& f) {
      for (uint32_t I = (uint32_t)((uint64_t)ntr * t / Tr); I < (uint32_t)((uint64_t)ntr * (t + 1) / Tr); ++I)
        for (uint32_t i = I * tb; i < std::min(nvar, (I + 1) * tb); ++i) f(I, i);
    };
    P.blk_off.resize((size_t)blk_base + 1 + nblk);
    uint32_t* const boff = P.blk_off.data() + blk_base + 1;
    run_threads(Tr, [&](uint32_t t) {
      tile_rows(t, [&](uint32_t I, uint32_t i) {
        uint64_t run = row_at[i];
        for (uint32_t b = blk_row[i]; b < blk_row[i + 1]; ++b) {
          tile_has[(size_t)I * ntr + blk_cols[b] / tb] = 1;
          run += blk_cnts[b];
          boff[b] = (uint32_t)run;
        }
      });
    });
    P.camera_pairs += nblk;
    for (uint32_t t = 0; t < ntr; ++t) tile_has[(size_t)t * ntr + t] = 1;
    // Compact tile ids, row-major.
    std::vector<uint32_t> tile_id((size_t)ntr * ntr, kNone);
    for (uint32_t I = 0; I < ntr; ++I)
      for (uint32_t J = 0; J <= I; ++J)
        if (tile_has[(size_t)I * ntr + J]) {
          tile_id[(size_t)I * ntr + J] = tile_count++;
          if (tr_base + I > 0xFFFFu || tr_base + J > 0xFFFFu)
            throw std::runtime_error("more than 65535 tile rows");
          P.tile_ij.push_back(((tr_base + I) << 16) | (tr_base + J));
        }
    // Block destinations.
    P.blk_dst.resize(blk_base + nblk);
    run_threads(Tr, [&](uint32_t t) {
      tile_rows(t, [&](uint32_t I, uint32_t i) {
        for (uint32_t b = blk_row[i]; b < blk_row[i + 1]; ++b) {
          const uint32_t jj = blk_cols[b];
          const uint32_t J = jj / tb, li = i % tb, lj = jj % tb;
          const uint32_t tt = tile_id[(size_t)I * ntr + J];
          PairIdx dst;
          dst.a = tt * tile_floats + (li * tb + lj) * kBlock;
          dst.b = (I == J) ? tt * tile_floats + (lj * tb + li) * kBlock : kNone;
          P.blk_dst[blk_base + b] = dst;
        }
      });
    });
    for (uint32_t s = 0; s < nslots; ++s) {
      const uint32_t I = s / tb, li = s % tb;
      P.diag_dst.push_back(tile_id[(size_t)I * ntr + I] * tile_floats + (li * tb + li) * kBlock);
    }
    // Tile-row partial lists: row sides (I, J <= I), then column sides (K > I, I).
    for (uint32_t I = 0; I < ntr; ++I) {
      for (uint32_t J = 0; J <= I; ++J) {
        const uint32_t t = tile_id[(size_t)I * ntr + J];
        if (t != kNone) P.tr_list.push_back(2 * t);
      }
      for (uint32_t K = I + 1; K < ntr; ++K) {
        const uint32_t t = tile_id[(size_t)K * ntr + I];
        if (t != kNone) P.tr_list.push_back(2 * t + 1);
      }
      P.tr_list_off.push_back((uint32_t)P.tr_list.size());
      P.tr_prob.push_back(pi);
    }
    // Point chunks of at most 256 points.
    for (uint32_t j0 = 0; j0 < nl; j0 += 256)
      P.chunk_point_begin.push_back(point_base + std::min(nl, j0 + 256));
    pose_base += np;
    point_base += nl;
    obs_base += no;
    slot_base += nslots;
    tr_base += ntr;
    P.prob_pose_begin.push_back(pose_base);
    P.prob_point_begin.push_back(point_base);
    P.prob_obs_begin.push_back(obs_base);
    P.prob_tr_begin.push_back(tr_base);
    P.prob_chunk_begin.push_back((uint32_t)P.chunk_point_begin.size() - 1);
    P.prob_camera_begin.push_back((uint32_t)P.cameras.size());
  }
  P.num_var_cams = slot_base;
  P.num_tile_rows = tr_base;
  // Partial slots: position of (tile, side) in the tile-row lists, so a row's
  // partials are contiguous.
  finish_tiles(P);
  if (!P.pairs_on_device) P.num_pairs = P.pairs.size();
  // Lanes per block in the off-diagonal assembly.  The lane count sets the
  // order of each block's sum, so it is the same for every problem and batch
  // (a result must not depend on what it is batched with).
  P.group = 4;
}

// Partial slots (positions of each tile's row and column side in the
// tile-row lists) and the per-tile metadata the PCG reads.
void finish_tiles(Plan& P) {
  P.tile_slot.assign(P.tile_ij.size(), PairIdx{kNone, kNone});
  for (uint32_t m = 0; m < (uint32_t)P.tr_list.size(); ++m) {
    const uint32_t t = P.tr_list[m] / 2, side = P.tr_list[m] % 2;
    if (side == 0) P.tile_slot[t].a = m;
    else P.tile_slot[t].b = m;
  }
  P.tile_meta.resize(4 * P.tile_ij.size());
  for (size_t t = 0; t < P.tile_ij.size(); ++t) {
    P.tile_meta[4 * t] = P.tile_ij[t];
    P.tile_meta[4 * t + 1] = P.tile_slot[t].a;
    P.tile_meta[4 * t + 2] = P.tile_slot[t].b;
    P.tile_meta[4 * t + 3] = P.tr_prob[P.tile_ij[t] >> 16];
  }
}

}  // namespace

void build_reduced_plan(uint32_t n, const uint32_t* edges, uint64_t ne, uint32_t tb,
                        const LmParams& params, Plan* plan) {
  Plan& P = *plan;
  P = Plan();
  if (n == 0) throw std::runtime_error("a reduced system of no nodes");
  if (ne >= kNone) throw std::runtime_error("more than 2^32 edges");
  P.tb = tb;
  P.group = 4;
  P.num_problems = 1;
  const uint32_t nslots = round_up(n, tb), ntr = nslots / tb;
  P.prob_pose_begin = {0, 0};
  P.prob_point_begin = {0, 0};
  P.prob_obs_begin = {0, 0};
  P.prob_tr_begin = {0, ntr};
  P.prob_chunk_begin = {0, 0};
  P.prob_camera_begin = {0, 0};
  P.params = {params};
  P.slot_prob.assign(nslots, 0u);
  P.pt_off = {0};
  P.cam_off.assign(nslots + 1, 0u);
  P.dup_off.assign(nslots + 1, 0u);
  P.chunk_point_begin = {0};
  P.num_var_cams = nslots;
  P.num_tile_rows = ntr;
  P.real_var_cams = n;
  // Tiles: the diagonal ones and those holding an edge's (b, a) block.
  std::vector<uint8_t> tile_has((size_t)ntr * ntr, 0);
  for (uint32_t t = 0; t < ntr; ++t) tile_has[(size_t)t * ntr + t] = 1;
  for (uint64_t e = 0; e < ne; ++e) {
    const uint32_t a = edges[2 * e], b = edges[2 * e + 1];
    if (!(a < b) || b >= n) throw std::runtime_error("edge (a, b) must have a < b < nodes");
    if (e && (uint64_t)edges[2 * e - 2] * n + edges[2 * e - 1] >= (uint64_t)a * n + b)
      throw std::runtime_error("edges must be sorted and distinct");
    tile_has[(size_t)(b / tb) * ntr + a / tb] = 1;
  }
  std::vector<uint32_t> tile_id((size_t)ntr * ntr, kNone);
  uint32_t count = 0;
  for (uint32_t I = 0; I < ntr; ++I)
    for (uint32_t J = 0; J <= I; ++J)
      if (tile_has[(size_t)I * ntr + J]) {
        if (I > 0xFFFFu) throw std::runtime_error("more than 65535 tile rows");
        tile_id[(size_t)I * ntr + J] = count++;
        P.tile_ij.push_back((I << 16) | J);
      }
  const uint32_t tf = tb * tb * kBlock;
  if ((uint64_t)count * tf >= kNone) throw std::runtime_error("reduced system exceeds 2^32 floats");
  P.blk_off.assign(ne + 1, 0u);
  P.blk_dst.resize(ne);
  for (uint64_t e = 0; e < ne; ++e) {
    const uint32_t a = edges[2 * e], b = edges[2 * e + 1];
    const uint32_t I = b / tb, J = a / tb, li = b % tb, lj = a % tb;
    const uint32_t t = tile_id[(size_t)I * ntr + J];
    P.blk_dst[e].a = t * tf + (li * tb + lj) * kBlock;
    P.blk_dst[e].b = (I == J) ? t * tf + (lj * tb + li) * kBlock : kNone;
  }
  for (uint32_t sidx = 0; sidx < nslots; ++sidx) {
    const uint32_t I = sidx / tb, li = sidx % tb;
    P.diag_dst.push_back(tile_id[(size_t)I * ntr + I] * tf + (li * tb + li) * kBlock);
  }
  P.tr_list_off = {0};
  for (uint32_t I = 0; I < ntr; ++I) {
    for (uint32_t J = 0; J <= I; ++J) {
      const uint32_t t = tile_id[(size_t)I * ntr + J];
      if (t != kNone) P.tr_list.push_back(2 * t);
    }
    for (uint32_t K = I + 1; K < ntr; ++K) {
      const uint32_t t = tile_id[(size_t)K * ntr + I];
      if (t != kNone) P.tr_list.push_back(2 * t + 1);
    }
    P.tr_list_off.push_back((uint32_t)P.tr_list.size());
    P.tr_prob.push_back(0);
  }
  P.camera_pairs = ne;
  finish_tiles(P);
}

void merge_plans(const std::vector<const Plan*>& parts, Plan* out) {
  Plan& P = *out;
  {
    // As in a rebuild in place: the large arrays keep their memory.
    Plan old = std::move(P);
    P = Plan();
    auto keep = [](auto& dst, auto& src) {
      dst.swap(src);
      dst.clear();
    };
    keep(P.pairs, old.pairs);
    keep(P.dup_pairs, old.dup_pairs);
    keep(P.obs_point, old.obs_point);
    keep(P.obs_pose, old.obs_pose);
    keep(P.obs_cam, old.obs_cam);
    keep(P.obs_slot, old.obs_slot);
    keep(P.obs_xy, old.obs_xy);
    keep(P.obs_w, old.obs_w);
    keep(P.obs_src, old.obs_src);
    keep(P.obs_kind, old.obs_kind);
    keep(P.obs_st, old.obs_st);
    keep(P.obs_rcam, old.obs_rcam);
    keep(P.cam_obs, old.cam_obs);
  }
  if (parts.empty()) throw std::runtime_error("merge of no plans");
  P.tb = parts[0]->tb;
  P.group = parts[0]->group;
  const uint32_t tf = P.tb * P.tb * kBlock;
  // Where each part starts in every concatenated array (prefix sums).
  struct Base {
    uint64_t prob, pose, point, obs, slot, tr, tile, cam, pair, dup, camobs, trl, chunk, blk;
  };
  const size_t np = parts.size();
  std::vector<Base> at(np + 1);
  at[0] = Base{};
  for (size_t i = 0; i < np; ++i) {
    const Plan& Q = *parts[i];
    if (Q.tb != P.tb || Q.group != P.group) throw std::runtime_error("plans of different shapes");
    Base b = at[i];
    b.prob += Q.num_problems;
    b.pose += Q.pose_prob.size();
    b.point += Q.point_prob.size();
    b.obs += Q.obs_pose.size();
    b.slot += Q.num_var_cams;
    b.tr += Q.num_tile_rows;
    b.tile += Q.tile_ij.size();
    b.cam += Q.cameras.size();
    b.pair += Q.pairs.size();
    b.dup += Q.dup_pairs.size();
    b.camobs += Q.cam_obs.size();
    b.trl += Q.tr_list.size();
    b.chunk += Q.chunk_point_begin.size() - 1;
    b.blk += Q.blk_dst.size();
    at[i + 1] = b;
    P.real_var_cams += Q.real_var_cams;
    P.var_points += Q.var_points;
    P.var_obs += Q.var_obs;
    P.camera_pairs += Q.camera_pairs;
  }
  const Base& T = at[np];
  if (T.pose >= kNone || T.point >= kNone || T.obs >= kNone)
    throw std::runtime_error("batch exceeds 2^32 poses, points or observations");
  if (T.pair >= kNone || T.dup >= kNone || T.camobs >= kNone)
    throw std::runtime_error("batch exceeds 2^32 Schur terms");
  if (T.tr > 0x10000u) throw std::runtime_error("more than 65535 tile rows");
  if (T.tile * tf >= kNone) throw std::runtime_error("reduced systems exceed 2^32 floats");
  P.num_problems = (uint32_t)T.prob;
  P.num_var_cams = (uint32_t)T.slot;
  P.num_tile_rows = (uint32_t)T.tr;
  // Sized once; every part then writes its own ranges.
  for (auto* v : {&P.prob_pose_begin, &P.prob_point_begin, &P.prob_obs_begin, &P.prob_tr_begin,
                  &P.prob_chunk_begin, &P.prob_camera_begin})
    v->assign(T.prob + 1, 0u);
  P.pose_prob.resize(T.pose);
  P.point_prob.resize(T.point);
  P.slot_prob.resize(T.slot);
  P.tr_prob.resize(T.tr);
  P.params.resize(T.prob);
  P.pose_q.resize(4 * T.pose);
  P.pose_t.resize(3 * T.pose);
  P.points.resize(3 * T.point);
  P.pose_slot.resize(T.pose);
  P.point_var.resize(T.point);
  P.cameras.resize(T.cam);
  P.pt_off.assign(T.point + 1, 0u);
  P.obs_point.resize(T.obs);
  P.obs_pose.resize(T.obs);
  P.obs_cam.resize(T.obs);
  P.obs_slot.resize(T.obs);
  P.obs_xy.resize(2 * T.obs);
  P.obs_src.resize(T.obs);
  bool weighted = false;
  for (const Plan* q : parts) weighted = weighted || !q->obs_w.empty();
  if (weighted) P.obs_w.resize(T.obs);
  bool stereo = false;
  for (const Plan* q : parts) stereo = stereo || !q->obs_kind.empty();
  if (stereo) {
    P.obs_kind.resize(T.obs);
    P.obs_st.resize(2 * T.obs);
    P.obs_rcam.resize(T.obs);
  }
  P.cam_off.assign(T.slot + 1, 0u);
  P.cam_obs.resize(T.camobs);
  P.tile_ij.resize(T.tile);
  P.blk_off.assign(T.blk + 1, 0u);
  P.pairs.resize(T.pair);
  P.blk_dst.resize(T.blk);
  P.diag_dst.resize(T.slot);
  P.dup_off.assign(T.slot + 1, 0u);
  P.dup_pairs.resize(T.dup);
  P.tr_list_off.assign(T.tr + 1, 0u);
  P.tr_list.resize(T.trl);
  P.chunk_point_begin.assign(T.chunk + 1, 0u);
  auto fill = [&](size_t i) {
    const Plan& Q = *parts[i];
    const Base& b = at[i];
    const uint32_t prob_b = (uint32_t)b.prob, pose_b = (uint32_t)b.pose, point_b = (uint32_t)b.point,
                   obs_b = (uint32_t)b.obs, slot_b = (uint32_t)b.slot, tr_b = (uint32_t)b.tr,
                   tile_b = (uint32_t)b.tile, cam_b = (uint32_t)b.cam, pair_b = (uint32_t)b.pair,
                   dup_b = (uint32_t)b.dup, camobs_b = (uint32_t)b.camobs, trl_b = (uint32_t)b.trl,
                   chunk_b = (uint32_t)b.chunk, blk_b = (uint32_t)b.blk;
    for (uint32_t qi = 0; qi < Q.num_problems; ++qi) {
      const size_t o = (size_t)prob_b + qi + 1;
      P.prob_pose_begin[o] = pose_b + Q.prob_pose_begin[qi + 1];
      P.prob_point_begin[o] = point_b + Q.prob_point_begin[qi + 1];
      P.prob_obs_begin[o] = obs_b + Q.prob_obs_begin[qi + 1];
      P.prob_tr_begin[o] = tr_b + Q.prob_tr_begin[qi + 1];
      P.prob_chunk_begin[o] = chunk_b + Q.prob_chunk_begin[qi + 1];
      P.prob_camera_begin[o] = cam_b + Q.prob_camera_begin[qi + 1];
      P.params[prob_b + qi] = Q.params[qi];
    }
    auto shift = [](auto& dst, size_t d0, const auto& src, uint32_t add) {
      for (size_t k = 0; k < src.size(); ++k) dst[d0 + k] = src[k] + add;
    };
    auto shift_none = [](auto& dst, size_t d0, const auto& src, uint32_t add) {
      for (size_t k = 0; k < src.size(); ++k) dst[d0 + k] = src[k] == kNone ? kNone : src[k] + add;
    };
    auto copy = [](auto& dst, size_t d0, const auto& src) {
      if (!src.empty()) std::memcpy(&dst[d0], src.data(), src.size() * sizeof(src[0]));
    };
    // Offset arrays: entries 1.. of the part after the previous parts' entries.
    auto shift_off = [](auto& dst, size_t d0, const auto& src, uint32_t add) {
      for (size_t k = 1; k < src.size(); ++k) dst[d0 + k] = src[k] + add;
    };
    shift(P.pose_prob, pose_b, Q.pose_prob, prob_b);
    shift(P.point_prob, point_b, Q.point_prob, prob_b);
    shift(P.slot_prob, slot_b, Q.slot_prob, prob_b);
    shift(P.tr_prob, tr_b, Q.tr_prob, prob_b);
    copy(P.pose_q, 4 * (size_t)pose_b, Q.pose_q);
    copy(P.pose_t, 3 * (size_t)pose_b, Q.pose_t);
    copy(P.points, 3 * (size_t)point_b, Q.points);
    shift_none(P.pose_slot, pose_b, Q.pose_slot, slot_b);
    copy(P.point_var, point_b, Q.point_var);
    copy(P.cameras, cam_b, Q.cameras);
    shift_off(P.pt_off, point_b, Q.pt_off, obs_b);
    shift(P.obs_point, obs_b, Q.obs_point, point_b);
    shift(P.obs_pose, obs_b, Q.obs_pose, pose_b);
    shift(P.obs_cam, obs_b, Q.obs_cam, cam_b);
    shift_none(P.obs_slot, obs_b, Q.obs_slot, slot_b);
    copy(P.obs_xy, 2 * (size_t)obs_b, Q.obs_xy);
    copy(P.obs_src, obs_b, Q.obs_src);
    if (stereo) {
      const size_t no = Q.obs_pose.size();
      if (Q.obs_kind.empty()) {
        std::fill_n(P.obs_kind.begin() + obs_b, no, (uint8_t)kObsMono);
        std::fill_n(P.obs_st.begin() + 2 * (size_t)obs_b, 2 * no, 0.0);
        std::fill_n(P.obs_rcam.begin() + obs_b, no, cam_b);
      } else {
        copy(P.obs_kind, obs_b, Q.obs_kind);
        copy(P.obs_st, 2 * (size_t)obs_b, Q.obs_st);
        shift(P.obs_rcam, obs_b, Q.obs_rcam, cam_b);
      }
    }
    if (weighted) {
      if (Q.obs_w.empty()) std::fill_n(P.obs_w.begin() + obs_b, Q.obs_pose.size(), 1.0);
      else copy(P.obs_w, obs_b, Q.obs_w);
    }
    shift_off(P.cam_off, slot_b, Q.cam_off, camobs_b);
    shift(P.cam_obs, camobs_b, Q.cam_obs, obs_b);
    for (size_t k = 0; k < Q.tile_ij.size(); ++k) {
      const uint32_t v = Q.tile_ij[k];
      P.tile_ij[tile_b + k] = (((v >> 16) + tr_b) << 16) | ((v & 0xFFFFu) + tr_b);
    }
    shift_off(P.blk_off, blk_b, Q.blk_off, pair_b);
    for (size_t k = 0; k < Q.pairs.size(); ++k)
      P.pairs[pair_b + k] = PairIdx{obs_b + Q.pairs[k].a, obs_b + Q.pairs[k].b};
    const uint32_t fo = tile_b * tf;
    for (size_t k = 0; k < Q.blk_dst.size(); ++k) {
      const PairIdx& v = Q.blk_dst[k];
      P.blk_dst[blk_b + k] = PairIdx{v.a + fo, v.b == kNone ? kNone : v.b + fo};
    }
    shift(P.diag_dst, slot_b, Q.diag_dst, fo);
    shift_off(P.dup_off, slot_b, Q.dup_off, dup_b);
    for (size_t k = 0; k < Q.dup_pairs.size(); ++k)
      P.dup_pairs[dup_b + k] = PairIdx{obs_b + Q.dup_pairs[k].a, obs_b + Q.dup_pairs[k].b};
    shift_off(P.tr_list_off, tr_b, Q.tr_list_off, trl_b);
    shift(P.tr_list, trl_b, Q.tr_list, 2 * tile_b);
    shift_off(P.chunk_point_begin, chunk_b, Q.chunk_point_begin, point_b);
  };
  const uint32_t nt = (uint32_t)std::max<size_t>(
      1, std::min<size_t>({np, std::max(1u, std::thread::hardware_concurrency()), T.obs / 65536 + 1}));
  std::atomic<size_t> next{0};
  run_threads(nt, [&](uint32_t) {
    for (size_t i; (i = next.fetch_add(1)) < np;) fill(i);
  });
  P.num_pairs = P.pairs.size();
  finish_tiles(P);
}

void build_plan(const vlba_problem* const* problems, const vlba_config* const* configs,
                uint32_t n, uint32_t tb, Plan* plan, uint32_t max_threads,
                const RowBlocksFn* device_rows) {
  if (max_threads == 0) max_threads = std::max(1u, std::thread::hardware_concurrency());
  if (n <= 1) {
    build_plan_serial(problems, configs, n, tb, plan, max_threads, device_rows);
    return;
  }
  // One plan per problem on the host's threads, then one merge: the same
  // per-problem layout as a single build, so results do not depend on it.
  std::vector<Plan> parts(n);
  std::atomic<uint32_t> next{0};
  std::exception_ptr err;
  std::atomic<bool> failed{false};
  auto work = [&] {
    for (uint32_t i; (i = next.fetch_add(1)) < n && !failed.load();) {
      try {
        build_plan_serial(problems + i, configs + i, 1, tb, &parts[i], 1, nullptr);
      } catch (...) {
        if (!failed.exchange(true)) err = std::current_exception();
      }
    }
  };
  const uint32_t nt = std::max(1u, std::min<uint32_t>(n, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  if (err) std::rethrow_exception(err);
  std::vector<const Plan*> ptrs;
  for (const Plan& q : parts) ptrs.push_back(&q);
  merge_plans(ptrs, plan);
}

// True when pred(i) holds for every i in [0, n); long ranges are checked on
// the host's threads.
template <typename F>
bool all_of_range(uint64_t n, F&& pred) {
  const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const uint32_t T = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(hw, n >> 16));
  std::atomic<bool> ok{true};
  run_threads(T, [&](uint32_t t) {
    for (uint64_t i = n * t / T, e = n * (t + 1) / T; i < e; ++i)
      if (!pred(i)) {
        ok = false;
        return;
      }
  });
  return ok;
}

std::string check_plan(const Plan& P) {
  const uint64_t nposes = P.pose_prob.size(), npts = P.point_prob.size(),
                 nobs = P.obs_pose.size(), ncam = P.cameras.size(), nslots = P.num_var_cams;
  const uint64_t ntiles = P.tile_ij.size();
  const uint64_t tile_floats = (uint64_t)P.tb * P.tb * kBlock;
  auto bad = [](const char* what) { return std::string("plan check failed: ") + what; };
  if (P.pt_off.size() != npts + 1 || P.pt_off.back() != nobs) return bad("pt_off");
  if (!all_of_range(npts, [&](uint64_t j) { return P.pt_off[j] <= P.pt_off[j + 1]; }))
    return bad("pt_off order");
  if (P.obs_cam.size() != nobs || P.obs_slot.size() != nobs || P.obs_xy.size() != 2 * nobs ||
      P.obs_point.size() != nobs || (!P.obs_w.empty() && P.obs_w.size() != nobs))
    return bad("obs sizes");
  if (!P.obs_kind.empty()) {
    if (P.obs_kind.size() != nobs || P.obs_st.size() != 2 * nobs || P.obs_rcam.size() != nobs)
      return bad("stereo sizes");
    if (!all_of_range(nobs, [&](uint64_t k) {
          return P.obs_kind[k] <= kObsGeneralStereo && P.obs_rcam[k] < ncam;
        }))
      return bad("stereo observations");
  }
  if (!all_of_range(nobs, [&](uint64_t k) {
        const uint32_t l = P.obs_point[k];
        return l < npts && P.pt_off[l] <= k && P.pt_off[l + 1] > k && P.obs_pose[k] < nposes &&
               P.obs_cam[k] < ncam && (P.obs_slot[k] == kNone || P.obs_slot[k] < nslots);
      }))
    return bad("observation arrays");
  for (uint64_t i = 0; i < nposes; ++i)
    if (P.pose_slot[i] != kNone && P.pose_slot[i] >= nslots) return bad("pose_slot");
  if (P.cam_off.size() != nslots + 1 || P.cam_off.back() != P.cam_obs.size()) return bad("cam_off");
  if (!all_of_range(nslots, [&](uint64_t s) { return P.cam_off[s] <= P.cam_off[s + 1]; }))
    return bad("cam_off order");
  if (!all_of_range(P.cam_obs.size(), [&](uint64_t q) { return P.cam_obs[q] < nobs; }))
    return bad("cam_obs");
  if (P.slot_prob.size() != nslots || nslots != (uint64_t)P.num_tile_rows * P.tb)
    return bad("slots");
  const uint64_t npairs = P.pairs_on_device ? P.num_pairs : P.pairs.size();
  if (P.blk_off.size() != P.blk_dst.size() + 1 || P.blk_off.back() != npairs)
    return bad("blk_off");
  if (!all_of_range(P.blk_off.size() - 1, [&](uint64_t b) { return P.blk_off[b] <= P.blk_off[b + 1]; }))
    return bad("blk_off order");
  // Terms built on the device are checked there, against the same ranges,
  // before any kernel reads them.
  if (P.pairs_on_device) {
    if (!P.pairs.empty() || P.num_problems != 1 || P.blk_col.size() != P.blk_dst.size() ||
        P.row_blk.size() != (size_t)P.num_var_cams + 1 || P.row_blk.back() != P.blk_col.size())
      return bad("device terms");
    if (!all_of_range(P.row_blk.size() - 1, [&](uint64_t i) { return P.row_blk[i] <= P.row_blk[i + 1]; }))
      return bad("row_blk order");
    if (!all_of_range(P.row_blk.size() - 1, [&](uint64_t i) {
          for (uint32_t b = P.row_blk[i]; b < P.row_blk[i + 1]; ++b)
            if (P.blk_col[b] >= i || (b > P.row_blk[i] && P.blk_col[b] <= P.blk_col[b - 1]))
              return false;
          return true;
        }))
      return bad("blk_col");
  }
  if (!all_of_range(P.pairs.size(), [&](uint64_t q) { return P.pairs[q].a < nobs && P.pairs[q].b < nobs; }))
    return bad("pairs");
  if (!all_of_range(P.blk_dst.size(), [&](uint64_t b) {
        const PairIdx& d = P.blk_dst[b];
        return (uint64_t)d.a + kBlock <= ntiles * tile_floats &&
               (d.b == kNone || (uint64_t)d.b + kBlock <= ntiles * tile_floats);
      }))
    return bad("blk_dst");
  if (P.diag_dst.size() != nslots) return bad("diag_dst size");
  for (uint32_t d : P.diag_dst)
    if ((uint64_t)d + kBlock > ntiles * tile_floats) return bad("diag_dst");
  if (P.dup_off.size() != nslots + 1 || P.dup_off.back() != P.dup_pairs.size()) return bad("dup_off");
  if (!all_of_range(P.dup_pairs.size(),
                    [&](uint64_t q) { return P.dup_pairs[q].a < nobs && P.dup_pairs[q].b < nobs; }))
    return bad("dup_pairs");
  for (uint32_t ij : P.tile_ij)
    if ((ij >> 16) >= P.num_tile_rows || (ij & 0xFFFFu) > (ij >> 16)) return bad("tile_ij");
  if (P.tr_list_off.size() != (uint64_t)P.num_tile_rows + 1 || P.tr_list_off.back() != P.tr_list.size())
    return bad("tr_list_off");
  for (uint32_t e : P.tr_list)
    if (e >= 2 * ntiles) return bad("tr_list");
  if (P.tile_slot.size() != ntiles) return bad("tile_slot size");
  for (uint64_t t = 0; t < ntiles; ++t) {
    const uint32_t I = P.tile_ij[t] >> 16, J = P.tile_ij[t] & 0xFFFFu;
    if (P.tile_slot[t].a >= P.tr_list.size()) return bad("tile_slot row");
    if ((I != J) != (P.tile_slot[t].b != kNone)) return bad("tile_slot column presence");
    if (I != J && P.tile_slot[t].b >= P.tr_list.size()) return bad("tile_slot column");
  }
  if (P.tr_prob.size() != P.num_tile_rows) return bad("tr_prob");
  for (uint32_t pr : P.tr_prob)
    if (pr >= P.num_problems) return bad("tr_prob value");
  if (P.chunk_point_begin.back() != npts) return bad("chunks");
  for (size_t c = 0; c + 1 < P.chunk_point_begin.size(); ++c) {
    const uint32_t lo = P.chunk_point_begin[c], hi = P.chunk_point_begin[c + 1];
    if (lo >= hi || hi - lo > 256) return bad("chunk size");
    if (P.point_prob[lo] != P.point_prob[hi - 1]) return bad("chunk spans problems");
  }
  if (P.prob_chunk_begin.size() != P.num_problems + 1u || P.prob_pose_begin.size() != P.num_problems + 1u ||
      P.prob_tr_begin.size() != P.num_problems + 1u)
    return bad("problem ranges");
  return std::string();
}

size_t Plan::device_bytes() const {
  const size_t npose = pose_prob.size(), npt = point_prob.size(), nobs = obs_pose.size();
  size_t b = 0;
  b += npose * (8 * (4 + 3 + 12) * 2 + 8 + 4 + 4);  // state x2, step, slot, prob
  b += npt * (8 * 3 * 2 + 4 + 1 + 4 + 36 + 64 + 96 + 32);  // points x2, off, var, prob, pt_h,
                                                           // pt_s, pt_c, pt_p
  b += nobs * (4 * 4 + 16 + 32 + 16);                // point, pose, cam, slot, xy, obs_h, obs_e
  b += obs_w.size() * 8 + obs_kind.size() * (1 + 16 + 4);
  b += cam_obs.size() * 8 + (pairs_on_device ? num_pairs : pairs.size()) * 12 + dup_pairs.size() * 8;
  b += blk_dst.size() * (8 + 4 + 32);
  b += tile_ij.size() * ((size_t)tb * tb * kBlock * 4 + 4 + 2 * (size_t)tb * 6 * 4);
  b += (size_t)num_var_cams * (4 + 4 + 4 + 4 + 36 * 4 + 6 * 4 * 6);
  b += tr_list.size() * 4 + (size_t)num_tile_rows * (4 + 4 + 16 * 8);
  b += chunk_point_begin.size() * (4 + 8 + 8 + 8);
  b += cameras.size() * sizeof(DevCamera);
  return b;
}

size_t Plan::upload_bytes() const {
  auto b = [](const auto& v) { return v.size() * sizeof(v[0]); };
  return b(prob_pose_begin) + b(prob_point_begin) + b(prob_tr_begin) + b(prob_chunk_begin) +
         b(pose_prob) + b(point_prob) + b(slot_prob) + b(params) + b(pose_q) + b(pose_t) +
         b(points) + b(pose_slot) + b(point_var) + b(cameras) + b(pt_off) + b(obs_point) + b(obs_pose) +
         b(obs_cam) + b(obs_slot) + b(obs_xy) + b(obs_w) + b(obs_kind) + b(obs_st) + b(obs_rcam) +
         b(cam_off) + b(cam_obs) + b(tile_ij) +
         b(blk_off) + b(pairs) + b(blk_dst) + b(diag_dst) + b(dup_off) + b(dup_pairs) +
         b(tr_list_off) + b(tr_list) + b(tr_prob) + b(chunk_point_begin) + b(tile_slot) + b(tile_meta) +
         b(row_blk) + b(blk_col);
}

double algorithmic_bytes(const Plan& P, double k, double* b_pcg_out) {
  // Counts of the byte model: N_o variable observations, N_p variable
  // points, N_c variable cameras, N_e camera pairs sharing a variable point.
  const double No = (double)P.var_obs, Np = (double)P.var_points,
               Nc = (double)P.real_var_cams, Ne = (double)P.camera_pairs;
  const double b_lin = 88.0 * No + 48.0 * Np + 156.0 * Nc;
  const double b_asm = 72.0 * No + 84.0 * Np + 144.0 * Ne + 168.0 * Nc;
  const double b_pcg = 148.0 * Ne + 288.0 * Nc;
  const double b_bs = 76.0 * No + 60.0 * Np;
  const double b_cost = 16.0 * No + 36.0 * Np + 96.0 * Nc;
  if (b_pcg_out) *b_pcg_out = b_pcg;
  return b_lin + b_asm + k * b_pcg + b_bs + b_cost;
}

std::string build_elimination_index(uint32_t n, const uint32_t* edges, uint64_t ne,
                                    uint32_t num_points, const uint64_t* point_off,
                                    const uint32_t* point_nodes, ElimIndex* out) {
  ElimIndex& X = *out;
  X = ElimIndex();
  X.n = n;
  X.num_points = num_points;
  X.num_edges = ne;
  if (ne >= (1ull << 31)) return "too many edges";
  if (point_off[0] != 0) return "point_off[0] is not 0";
  const uint64_t nobs = point_off[num_points];
  if (nobs >= (1ull << 32)) return "too many camera-point blocks";
  X.num_obs = nobs;
  // Edges: ascending, s < t < n; each node's range.
  X.row_off.assign((size_t)n + 1, 0);
  X.edge_t.resize(ne);
  for (uint64_t e = 0; e < ne; ++e) {
    const uint32_t s = edges[2 * e], t = edges[2 * e + 1];
    if (!(s < t && t < n)) return "edge " + std::to_string(e) + " is not (s, t) with s < t < n";
    if (e && (s < edges[2 * e - 2] || (s == edges[2 * e - 2] && t <= edges[2 * e - 1])))
      return "edges are not sorted at " + std::to_string(e);
    X.edge_t[e] = t;
    ++X.row_off[s + 1];
  }
  for (uint32_t s = 0; s < n; ++s) X.row_off[s + 1] += X.row_off[s];
  const uint32_t T = std::max(1u, std::min<uint32_t>(std::thread::hardware_concurrency(), 64u));
  auto plo = [&](uint32_t t) { return (uint32_t)((uint64_t)num_points * t / T); };
  // Each point's nodes checked; its blocks' point.
  X.obs_point.resize(nobs);
  X.point_off.resize((size_t)num_points + 1);
  std::vector<std::string> err(T);
  run_threads(T, [&](uint32_t t) {
    for (uint32_t p = plo(t); p < plo(t + 1) && err[t].empty(); ++p) {
      const uint64_t a = point_off[p], b = point_off[p + 1];
      if (b < a || b > nobs) {
        err[t] = "point_off is not ascending at point " + std::to_string(p);
        break;
      }
      X.point_off[p] = (uint32_t)a;
      for (uint64_t i = a; i < b; ++i) {
        if (point_nodes[i] >= n || (i > a && point_nodes[i] <= point_nodes[i - 1])) {
          err[t] = "nodes of point " + std::to_string(p) + " are not ascending below n";
          break;
        }
        X.obs_point[i] = p;
      }
    }
  });
  for (auto& e : err)
    if (!e.empty()) return e;
  X.point_off[num_points] = (uint32_t)nobs;
  // Per node, its blocks in index (= point) order: a stable counting sort.
  X.slot_obs.resize(nobs);
  X.slot_off.resize((size_t)n + 1);
  counting_sort((uint32_t)nobs, n, T, [&](uint32_t i) { return point_nodes[i]; }, 0u,
                X.slot_obs.data(), X.slot_off.data());
  return "";
}

}  // namespace vlba
