// ba_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the reference's bundle-adjustment
// Levenberg-Marquardt solve (MarvinSt/visloc-rs), used as the checker for the
// CUDA solver and as the timed CPU baseline.  Nothing in the product links or
// calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load the shared library built from it.
//
// The reference is Rust (no Rust toolchain exists here), so it cannot be
// compiled or imported; this file restates its algorithm step by step:
//   LM control and gates ........ pipelines/slam/src/bundle/lm.rs:162-1017
//   validation .................. lm.rs:168-229
//   variable slots .............. lm.rs:234-249
//   normal equations (mono) ..... bundle/normal_equations.rs:421-493
//   normal equations (rig) ...... normal_equations.rs:618-660,
//                                 rig_residual_jacobians sqrt_qr.rs:960-1001
//   projection + Jacobian ....... bundle/jacobians.rs:18-124
//   Schur reduction (sparse) .... normal_equations.rs:1621-1733
//   dense solve (Cholesky->LU) .. pipelines/slam/src/pose_graph.rs:2259-2270
//   landmark-only step .......... normal_equations.rs:1332-1371
//   robust kernels .............. pose_graph.rs:87-138
//   cost / non-projectable ...... bundle/problem.rs:252-304, 497-560
//   SE3 exp / compose ........... crates/core/src/geometry/se3.rs:32-121
//   Camera::project ............. crates/core/src/types/camera.rs:351-432
//   quaternion arithmetic ....... nalgebra 0.33.3 (UnitQuaternion *, transform,
//                                 from_scaled_axis, to_rotation_matrix)
//   reduced-camera PCG .......... colmap_incremental/rig_ba_solver.rs:1406-1480
//                                 (pcg_core, with edge_product :1314-1331 and
//                                 the run and coarse preconditioners)
//   matrix-free LM backend ...... bundle/implicit_schur.rs:108-300 (operator,
//                                 block-Jacobi), :302-376 (cluster8), :390-473
//                                 (apply, preconditioner), :522-736 (PCG),
//                                 :789-828 (complete_delta); step dispatch
//                                 bundle/matrix_free.rs:1106-1190, entry
//                                 bundle/optimize.rs:105-139
//
// Parallel loops (OpenMP) never change a result: every accumulator is owned by
// one thread and visited in the serial order, as the reference's rayon paths
// guarantee (bundle/mod.rs:22-70).  Compiled with -ffp-contract=off so no
// multiply-add is fused, matching Rust's arithmetic, except where the
// reference itself fuses (edge_product's mul_add, restated with std::fma).

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/visloc_ba_cuda.h"

namespace {

// ------------------------------------------------------------ small algebra
struct Quat { double w, i, j, k; };
struct V3 { double x, y, z; };

inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
inline V3 cross(const V3& a, const V3& b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// nalgebra UnitQuaternion::to_rotation_matrix (row-major result).
void quat_to_matrix(const Quat& q, double m[9]) {
  const double i = q.i, j = q.j, k = q.k, w = q.w;
  const double ww = w * w, ii = i * i, jj = j * j, kk = k * k;
  const double ij = i * j * 2.0, wk = w * k * 2.0, wj = w * j * 2.0;
  const double ik = i * k * 2.0, jk = j * k * 2.0, wi = w * i * 2.0;
  m[0] = ww + ii - jj - kk; m[1] = ij - wk;           m[2] = wj + ik;
  m[3] = wk + ij;           m[4] = ww - ii + jj - kk; m[5] = jk - wi;
  m[6] = ik - wj;           m[7] = wi + jk;           m[8] = ww - ii - jj + kk;
}

// nalgebra UnitQuaternion * Vector3: t = 2 (v x p); p + w t + v x t.
V3 quat_rotate(const Quat& q, const V3& p) {
  const V3 v = v3(q.i, q.j, q.k);
  V3 t = cross(v, p);
  t = v3(t.x * 2.0, t.y * 2.0, t.z * 2.0);
  const V3 c = cross(v, t);
  return v3(t.x * q.w + c.x + p.x, t.y * q.w + c.y + p.y, t.z * q.w + c.z + p.z);
}

// Hamilton product a * b.
Quat quat_mul(const Quat& a, const Quat& b) {
  return Quat{a.w * b.w - a.i * b.i - a.j * b.j - a.k * b.k,
              a.w * b.i + a.i * b.w + a.j * b.k - a.k * b.j,
              a.w * b.j - a.i * b.k + a.j * b.w + a.k * b.i,
              a.w * b.k + a.i * b.j - a.j * b.i + a.k * b.w};
}

// UnitQuaternion::from_scaled_axis = exp(Quaternion::from_imag(w / 2)).
Quat quat_from_scaled_axis(const V3& w) {
  const V3 h = v3(w.x / 2.0, w.y / 2.0, w.z / 2.0);
  const double nn = h.x * h.x + h.y * h.y + h.z * h.z;
  const double eps = std::numeric_limits<double>::epsilon();
  if (nn <= eps * eps) return Quat{1.0, 0.0, 0.0, 0.0};
  const double n = std::sqrt(nn);
  const double s = std::sin(n) / n;
  return Quat{std::cos(n), h.x * s, h.y * s, h.z * s};
}

void skew(const V3& v, double m[9]) {
  m[0] = 0.0;  m[1] = -v.z; m[2] = v.y;
  m[3] = v.z;  m[4] = 0.0;  m[5] = -v.x;
  m[6] = -v.y; m[7] = v.x;  m[8] = 0.0;
}

void mat3_mul(const double a[9], const double b[9], double c[9]) {
  for (int r = 0; r < 3; ++r)
    for (int col = 0; col < 3; ++col) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += a[r * 3 + k] * b[k * 3 + col];
      c[r * 3 + col] = s;
    }
}

// so3_left_jacobian (se3.rs:109-121).
void so3_left_jacobian(const V3& w, double v[9]) {
  const double theta_sq = w.x * w.x + w.y * w.y + w.z * w.z;
  double s[9], s2[9];
  skew(w, s);
  mat3_mul(s, s, s2);
  double a, b;
  if (theta_sq < 1e-10) {
    a = 0.5;
    b = 1.0 / 6.0;
  } else {
    const double theta = std::sqrt(theta_sq);
    a = (1.0 - std::cos(theta)) / theta_sq;
    b = (theta - std::sin(theta)) / (theta * theta_sq);
  }
  for (int e = 0; e < 9; ++e) v[e] = (e % 4 == 0 ? 1.0 : 0.0) + a * s[e] + b * s2[e];
}

struct Se3 { Quat q; V3 t; };

// SE3::exp (se3.rs:72-82), tangent [rho; omega].
Se3 se3_exp(const double xi[6]) {
  const V3 rho = v3(xi[0], xi[1], xi[2]);
  const V3 omega = v3(xi[3], xi[4], xi[5]);
  Se3 out;
  out.q = quat_from_scaled_axis(omega);
  double v[9];
  so3_left_jacobian(omega, v);
  out.t = v3(v[0] * rho.x + v[1] * rho.y + v[2] * rho.z,
             v[3] * rho.x + v[4] * rho.y + v[5] * rho.z,
             v[6] * rho.x + v[7] * rho.y + v[8] * rho.z);
  return out;
}

// SE3::compose (se3.rs:32-37): self * other.
Se3 se3_compose(const Se3& a, const Se3& b) {
  Se3 out;
  out.q = quat_mul(a.q, b.q);
  const V3 r = quat_rotate(a.q, b.t);
  out.t = v3(r.x + a.t.x, r.y + a.t.y, r.z + a.t.z);
  return out;
}

V3 se3_transform(const Se3& T, const V3& p) {
  const V3 r = quat_rotate(T.q, p);
  return v3(r.x + T.t.x, r.y + T.t.y, r.z + T.t.z);
}

// -------------------------------------------------------------- cameras
struct Cam {
  double fx, fy, cx, cy, k1, k2;
  bool radial;        // MonoProjection::Radial (k1 or k2 nonzero)
  bool rig;           // observation carries sensor_from_rig
  Se3 sensor_from_rig;
};

// Camera::intrinsics / radial_distortion (camera.rs:213-260) restricted to
// the radial pinhole family; false for any other model (the reference admits
// them through Camera::project_with_point_jacobian, which this restatement,
// like the CUDA solver, does not cover).
bool resolve_camera(const vlba_camera& c, Cam* out) {
  const double* p = c.params;
  const uint32_t n = c.num_params;
  double fx, fy, cx, cy, k1 = 0.0, k2 = 0.0;
  bool has_radial = false;
  switch (c.model) {
    case VLBA_CAMERA_PINHOLE:
      if (n < 4) return false;
      fx = p[0]; fy = p[1]; cx = p[2]; cy = p[3];
      if (n >= 5) { has_radial = true; k1 = p[4]; k2 = n >= 6 ? p[5] : 0.0; }
      break;
    case VLBA_CAMERA_OPENCV:
      if (n < 4) return false;
      fx = p[0]; fy = p[1]; cx = p[2]; cy = p[3];
      if ((n >= 7 && p[6] != 0.0) || (n >= 8 && p[7] != 0.0)) return false;  // tangential
      if (n >= 5) { has_radial = true; k1 = p[4]; k2 = n >= 6 ? p[5] : 0.0; }
      break;
    case VLBA_CAMERA_SIMPLE_PINHOLE:
      if (n < 3) return false;
      fx = fy = p[0]; cx = p[1]; cy = p[2];
      break;
    case VLBA_CAMERA_SIMPLE_RADIAL:
      if (n < 3) return false;
      fx = fy = p[0]; cx = p[1]; cy = p[2];
      if (n >= 4) { has_radial = true; k1 = p[3]; k2 = 0.0; }
      break;
    case VLBA_CAMERA_RADIAL:
      if (n < 3) return false;
      fx = fy = p[0]; cx = p[1]; cy = p[2];
      if (n >= 4) { has_radial = true; k1 = p[3]; k2 = n >= 5 ? p[4] : 0.0; }
      break;
    default:
      return false;
  }
  out->fx = fx; out->fy = fy; out->cx = cx; out->cy = cy;
  out->k1 = k1; out->k2 = k2;
  out->radial = has_radial && (k1 != 0.0 || k2 != 0.0);
  out->sensor_from_rig.q = Quat{c.sensor_from_rig_q[0], c.sensor_from_rig_q[1],
                                c.sensor_from_rig_q[2], c.sensor_from_rig_q[3]};
  out->sensor_from_rig.t = v3(c.sensor_from_rig_t[0], c.sensor_from_rig_t[1],
                              c.sensor_from_rig_t[2]);
  out->rig = false;
  return true;
}

// Camera::project for the radial pinhole family (camera.rs:351-432).
bool camera_project(const Cam& c, const V3& p, double out[2]) {
  if (!(std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z))) return false;
  if (p.z <= 0.0) return false;
  double x = p.x / p.z;
  double y = p.y / p.z;
  if (c.radial) {
    const double r2 = x * x + y * y;
    const double d = 1.0 + c.k1 * r2 + c.k2 * r2 * r2;
    x *= d;
    y *= d;
  }
  out[0] = c.fx * x + c.cx;
  out[1] = c.fy * y + c.cy;
  return true;
}

// mono_project_with_jacobian (jacobians.rs:63-113); j is row-major 2x3.
bool mono_project_with_jacobian(const Cam& c, const V3& xc, double pred[2], double j[6]) {
  if (xc.z <= 0.0) return false;
  if (!c.radial) {
    // project_pinhole (jacobians.rs:115-124) + the closed-form J_pi.
    pred[0] = c.fx * xc.x / xc.z + c.cx;
    pred[1] = c.fy * xc.y / xc.z + c.cy;
    const double z_inv = 1.0 / xc.z;
    j[0] = c.fx * z_inv;
    j[1] = 0.0;
    j[2] = -c.fx * xc.x * z_inv * z_inv;
    j[3] = 0.0;
    j[4] = c.fy * z_inv;
    j[5] = -c.fy * xc.y * z_inv * z_inv;
    return true;
  }
  const double x = xc.x / xc.z;
  const double y = xc.y / xc.z;
  const double r2 = x * x + y * y;
  const double d = 1.0 + c.k1 * r2 + c.k2 * r2 * r2;
  pred[0] = c.fx * (x * d) + c.cx;
  pred[1] = c.fy * (y * d) + c.cy;
  const double g = c.k1 + 2.0 * c.k2 * r2;
  const double d11 = d + 2.0 * x * x * g;
  const double d12 = 2.0 * x * y * g;
  const double d22 = d + 2.0 * y * y * g;
  const double z_inv = 1.0 / xc.z;
  j[0] = c.fx * d11 * z_inv;
  j[1] = c.fx * d12 * z_inv;
  j[2] = -c.fx * (d11 * x + d12 * y) * z_inv;
  j[3] = c.fy * d12 * z_inv;
  j[4] = c.fy * d22 * z_inv;
  j[5] = -c.fy * (d12 * x + d22 * y) * z_inv;
  for (int e = 0; e < 2; ++e)
    if (!std::isfinite(pred[e])) return false;
  for (int e = 0; e < 6; ++e)
    if (!std::isfinite(j[e])) return false;
  return true;
}

// ---------------------------------------------------------- robust kernels
struct Kernel {
  uint32_t kind;
  double p;
  // RobustKernel::cost (pose_graph.rs:103-120).
  double cost(double s) const {
    if (kind == VLBA_KERNEL_HUBER) {
      const double dsq = p * p;
      return s <= dsq ? s : 2.0 * p * std::sqrt(s) - dsq;
    }
    if (kind == VLBA_KERNEL_CAUCHY) {
      const double csq = p * p;
      return csq * std::log(1.0 + s / csq);
    }
    return s;
  }
  // RobustKernel::weight (pose_graph.rs:122-138).
  double weight(double s) const {
    if (kind == VLBA_KERNEL_HUBER) {
      const double dsq = p * p;
      return s <= dsq ? 1.0 : p / std::sqrt(s);
    }
    if (kind == VLBA_KERNEL_CAUCHY) {
      const double csq = p * p;
      return 1.0 / (1.0 + s / csq);
    }
    return 1.0;
  }
};

// ------------------------------------------------------------ the problem
struct Problem {
  const vlba_problem* p;
  std::vector<Cam> cams;
  bool per_obs_camera;
  std::vector<Se3> poses;
  std::vector<V3> points;
  Kernel kernel;

  const Cam& cam_of(size_t o) const {
    return per_obs_camera ? cams[p->obs_camera[o]] : cams[0];
  }
};

int threads_or_default(int threads) {
#ifdef _OPENMP
  return threads > 0 ? threads : omp_get_max_threads();
#else
  (void)threads;
  return 1;
#endif
}

// Per-observation residual and Jacobians.  Monocular: normal_equations.rs
// :421-470; rig: rig_residual_jacobians (sqrt_qr.rs:960-1001).
bool residual_jacobians(const Problem& P, size_t o, double r[2], double jp[12], double jl[6]) {
  const uint32_t pi = P.p->obs_pose[o];
  const uint32_t li = P.p->obs_landmark[o];
  const Se3& T = P.poses[pi];
  const V3& X = P.points[li];
  const Cam& c = P.cam_of(o);
  double R[9];
  quat_to_matrix(T.q, R);
  double xs[9];
  skew(X, xs);
  double rxs[9];  // R * [X]x
  mat3_mul(R, xs, rxs);
  double pred[2], jpi[6];
  if (!P.per_obs_camera) {
    const V3 xc = se3_transform(T, X);
    if (xc.z <= 0.0) return false;
    if (!mono_project_with_jacobian(c, xc, pred, jpi)) return false;
    r[0] = pred[0] - P.p->obs_xy[2 * o];
    r[1] = pred[1] - P.p->obs_xy[2 * o + 1];
    // dx_dxi = [R | -R [X]x]; j_pose = j_pi * dx_dxi; j_lm = j_pi * R.
    double dx[18];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        dx[a * 6 + b] = R[a * 3 + b];
        dx[a * 6 + 3 + b] = -rxs[a * 3 + b];
      }
    for (int a = 0; a < 2; ++a) {
      for (int b = 0; b < 6; ++b) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += jpi[a * 3 + k] * dx[k * 6 + b];
        jp[a * 6 + b] = s;
      }
      for (int b = 0; b < 3; ++b) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += jpi[a * 3 + k] * R[k * 3 + b];
        jl[a * 3 + b] = s;
      }
    }
    return true;
  }
  // Rig observation.
  const V3 prig = se3_transform(T, X);
  const V3 ps = se3_transform(c.sensor_from_rig, prig);
  if (!c.radial) {
    if (ps.z <= 0.0) return false;
    pred[0] = c.fx * ps.x / ps.z + c.cx;
    pred[1] = c.fy * ps.y / ps.z + c.cy;
    const double z_inv = 1.0 / ps.z;  // pinhole_projection_jacobian (sqrt_qr.rs:445-463)
    const double z_inv2 = z_inv * z_inv;
    jpi[0] = c.fx * z_inv; jpi[1] = 0.0; jpi[2] = -c.fx * ps.x * z_inv2;
    jpi[3] = 0.0; jpi[4] = c.fy * z_inv; jpi[5] = -c.fy * ps.y * z_inv2;
  } else if (!mono_project_with_jacobian(c, ps, pred, jpi)) {
    return false;
  }
  r[0] = pred[0] - P.p->obs_xy[2 * o];
  r[1] = pred[1] - P.p->obs_xy[2 * o + 1];
  double Rs[9];
  quat_to_matrix(c.sensor_from_rig.q, Rs);
  double drig[18];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      drig[a * 6 + b] = R[a * 3 + b];
      drig[a * 6 + 3 + b] = -rxs[a * 3 + b];
    }
  double pr[6];  // projection * R_sensor<-rig (2x3)
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 3; ++b) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += jpi[a * 3 + k] * Rs[k * 3 + b];
      pr[a * 3 + b] = s;
    }
  for (int a = 0; a < 2; ++a) {
    for (int b = 0; b < 6; ++b) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += pr[a * 3 + k] * drig[k * 6 + b];
      jp[a * 6 + b] = s;
    }
    for (int b = 0; b < 3; ++b) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += pr[a * 3 + k] * R[k * 3 + b];
      jl[a * 3 + b] = s;
    }
  }
  return true;
}

// Stereo observations (vlba_problem.obs_kind 1 and 2): rectified,
// normal_equations.rs:496-570 -- r = (u_l, v_l, u_r) with u_r predicted as
// u_l - fx b / z -- and calibrated general stereo, general_stereo_residual_
// jacobians (sqrt_qr.rs:465-518) -- r = (u_l, v_l, u_r, v_r) with the right
// point T_right<-left x_left.  Both through the pinhole intrinsics of
// BundleAdjustment::camera (cams[0]) and the right camera, no distortion.
// Returns the number of residual rows, 0 when a camera sees the point at
// z <= 0; jp is m x 6, jl m x 3, row-major.
int stereo_residual_jacobians(const Problem& P, size_t o, uint32_t kind, double* r, double* jp,
                              double* jl) {
  const Se3& T = P.poses[P.p->obs_pose[o]];
  const V3& X = P.points[P.p->obs_landmark[o]];
  const Cam& cl = P.cams[0];
  double R[9], xsk[9], rxs[9];
  quat_to_matrix(T.q, R);
  skew(X, xsk);
  mat3_mul(R, xsk, rxs);
  double D[18];  // d x_left / d xi = [R | -R [X]x]
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      D[a * 6 + b] = R[a * 3 + b];
      D[a * 6 + 3 + b] = -rxs[a * 3 + b];
    }
  const V3 xl = se3_transform(T, X);
  if (xl.z <= 0.0) return 0;
  const double* xy = P.p->obs_xy + 2 * o;
  const double* st = P.p->obs_stereo + 2 * o;
  // Rows (u, v) of a pinhole camera at point p: pixel and d/d p.
  auto rows = [](const Cam& c, const V3& p, double* pix, double* j) {
    const double z_inv = 1.0 / p.z, z_inv2 = z_inv * z_inv;
    pix[0] = c.fx * p.x / p.z + c.cx;
    pix[1] = c.fy * p.y / p.z + c.cy;
    j[0] = c.fx * z_inv; j[1] = 0.0; j[2] = -c.fx * p.x * z_inv2;
    j[3] = 0.0; j[4] = c.fy * z_inv; j[5] = -c.fy * p.y * z_inv2;
  };
  double pix[2], jpi[12];  // up to 4 rows of d pixel / d x_left
  rows(cl, xl, pix, jpi);
  r[0] = pix[0] - xy[0];
  r[1] = pix[1] - xy[1];
  int m;
  if (kind == 1) {
    const double b = P.p->stereo_baseline;
    const double z_inv = 1.0 / xl.z;
    r[2] = (pix[0] - cl.fx * b / xl.z) - st[0];
    jpi[6] = cl.fx * z_inv;
    jpi[7] = 0.0;
    jpi[8] = -cl.fx * (xl.x - b) * z_inv * z_inv;
    m = 3;
  } else {
    const Cam& cr = P.cams[P.p->obs_right_camera[o]];
    const V3 xr = se3_transform(cr.sensor_from_rig, xl);
    if (xr.z <= 0.0) return 0;
    double pr[2], jr[6], Rr[9];
    rows(cr, xr, pr, jr);
    r[2] = pr[0] - st[0];
    r[3] = pr[1] - st[1];
    quat_to_matrix(cr.sensor_from_rig.q, Rr);
    for (int a = 0; a < 2; ++a)  // d right pixel / d x_left = j_right Rr
      for (int b = 0; b < 3; ++b) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += jr[a * 3 + k] * Rr[k * 3 + b];
        jpi[6 + a * 3 + b] = s;
      }
    m = 4;
  }
  for (int a = 0; a < m; ++a) {
    for (int b = 0; b < 6; ++b) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += jpi[a * 3 + k] * D[k * 6 + b];
      jp[a * 6 + b] = s;
    }
    for (int b = 0; b < 3; ++b) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += jpi[a * 3 + k] * R[k * 3 + b];
      jl[a * 3 + b] = s;
    }
  }
  return m;
}

// Any observation: its residual rows (2, 3 or 4; 0 = not evaluable).
int obs_residual_jacobians(const Problem& P, size_t o, double* r, double* jp, double* jl) {
  const uint32_t kind = P.p->obs_kind ? P.p->obs_kind[o] : 0u;
  if (kind == 0) return residual_jacobians(P, o, r, jp, jl) ? 2 : 0;
  return stereo_residual_jacobians(P, o, kind, r, jp, jl);
}

// robust_cost_weighted + nonprojectable_observation_count (problem.rs:252-304,
// 497-560): cost over projectable observations, count of the others.
void cost_and_nonprojectable(const Problem& P, int threads, double* cost, uint64_t* bad) {
  const size_t n = P.p->num_observations;
  const size_t chunk = 4096;
  const size_t nchunks = (n + chunk - 1) / chunk;
  std::vector<double> part(nchunks, 0.0);
  std::vector<uint64_t> partbad(nchunks, 0);
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long long ci = 0; ci < (long long)nchunks; ++ci) {
    double s = 0.0;
    uint64_t b = 0;
    const size_t lo = (size_t)ci * chunk, hi = std::min(n, lo + chunk);
    for (size_t o = lo; o < hi; ++o) {
      if (P.p->obs_kind && P.p->obs_kind[o] != 0) {
        // Stereo: robust cost of the squared norm of its residual rows.
        double r[4], jp[24], jl[12];
        const int m = obs_residual_jacobians(P, o, r, jp, jl);
        if (!m) {
          ++b;
          continue;
        }
        double ss = 0.0;
        for (int i = 0; i < m; ++i) ss += r[i] * r[i];
        const double rc = P.kernel.cost(ss);
        s += P.p->obs_weight ? P.p->obs_weight[o] * rc : rc;
        continue;
      }
      const Se3& T = P.poses[P.p->obs_pose[o]];
      const V3& X = P.points[P.p->obs_landmark[o]];
      const Cam& c = P.cam_of(o);
      V3 xc = se3_transform(T, X);
      if (P.per_obs_camera) xc = se3_transform(c.sensor_from_rig, xc);
      double pred[2];
      if (xc.z <= 0.0 || !camera_project(c, xc, pred)) {
        ++b;
        continue;
      }
      const double rx = pred[0] - P.p->obs_xy[2 * o];
      const double ry = pred[1] - P.p->obs_xy[2 * o + 1];
      // w * kernel.cost(s), the external weight 1 when absent (problem.rs:547-548).
      const double rc = P.kernel.cost(rx * rx + ry * ry);
      s += P.p->obs_weight ? P.p->obs_weight[o] * rc : rc;
    }
    part[ci] = s;
    partbad[ci] = b;
  }
  double total = 0.0;
  uint64_t tb = 0;
  for (size_t ci = 0; ci < nchunks; ++ci) {
    total += part[ci];
    tb += partbad[ci];
  }
  *cost = total;
  *bad = tb;
}

// ------------------------------------------------------- dense factorisation
// In-place Cholesky of the symmetric n x n row-major matrix `a` (lower
// triangle used).  Blocked right-looking; trailing updates in parallel.
bool cholesky(std::vector<double>& a, size_t n, int threads) {
  const size_t nb = 48;
  for (size_t k0 = 0; k0 < n; k0 += nb) {
    const size_t k1 = std::min(n, k0 + nb);
    // Factor the diagonal block.
    for (size_t j = k0; j < k1; ++j) {
      double s = a[j * n + j];
      for (size_t q = k0; q < j; ++q) s -= a[j * n + q] * a[j * n + q];
      if (!(s > 0.0) || !std::isfinite(s)) return false;
      const double ljj = std::sqrt(s);
      a[j * n + j] = ljj;
      for (size_t i = j + 1; i < k1; ++i) {
        double t = a[i * n + j];
        for (size_t q = k0; q < j; ++q) t -= a[i * n + q] * a[j * n + q];
        a[i * n + j] = t / ljj;
      }
    }
    // Panel below the diagonal block.
#pragma omp parallel for schedule(static) num_threads(threads)
    for (long long ii = (long long)k1; ii < (long long)n; ++ii) {
      const size_t i = (size_t)ii;
      for (size_t j = k0; j < k1; ++j) {
        double t = a[i * n + j];
        for (size_t q = k0; q < j; ++q) t -= a[i * n + q] * a[j * n + q];
        a[i * n + j] = t / a[j * n + j];
      }
    }
    // Trailing update A22 -= L21 L21^T (lower triangle).
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (long long ii = (long long)k1; ii < (long long)n; ++ii) {
      const size_t i = (size_t)ii;
      const double* li = &a[i * n + k0];
      for (size_t j = k1; j <= i; ++j) {
        const double* lj = &a[j * n + k0];
        double t = 0.0;
        for (size_t q = 0; q < k1 - k0; ++q) t += li[q] * lj[q];
        a[i * n + j] -= t;
      }
    }
  }
  return true;
}

void cholesky_solve(const std::vector<double>& l, size_t n, std::vector<double>& x) {
  for (size_t i = 0; i < n; ++i) {
    double s = x[i];
    for (size_t q = 0; q < i; ++q) s -= l[i * n + q] * x[q];
    x[i] = s / l[i * n + i];
  }
  for (size_t ii = n; ii-- > 0;) {
    double s = x[ii];
    for (size_t q = ii + 1; q < n; ++q) s -= l[q * n + ii] * x[q];
    x[ii] = s / l[ii * n + ii];
  }
}

// LU with partial pivoting (nalgebra's lu().solve fallback); false if singular.
bool lu_solve(std::vector<double> a, size_t n, std::vector<double>& x) {
  std::vector<size_t> piv(n);
  for (size_t k = 0; k < n; ++k) {
    size_t p = k;
    double best = std::fabs(a[k * n + k]);
    for (size_t i = k + 1; i < n; ++i)
      if (std::fabs(a[i * n + k]) > best) { best = std::fabs(a[i * n + k]); p = i; }
    if (best == 0.0) return false;
    piv[k] = p;
    if (p != k) {
      for (size_t c = 0; c < n; ++c) std::swap(a[k * n + c], a[p * n + c]);
      std::swap(x[k], x[p]);
    }
    const double inv = 1.0 / a[k * n + k];
    for (size_t i = k + 1; i < n; ++i) {
      const double f = a[i * n + k] * inv;
      a[i * n + k] = f;
      for (size_t c = k + 1; c < n; ++c) a[i * n + c] -= f * a[k * n + c];
      x[i] -= f * x[k];
    }
  }
  for (size_t ii = n; ii-- > 0;) {
    double s = x[ii];
    for (size_t c = ii + 1; c < n; ++c) s -= a[ii * n + c] * x[c];
    x[ii] = s / a[ii * n + ii];
  }
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}

// nalgebra Matrix3::try_inverse: cofactor inverse, None when det == 0.
bool try_inverse3(const double m[9], double inv[9]) {
  const double m11 = m[0], m12 = m[1], m13 = m[2];
  const double m21 = m[3], m22 = m[4], m23 = m[5];
  const double m31 = m[6], m32 = m[7], m33 = m[8];
  const double minor_m12_m23 = m22 * m33 - m32 * m23;
  const double minor_m11_m23 = m21 * m33 - m31 * m23;
  const double minor_m11_m22 = m21 * m32 - m31 * m22;
  const double det = m11 * minor_m12_m23 - m12 * minor_m11_m23 + m13 * minor_m11_m22;
  if (det == 0.0) return false;
  inv[0] = minor_m12_m23 / det;
  inv[1] = (m13 * m32 - m33 * m12) / det;
  inv[2] = (m12 * m23 - m22 * m13) / det;
  inv[3] = -minor_m11_m23 / det;
  inv[4] = (m11 * m33 - m31 * m13) / det;
  inv[5] = (m13 * m21 - m23 * m11) / det;
  inv[6] = minor_m11_m22 / det;
  inv[7] = (m12 * m31 - m32 * m11) / det;
  inv[8] = (m11 * m22 - m21 * m12) / det;
  return true;
}

// ------------------------------------------------------- normal equations
struct Cross { uint32_t pose; double a[18]; };  // 6x3 row-major

struct Normal {
  std::vector<double> h_pp;   // 36 per variable pose
  std::vector<double> b_p;    // 6 per variable pose
  std::vector<double> h_ll;   // 9 per variable landmark
  std::vector<double> b_l;    // 3 per variable landmark
  std::vector<std::vector<Cross>> cross;  // per variable landmark
};

struct Slots {
  std::vector<int64_t> pose_slot;  // -1: fixed
  std::vector<int64_t> lm_slot;
  std::vector<uint32_t> var_poses, var_lms;
};

void build_slots(const vlba_problem* p, Slots* s) {
  s->pose_slot.assign(p->num_poses, -1);
  s->lm_slot.assign(p->num_landmarks, -1);
  for (uint64_t i = 0; i < p->num_poses; ++i)
    if (!(p->pose_fixed && p->pose_fixed[i])) {
      s->pose_slot[i] = (int64_t)s->var_poses.size();
      s->var_poses.push_back((uint32_t)i);
    }
  for (uint64_t i = 0; i < p->num_landmarks; ++i)
    if (!(p->landmark_fixed && p->landmark_fixed[i])) {
      s->lm_slot[i] = (int64_t)s->var_lms.size();
      s->var_lms.push_back((uint32_t)i);
    }
}

// build_normal_equations (normal_equations.rs:352-493, 618-660): per-obs
// contributions computed in parallel, accumulated by owner in obs order.
void build_normal(const Problem& P, const Slots& S, int threads, Normal* N) {
  const size_t np = S.var_poses.size(), nl = S.var_lms.size();
  const size_t no = P.p->num_observations;
  N->h_pp.assign(np * 36, 0.0);
  N->b_p.assign(np * 6, 0.0);
  N->h_ll.assign(nl * 9, 0.0);
  N->b_l.assign(nl * 3, 0.0);
  N->cross.assign(nl, {});
  struct Contrib { double r[4], jp[24], jl[12], w; int m; bool ok; };
  std::vector<Contrib> c(no);
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long long oo = 0; oo < (long long)no; ++oo) {
    Contrib& k = c[oo];
    k.m = obs_residual_jacobians(P, (size_t)oo, k.r, k.jp, k.jl);
    k.ok = k.m > 0;
    // kernel.weight(s) * the external weight (normal_equations.rs:458).
    if (k.ok) {
      double s = 0.0;
      for (int i = 0; i < k.m; ++i) s += k.r[i] * k.r[i];
      k.w = P.kernel.weight(s);
      if (P.p->obs_weight) k.w *= P.p->obs_weight[oo];
    }
  }
  // Pose blocks: each thread owns poses p with p % nt == tid.
#pragma omp parallel num_threads(threads)
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num(), nt = omp_get_num_threads();
#else
    const int tid = 0, nt = 1;
#endif
    for (size_t o = 0; o < no; ++o) {
      const Contrib& k = c[o];
      if (!k.ok) continue;
      const int64_t ps = S.pose_slot[P.p->obs_pose[o]];
      if (ps >= 0 && (ps % nt) == tid) {
        double* h = &N->h_pp[ps * 36];
        double* b = &N->b_p[ps * 6];
        for (int rr = 0; rr < 6; ++rr) {
          for (int cc = 0; cc < 6; ++cc) {
            double v = 0.0;
            for (int i = 0; i < k.m; ++i) v += k.jp[6 * i + rr] * k.jp[6 * i + cc];
            h[rr * 6 + cc] += k.w * v;
          }
          double g = 0.0;
          for (int i = 0; i < k.m; ++i) g += k.jp[6 * i + rr] * k.r[i];
          b[rr] += k.w * g;
        }
      }
      const int64_t ls = S.lm_slot[P.p->obs_landmark[o]];
      if (ls >= 0 && (ls % nt) == tid) {
        double* h = &N->h_ll[ls * 9];
        double* b = &N->b_l[ls * 3];
        for (int rr = 0; rr < 3; ++rr) {
          for (int cc = 0; cc < 3; ++cc) {
            double v = 0.0;
            for (int i = 0; i < k.m; ++i) v += k.jl[3 * i + rr] * k.jl[3 * i + cc];
            h[rr * 3 + cc] += k.w * v;
          }
          double g = 0.0;
          for (int i = 0; i < k.m; ++i) g += k.jl[3 * i + rr] * k.r[i];
          b[rr] += k.w * g;
        }
        if (ps >= 0) {
          Cross x;
          x.pose = (uint32_t)ps;
          for (int rr = 0; rr < 6; ++rr)
            for (int cc = 0; cc < 3; ++cc) {
              double v = 0.0;
              for (int i = 0; i < k.m; ++i) v += k.jp[6 * i + rr] * k.jl[3 * i + cc];
              x.a[rr * 3 + cc] = k.w * v;
            }
          N->cross[ls].push_back(x);
        }
      }
    }
  }
}

// The reduced camera system S = D + lambda I - sum_l A H^-1 B^T (lower
// blocks, mirrored), rhs = -b_p + sum_l A H^-1 b_l, as
// solve_step_pose_blocks_with_debug (normal_equations.rs:1621-1700).
void reduce(const Normal& N, size_t np, size_t nl, double lambda, int threads,
            std::vector<double>& s, std::vector<double>& rhs,
            std::vector<uint8_t>& inv_ok, std::vector<double>& hinv) {
  const size_t dim = np * 6;
  s.assign(dim * dim, 0.0);
  rhs.assign(dim, 0.0);
  for (size_t p = 0; p < np; ++p) {
    for (int rr = 0; rr < 6; ++rr)
      for (int cc = 0; cc < 6; ++cc) {
        double v = N.h_pp[p * 36 + rr * 6 + cc];
        if (rr == cc && lambda > 0.0) v += lambda;
        s[(p * 6 + rr) * dim + p * 6 + cc] = v;
      }
    for (int k = 0; k < 6; ++k) rhs[p * 6 + k] = -N.b_p[p * 6 + k];
  }
  inv_ok.assign(nl, 0);
  hinv.assign(nl * 9, 0.0);
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long long ll = 0; ll < (long long)nl; ++ll) {
    double h[9];
    std::memcpy(h, &N.h_ll[ll * 9], sizeof h);
    if (lambda > 0.0) { h[0] += lambda; h[4] += lambda; h[8] += lambda; }
    inv_ok[ll] = try_inverse3(h, &hinv[ll * 9]) ? 1 : 0;
  }
#pragma omp parallel num_threads(threads)
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num(), nt = omp_get_num_threads();
#else
    const int tid = 0, nt = 1;
#endif
    for (size_t l = 0; l < nl; ++l) {
      if (!inv_ok[l]) continue;
      const double* hi = &hinv[l * 9];
      const std::vector<Cross>& cr = N.cross[l];
      for (const Cross& a : cr) {
        if ((int)(a.pose % nt) != tid) continue;
        double ah[18];
        for (int rr = 0; rr < 6; ++rr)
          for (int cc = 0; cc < 3; ++cc) {
            double t = 0.0;
            for (int k = 0; k < 3; ++k) t += a.a[rr * 3 + k] * hi[k * 3 + cc];
            ah[rr * 3 + cc] = t;
          }
        for (const Cross& b : cr) {
          if (a.pose < b.pose) continue;
          double* dst = &s[(size_t)a.pose * 6 * dim + (size_t)b.pose * 6];
          for (int rr = 0; rr < 6; ++rr)
            for (int cc = 0; cc < 6; ++cc) {
              double t = 0.0;
              for (int k = 0; k < 3; ++k) t += ah[rr * 3 + k] * b.a[cc * 3 + k];
              dst[rr * dim + cc] -= t;
            }
        }
        const double* bl = &N.b_l[l * 3];
        for (int k = 0; k < 6; ++k) {
          double t = 0.0;
          for (int q = 0; q < 3; ++q) t += ah[k * 3 + q] * bl[q];
          rhs[a.pose * 6 + k] += t;
        }
      }
    }
  }
  // Mirror the lower block triangle.
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long long ii = 0; ii < (long long)dim; ++ii)
    for (size_t j = (size_t)ii + 1; j < dim; ++j) {
      const size_t bi = (size_t)ii / 6, bj = j / 6;
      if (bj > bi) s[(size_t)ii * dim + j] = s[j * dim + (size_t)ii];
    }
}

// ----------------------------------------------------- banded sparse solve
// LinearSolver::Sparse on a reduced system whose blocks lie in a band (a
// street loop: covisible cameras are near each other along the capture
// order, and the loop closes back to the start).  The reference factors S
// with a block Cholesky in a fill-reducing order (block_cholesky.rs:13-120,
// 250-310, order from reordering.rs); any symmetric order gives the same
// solution up to rounding, and here it is a bandwidth-reducing one: the
// capture order, or the "fold" order 0, n-1, 1, n-2, ... that turns a closed
// loop's cyclic band into a plain band of twice the width.  S's lower band
// is stored row-major, W + 1 scalars per row (W = 6 w + 5 for a block
// half-bandwidth w), and factored in place column by column.
struct Band {
  size_t n = 0, W = 0;
  std::vector<uint32_t> pos;  // permuted position of each variable pose
  std::vector<double> a;      // [n (W + 1)]: entry (i, j), i - W <= j <= i, at i (W+1) + j - i + W
  double& at(size_t i, size_t j) { return a[i * (W + 1) + j + W - i]; }
  double at(size_t i, size_t j) const { return a[i * (W + 1) + j + W - i]; }
};

// Block half-bandwidth of the reduced system under `pos`: the largest
// |pos(i) - pos(j)| over camera pairs that share a landmark with an inverse.
size_t band_width(const Normal& N, const std::vector<uint8_t>& ok, const std::vector<uint32_t>& pos) {
  size_t w = 0;
  for (size_t l = 0; l < N.cross.size(); ++l) {
    if (!ok[l] || N.cross[l].empty()) continue;
    uint32_t lo = ~0u, hi = 0;
    for (const Cross& c : N.cross[l]) {
      lo = std::min(lo, pos[c.pose]);
      hi = std::max(hi, pos[c.pose]);
    }
    w = std::max(w, (size_t)(hi - lo));
  }
  return w;
}

// The damped reduced system in band storage and its rhs (original pose
// order), with the block order of smaller bandwidth; false when even that
// band is wider than a third of the system (then the dense path is cheaper).
bool reduce_banded(const Normal& N, size_t np, size_t nl, double lambda, int threads, Band& B,
                   std::vector<double>& rhs, std::vector<uint8_t>& inv_ok,
                   std::vector<double>& hinv) {
  inv_ok.assign(nl, 0);
  hinv.assign(nl * 9, 0.0);
  for (size_t l = 0; l < nl; ++l) {
    double h[9];
    std::memcpy(h, &N.h_ll[l * 9], sizeof h);
    if (lambda > 0.0) { h[0] += lambda; h[4] += lambda; h[8] += lambda; }
    inv_ok[l] = try_inverse3(h, &hinv[l * 9]) ? 1 : 0;
  }
  std::vector<uint32_t> ident(np), fold(np);
  for (size_t i = 0; i < np; ++i) {
    ident[i] = (uint32_t)i;
    fold[i] = (uint32_t)(i < (np + 1) / 2 ? 2 * i : 2 * (np - 1 - i) + 1);
  }
  const size_t wi = band_width(N, inv_ok, ident), wf = band_width(N, inv_ok, fold);
  B.pos = wf < wi ? fold : ident;
  const size_t w = std::min(wi, wf);
  if (3 * w > np) return false;
  B.n = np * 6;
  B.W = 6 * w + 5;
  B.a.assign(B.n * (B.W + 1), 0.0);
  rhs.assign(np * 6, 0.0);
  for (size_t p = 0; p < np; ++p) {
    const size_t P = B.pos[p];
    for (int r = 0; r < 6; ++r) {
      for (int c = 0; c <= r; ++c) {
        double v = N.h_pp[p * 36 + r * 6 + c];
        if (r == c && lambda > 0.0) v += lambda;
        B.at(6 * P + r, 6 * P + c) = v;
      }
      rhs[p * 6 + r] = -N.b_p[p * 6 + r];
    }
  }
  // Schur terms, each permuted block row owned by one thread (landmark order).
#pragma omp parallel num_threads(threads)
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num(), nt = omp_get_num_threads();
#else
    const int tid = 0, nt = 1;
#endif
    for (size_t l = 0; l < nl; ++l) {
      if (!inv_ok[l]) continue;
      const double* hi = &hinv[l * 9];
      const std::vector<Cross>& cr = N.cross[l];
      for (const Cross& a : cr) {
        const size_t Pa = B.pos[a.pose];
        if ((int)(Pa % nt) != tid) continue;
        double ah[18];
        for (int r = 0; r < 6; ++r)
          for (int c = 0; c < 3; ++c) {
            double t = 0.0;
            for (int k = 0; k < 3; ++k) t += a.a[r * 3 + k] * hi[k * 3 + c];
            ah[r * 3 + c] = t;
          }
        for (const Cross& b : cr) {
          const size_t Pb = B.pos[b.pose];
          if (Pb > Pa) continue;
          for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) {
              if (Pb == Pa && c > r) continue;
              double t = 0.0;
              for (int k = 0; k < 3; ++k) t += ah[r * 3 + k] * b.a[c * 3 + k];
              B.at(6 * Pa + r, 6 * Pb + c) -= t;
            }
        }
        const double* bl = &N.b_l[l * 3];
        for (int k = 0; k < 6; ++k) {
          double t = 0.0;
          for (int q = 0; q < 3; ++q) t += ah[k * 3 + q] * bl[q];
          rhs[a.pose * 6 + k] += t;
        }
      }
    }
  }
  return true;
}

// In-place band Cholesky (left-looking, column by column; the rows of a
// column in parallel).  False when not positive definite.
bool band_cholesky(Band& B, int threads) {
  const size_t n = B.n, W = B.W;
  for (size_t j = 0; j < n; ++j) {
    const size_t k0 = j > W ? j - W : 0;
    double d = B.at(j, j);
    for (size_t k = k0; k < j; ++k) d -= B.at(j, k) * B.at(j, k);
    if (!(d > 0.0) || !std::isfinite(d)) return false;
    const double ljj = std::sqrt(d);
    B.at(j, j) = ljj;
    const size_t i1 = std::min(n - 1, j + W);
#pragma omp parallel for schedule(static) num_threads(threads) if (i1 - j > 64)
    for (long long ii = (long long)j + 1; ii <= (long long)i1; ++ii) {
      const size_t i = (size_t)ii;
      const size_t q0 = std::max(k0, i > W ? i - W : 0);
      double t = B.at(i, j);
      for (size_t k = q0; k < j; ++k) t -= B.at(i, k) * B.at(j, k);
      B.at(i, j) = t / ljj;
    }
  }
  return true;
}

void band_solve(const Band& B, std::vector<double>& x) {
  const size_t n = B.n, W = B.W;
  for (size_t i = 0; i < n; ++i) {
    double s = x[i];
    for (size_t k = i > W ? i - W : 0; k < i; ++k) s -= B.at(i, k) * x[k];
    x[i] = s / B.at(i, i);
  }
  for (size_t ii = n; ii-- > 0;) {
    double s = x[ii];
    for (size_t k = ii + 1; k <= std::min(n - 1, ii + W); ++k) s -= B.at(k, ii) * x[k];
    x[ii] = s / B.at(ii, ii);
  }
}

// solve_step (normal_equations.rs:1314-1733).  Returns false on
// BaError::SingularSystem.
bool solve_step(const Normal& N, size_t np, size_t nl, double lambda, int solver,
                int threads, std::vector<double>& dp, std::vector<double>& dl) {
  dp.assign(np * 6, 0.0);
  dl.assign(nl * 3, 0.0);
  if (np == 0) {  // landmark-only (normal_equations.rs:1332-1371)
    for (size_t l = 0; l < nl; ++l) {
      double h[9], hi[9];
      std::memcpy(h, &N.h_ll[l * 9], sizeof h);
      if (lambda > 0.0) { h[0] += lambda; h[4] += lambda; h[8] += lambda; }
      if (!try_inverse3(h, hi)) return false;
      for (int k = 0; k < 3; ++k)
        dl[l * 3 + k] = -(hi[k * 3] * N.b_l[l * 3] + hi[k * 3 + 1] * N.b_l[l * 3 + 1] +
                          hi[k * 3 + 2] * N.b_l[l * 3 + 2]);
    }
    return true;
  }
  std::vector<double> s, rhs, hinv;
  std::vector<uint8_t> ok;
  Band band;
  if (solver == 2 && reduce_banded(N, np, nl, lambda, threads, band, rhs, ok, hinv)) {
    // LinearSolver::Sparse, factored in band storage (Cholesky only).
    if (!band_cholesky(band, threads)) return false;
    std::vector<double> x(np * 6);
    for (size_t p = 0; p < np; ++p)
      for (int r = 0; r < 6; ++r) x[6 * band.pos[p] + r] = rhs[p * 6 + r];
    band_solve(band, x);
    dp.resize(np * 6);
    for (size_t p = 0; p < np; ++p)
      for (int r = 0; r < 6; ++r) dp[p * 6 + r] = x[6 * band.pos[p] + r];
  } else {
    reduce(N, np, nl, lambda, threads, s, rhs, ok, hinv);
    const size_t dim = np * 6;
    std::vector<double> x = rhs;
    std::vector<double> a = s;
    if (cholesky(a, dim, threads)) {
      cholesky_solve(a, dim, x);
    } else {
      if (solver >= 1) return false;  // LinearSolver::Sparse: block Cholesky only
      x = rhs;
      if (!lu_solve(s, dim, x)) return false;
    }
    dp = x;
  }
  // Back-substitution (normal_equations.rs:1717-1733).
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long long ll = 0; ll < (long long)nl; ++ll) {
    const size_t l = (size_t)ll;
    if (!ok[l]) continue;
    double acc[3] = {-N.b_l[l * 3], -N.b_l[l * 3 + 1], -N.b_l[l * 3 + 2]};
    for (const Cross& c : N.cross[l]) {
      for (int k = 0; k < 3; ++k) {
        double t = 0.0;
        for (int q = 0; q < 6; ++q) t += c.a[q * 3 + k] * dp[c.pose * 6 + q];
        acc[k] -= t;
      }
    }
    const double* hi = &hinv[l * 9];
    for (int k = 0; k < 3; ++k)
      dl[l * 3 + k] = hi[k * 3] * acc[0] + hi[k * 3 + 1] * acc[1] + hi[k * 3 + 2] * acc[2];
  }
  return true;
}

bool load_problem(const vlba_problem* p, const vlba_config* cfg, Problem* P, int* status,
                  uint64_t* err_index) {
  *status = VLBA_OK;
  if (!p || !cfg) { *status = VLBA_ERR_INVALID_ARGUMENT; return false; }
  // validate_observation_weights (optimize.rs:628-650) runs before the
  // solve's own checks (optimize.rs:48); the count is num_observations by
  // construction here.
  if (p->obs_weight)
    for (uint64_t o = 0; o < p->num_observations; ++o)
      if (!std::isfinite(p->obs_weight[o]) || p->obs_weight[o] < 0.0) {
        *status = VLBA_ERR_INVALID_OBSERVATION_WEIGHT;
        if (err_index) *err_index = o;
        return false;
      }
  if (p->num_cameras == 0 || !p->cameras) { *status = VLBA_ERR_UNSUPPORTED_CAMERA_MODEL; return false; }
  P->p = p;
  P->per_obs_camera = p->obs_camera != nullptr;
  P->cams.resize(p->num_cameras);
  for (uint32_t c = 0; c < p->num_cameras; ++c)
    if (!resolve_camera(p->cameras[c], &P->cams[c])) {
      *status = VLBA_ERR_UNSUPPORTED_CAMERA_MODEL;
      return false;
    }
  // Order of the checks of lm.rs:168-229: the stereo camera model
  // (check_stereo_camera_model, problem.rs:733-745), then counts, then each
  // observation list in turn -- monocular, rectified stereo (its baseline
  // first), general stereo, rig.
  bool rectified = false, general = false;
  if (p->obs_kind)
    for (uint64_t o = 0; o < p->num_observations; ++o) {
      if (p->obs_kind[o] > 2) { *status = VLBA_ERR_INVALID_ARGUMENT; return false; }
      rectified = rectified || p->obs_kind[o] == 1;
      general = general || p->obs_kind[o] == 2;
    }
  if (((rectified || general) && !p->obs_stereo) || (general && !p->obs_right_camera)) {
    *status = VLBA_ERR_INVALID_ARGUMENT;
    return false;
  }
  if ((rectified || general) && p->cameras[0].model != VLBA_CAMERA_PINHOLE &&
      p->cameras[0].model != VLBA_CAMERA_SIMPLE_PINHOLE) {
    *status = VLBA_ERR_UNSUPPORTED_CAMERA_MODEL;
    return false;
  }
  if (p->num_poses == 0) { *status = VLBA_ERR_NO_POSES; return false; }
  if (p->num_observations == 0) { *status = VLBA_ERR_NO_OBSERVATIONS; return false; }
  if (p->num_landmarks == 0) { *status = VLBA_ERR_NO_LANDMARKS; return false; }
  const int order[4] = {P->per_obs_camera ? -1 : 0, 1, 2, P->per_obs_camera ? 0 : -1};
  for (int li = 0; li < 4; ++li) {
    const int kind = order[li];
    if (kind < 0) continue;
    if (kind == 1 && rectified &&
        !(std::isfinite(p->stereo_baseline) && p->stereo_baseline > 0.0)) {
      *status = VLBA_ERR_MISSING_STEREO_BASELINE;
      return false;
    }
    for (uint64_t o = 0; o < p->num_observations; ++o) {
      if ((p->obs_kind ? (int)p->obs_kind[o] : 0) != kind) continue;
      if (p->obs_pose[o] >= p->num_poses) {
        *status = VLBA_ERR_MISSING_POSE;
        if (err_index) *err_index = p->obs_pose[o];
        return false;
      }
      if (p->obs_landmark[o] >= p->num_landmarks) {
        *status = VLBA_ERR_MISSING_LANDMARK;
        if (err_index) *err_index = p->obs_landmark[o];
        return false;
      }
      if ((kind == 0 && P->per_obs_camera && p->obs_camera[o] >= p->num_cameras) ||
          (kind == 2 && p->obs_right_camera[o] >= p->num_cameras)) {
        *status = VLBA_ERR_INVALID_ARGUMENT;
        if (err_index) *err_index = o;
        return false;
      }
    }
  }
  P->poses.resize(p->num_poses);
  for (uint64_t i = 0; i < p->num_poses; ++i) {
    P->poses[i].q = Quat{p->pose_q[4 * i], p->pose_q[4 * i + 1], p->pose_q[4 * i + 2],
                         p->pose_q[4 * i + 3]};
    P->poses[i].t = v3(p->pose_t[3 * i], p->pose_t[3 * i + 1], p->pose_t[3 * i + 2]);
  }
  P->points.resize(p->num_landmarks);
  for (uint64_t i = 0; i < p->num_landmarks; ++i)
    P->points[i] = v3(p->landmarks[3 * i], p->landmarks[3 * i + 1], p->landmarks[3 * i + 2]);
  P->kernel = Kernel{cfg->robust_kernel, cfg->robust_parameter};
  return true;
}

void store_problem(const Problem& P, vlba_problem* p) {
  for (uint64_t i = 0; i < p->num_poses; ++i) {
    p->pose_q[4 * i] = P.poses[i].q.w;
    p->pose_q[4 * i + 1] = P.poses[i].q.i;
    p->pose_q[4 * i + 2] = P.poses[i].q.j;
    p->pose_q[4 * i + 3] = P.poses[i].q.k;
    p->pose_t[3 * i] = P.poses[i].t.x;
    p->pose_t[3 * i + 1] = P.poses[i].t.y;
    p->pose_t[3 * i + 2] = P.poses[i].t.z;
  }
  for (uint64_t i = 0; i < p->num_landmarks; ++i) {
    p->landmarks[3 * i] = P.points[i].x;
    p->landmarks[3 * i + 1] = P.points[i].y;
    p->landmarks[3 * i + 2] = P.points[i].z;
  }
}

// ------------------------------------------------ matrix-free implicit Schur
// ImplicitSchurOperator (bundle/implicit_schur.rs:108-300): the reduced
// camera system S = D + lambda I - sum_l sum_(a,b) A_a H_l^-1 A_b^T applied
// without forming it.  Errors mirror ImplicitSchurError; the LM treats any of
// them as BaError::SingularSystem (bundle/lm.rs:574-590: reject, lambda up).
enum MfError {
  kMfOk = 0,
  kMfNonFinite = 1,
  kMfNonSpdPreconditioner = 2,
  kMfMaxIterations = 3,
  kMfNonPositiveCurvature = 4,
  kMfResidualCheckFailed = 5,
  kMfEmptySystem = 6,
  kMfInvalidTolerance = 7,
};

bool all_finite(const double* v, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(v[i])) return false;
  return true;
}

// In-place inverse of the SPD n x n row-major matrix through its Cholesky
// factor (nalgebra block.cholesky().inverse()); false when not positive
// definite.
bool spd_inverse(std::vector<double>& a, size_t n) {
  std::vector<double> l = a;
  if (!cholesky(l, n, 1)) return false;
  std::vector<double> col(n);
  for (size_t c = 0; c < n; ++c) {
    std::fill(col.begin(), col.end(), 0.0);
    col[c] = 1.0;
    cholesky_solve(l, n, col);
    for (size_t r = 0; r < n; ++r) a[r * n + c] = col[r];
  }
  return true;
}

struct MfOperator {
  size_t np = 0, nl = 0;
  const Normal* N = nullptr;
  std::vector<double> diag;    // [36 np] damped pose blocks
  std::vector<double> hinv;    // [9 nl] damped landmark inverses
  std::vector<uint8_t> inv_ok; // try_inverse succeeded
  std::vector<double> pinv;    // [36 np] block-Jacobi inverses
  std::vector<std::vector<double>> cluster;  // cluster8 inverses (6k x 6k)
  std::vector<double> rhs;     // [6 np]
  // Per pose, its cross blocks (landmark, index) in landmark order, so the
  // parallel apply subtracts them in the serial order of the reference.
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> at_pose;
};

// ImplicitSchurOperator::new_with_debug (implicit_schur.rs:133-300).
int mf_build(const Normal& N, size_t np, size_t nl, double lambda, int threads, MfOperator* op) {
  if (!std::isfinite(lambda) || lambda < 0.0) return kMfNonFinite;
  if (np == 0) return kMfEmptySystem;
  op->np = np;
  op->nl = nl;
  op->N = &N;
  if (!all_finite(N.b_p.data(), N.b_p.size()) || !all_finite(N.h_pp.data(), N.h_pp.size()))
    return kMfNonFinite;
  op->diag = N.h_pp;
  if (lambda > 0.0)
    for (size_t p = 0; p < np; ++p)
      for (int c = 0; c < 6; ++c) op->diag[p * 36 + c * 7] += lambda;
  op->hinv.assign(nl * 9, 0.0);
  op->inv_ok.assign(nl, 0);
  op->rhs.resize(np * 6);
  for (size_t i = 0; i < np * 6; ++i) op->rhs[i] = -N.b_p[i];
  for (size_t l = 0; l < nl; ++l) {
    if (!all_finite(&N.h_ll[l * 9], 9) || !all_finite(&N.b_l[l * 3], 3)) return kMfNonFinite;
    for (const Cross& c : N.cross[l])
      if (!all_finite(c.a, 18)) return kMfNonFinite;
    double h[9];
    std::memcpy(h, &N.h_ll[l * 9], sizeof h);
    if (lambda > 0.0) { h[0] += lambda; h[4] += lambda; h[8] += lambda; }
    double* hi = &op->hinv[l * 9];
    if (!try_inverse3(h, hi)) continue;  // skipped, as solve_step skips it
    if (!all_finite(hi, 9)) return kMfNonFinite;
    op->inv_ok[l] = 1;
    // rhs += A H^-1 b_l per cross block.
    const double* bl = &N.b_l[l * 3];
    const double v[3] = {hi[0] * bl[0] + hi[1] * bl[1] + hi[2] * bl[2],
                         hi[3] * bl[0] + hi[4] * bl[1] + hi[5] * bl[2],
                         hi[6] * bl[0] + hi[7] * bl[1] + hi[8] * bl[2]};
    for (const Cross& c : N.cross[l])
      for (int r = 0; r < 6; ++r)
        op->rhs[c.pose * 6 + r] += c.a[r * 3] * v[0] + c.a[r * 3 + 1] * v[1] + c.a[r * 3 + 2] * v[2];
  }
  if (!all_finite(op->rhs.data(), op->rhs.size())) return kMfNonFinite;
  // Block-Jacobi: D + lambda - G H^-1 G^T with the cross blocks of one pose
  // grouped first (two sensors of one rig frame share the pose block).
  op->pinv = op->diag;
  for (size_t l = 0; l < nl; ++l) {
    if (!op->inv_ok[l]) continue;
    const std::vector<Cross>& cr = N.cross[l];
    std::vector<std::pair<uint32_t, std::array<double, 18>>> grouped;  // ascending pose
    for (const Cross& c : cr) {
      auto it = std::lower_bound(grouped.begin(), grouped.end(), c.pose,
                                 [](const auto& e, uint32_t p) { return e.first < p; });
      if (it == grouped.end() || it->first != c.pose) {
        std::array<double, 18> z{};
        it = grouped.insert(it, {c.pose, z});
      }
      for (int e = 0; e < 18; ++e) it->second[e] += c.a[e];
    }
    const double* hi = &op->hinv[l * 9];
    for (const auto& g : grouped) {
      double gh[18];
      for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 3; ++c)
          gh[r * 3 + c] = g.second[r * 3] * hi[c] + g.second[r * 3 + 1] * hi[3 + c] +
                          g.second[r * 3 + 2] * hi[6 + c];
      double* blk = &op->pinv[g.first * 36];
      for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c)
          blk[r * 6 + c] -= gh[r * 3] * g.second[c * 3] + gh[r * 3 + 1] * g.second[c * 3 + 1] +
                            gh[r * 3 + 2] * g.second[c * 3 + 2];
    }
  }
  if (!all_finite(op->pinv.data(), op->pinv.size())) return kMfNonFinite;
  for (size_t p = 0; p < np; ++p) {
    std::vector<double> blk(op->pinv.begin() + p * 36, op->pinv.begin() + p * 36 + 36);
    if (!spd_inverse(blk, 6)) return kMfNonSpdPreconditioner;
    if (!all_finite(blk.data(), 36)) return kMfNonFinite;
    std::copy(blk.begin(), blk.end(), op->pinv.begin() + p * 36);
  }
  op->at_pose.assign(np, {});
  for (size_t l = 0; l < nl; ++l) {
    if (!op->inv_ok[l]) continue;
    for (uint32_t k = 0; k < (uint32_t)N.cross[l].size(); ++k)
      op->at_pose[N.cross[l][k].pose].push_back({(uint32_t)l, k});
  }
  (void)threads;
  return kMfOk;
}

// with_cluster8 (implicit_schur.rs:302-376): principal Schur blocks of
// consecutive groups of eight poses, inverted by Cholesky; replaces the
// block-Jacobi preconditioner.
int mf_cluster8(MfOperator* op) {
  constexpr size_t K = 8;
  const size_t np = op->np;
  const size_t nc = (np + K - 1) / K;
  op->cluster.assign(nc, {});
  for (size_t c = 0; c < nc; ++c) {
    const size_t n = std::min(K, np - c * K) * 6;
    std::vector<double>& b = op->cluster[c];
    b.assign(n * n, 0.0);
    for (size_t s = 0; s < n / 6; ++s)
      for (int r = 0; r < 6; ++r)
        for (int q = 0; q < 6; ++q) b[(s * 6 + r) * n + s * 6 + q] = op->diag[(c * K + s) * 36 + r * 6 + q];
  }
  const Normal& N = *op->N;
  for (size_t l = 0; l < op->nl; ++l) {
    if (!op->inv_ok[l]) continue;
    // Cross sums per pose, members per cluster in first-seen order.
    std::vector<std::pair<uint32_t, std::array<double, 18>>> sums;  // first-seen order
    for (const Cross& x : N.cross[l]) {
      auto it = std::find_if(sums.begin(), sums.end(), [&](const auto& e) { return e.first == x.pose; });
      if (it == sums.end()) {
        std::array<double, 18> z{};
        sums.push_back({x.pose, z});
        it = sums.end() - 1;
      }
      for (int e = 0; e < 18; ++e) it->second[e] += x.a[e];
    }
    const double* hi = &op->hinv[l * 9];
    for (const auto& a : sums) {
      double left[18];
      for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 3; ++c)
          left[r * 3 + c] = a.second[r * 3] * hi[c] + a.second[r * 3 + 1] * hi[3 + c] +
                            a.second[r * 3 + 2] * hi[6 + c];
      for (const auto& b : sums) {
        if (a.first / K != b.first / K) continue;
        std::vector<double>& blk = op->cluster[a.first / K];
        const size_t n = (size_t)std::sqrt((double)blk.size());
        for (int r = 0; r < 6; ++r)
          for (int c = 0; c < 6; ++c)
            blk[((a.first % K) * 6 + r) * n + (b.first % K) * 6 + c] -=
                left[r * 3] * b.second[c * 3] + left[r * 3 + 1] * b.second[c * 3 + 1] +
                left[r * 3 + 2] * b.second[c * 3 + 2];
      }
    }
  }
  for (size_t c = 0; c < nc; ++c) {
    std::vector<double>& blk = op->cluster[c];
    if (!all_finite(blk.data(), blk.size())) return kMfNonFinite;
    const size_t n = (size_t)std::sqrt((double)blk.size());
    if (!spd_inverse(blk, n)) return kMfNonSpdPreconditioner;
    if (!all_finite(blk.data(), blk.size())) return kMfNonFinite;
  }
  return kMfOk;
}

// apply (implicit_schur.rs:390-431): D x - sum_l sum_a A_a H^-1 (sum_b A_b^T
// x_b), every cross block kept (repeated pose slots are separate sensor
// rows).  Per landmark in parallel, then per pose in landmark order.
void mf_apply(const MfOperator& op, const double* x, double* out, int threads) {
  const Normal& N = *op.N;
  std::vector<double> red(op.nl * 3, 0.0);
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long long ll = 0; ll < (long long)op.nl; ++ll) {
    const size_t l = (size_t)ll;
    if (!op.inv_ok[l]) continue;
    double pr[3] = {0.0, 0.0, 0.0};
    for (const Cross& c : N.cross[l]) {
      const double* xp = x + c.pose * 6;
      for (int k = 0; k < 3; ++k) {
        double t = 0.0;
        for (int r = 0; r < 6; ++r) t += c.a[r * 3 + k] * xp[r];
        pr[k] += t;
      }
    }
    const double* hi = &op.hinv[l * 9];
    for (int k = 0; k < 3; ++k) red[l * 3 + k] = hi[k * 3] * pr[0] + hi[k * 3 + 1] * pr[1] + hi[k * 3 + 2] * pr[2];
  }
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long long pp = 0; pp < (long long)op.np; ++pp) {
    const size_t p = (size_t)pp;
    const double* blk = &op.diag[p * 36];
    const double* xp = x + p * 6;
    double o[6];
    for (int r = 0; r < 6; ++r) {
      double t = 0.0;
      for (int c = 0; c < 6; ++c) t += blk[r * 6 + c] * xp[c];
      o[r] = t;
    }
    for (const auto& lk : op.at_pose[p]) {
      const Cross& c = N.cross[lk.first][lk.second];
      const double* rl = &red[lk.first * 3];
      for (int r = 0; r < 6; ++r) o[r] -= c.a[r * 3] * rl[0] + c.a[r * 3 + 1] * rl[1] + c.a[r * 3 + 2] * rl[2];
    }
    for (int r = 0; r < 6; ++r) out[p * 6 + r] = o[r];
  }
}

// apply_preconditioner (implicit_schur.rs:433-473).
void mf_precondition(const MfOperator& op, const double* r, double* z) {
  if (!op.cluster.empty()) {
    size_t off = 0;
    for (const std::vector<double>& inv : op.cluster) {
      const size_t n = (size_t)std::sqrt((double)inv.size());
      for (size_t a = 0; a < n; ++a) {
        double t = 0.0;
        for (size_t b = 0; b < n; ++b) t += inv[a * n + b] * r[off + b];
        z[off + a] = t;
      }
      off += n;
    }
    return;
  }
  for (size_t p = 0; p < op.np; ++p) {
    const double* blk = &op.pinv[p * 36];
    for (int a = 0; a < 6; ++a) {
      double t = 0.0;
      for (int b = 0; b < 6; ++b) t += blk[a * 6 + b] * r[p * 6 + b];
      z[p * 6 + a] = t;
    }
  }
}

double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}

struct MfPcgOptions {
  uint32_t max_iterations;
  double relative_tolerance, absolute_tolerance;
};

// solve_pcg (implicit_schur.rs:475-736 with no restarts): x = 0, r = b;
// stop once |r| <= max(abs, rel |b|) and the true residual |b - A x| agrees,
// else fail: MaxIterations at the cap (unless the true residual meets the
// target there), NonPositiveCurvature for p.Ap <= 0 or r.z <= 0,
// ResidualCheckFailed when the recursive residual met the target but the
// true one did not.
int mf_solve_pcg(const MfOperator& op, const std::vector<double>& b, const MfPcgOptions& o,
                 int threads, std::vector<double>& x, uint32_t* iterations, double* residual,
                 double* target_out) {
  const size_t n = op.np * 6;
  *iterations = 0;
  if (!all_finite(b.data(), n)) return kMfNonFinite;
  if (!std::isfinite(o.relative_tolerance) || o.relative_tolerance < 0.0 ||
      !std::isfinite(o.absolute_tolerance) || o.absolute_tolerance < 0.0)
    return kMfInvalidTolerance;
  const double bnorm = std::sqrt(dot(b, b));
  const double target = std::max(o.absolute_tolerance, o.relative_tolerance * bnorm);
  if (target_out) *target_out = target;
  if (!std::isfinite(target)) return kMfNonFinite;
  x.assign(n, 0.0);
  std::vector<double> r = b, z(n), p(n), q(n);
  double rn = std::sqrt(dot(r, r));
  if (!std::isfinite(rn)) return kMfNonFinite;
  auto true_norm = [&]() {
    mf_apply(op, x.data(), q.data(), threads);
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += (b[i] - q[i]) * (b[i] - q[i]);
    return std::sqrt(s);
  };
  if (rn <= target) {
    const double t = true_norm();
    *residual = t;
    return t <= target ? kMfOk : kMfResidualCheckFailed;
  }
  if (o.max_iterations == 0) {
    *residual = rn;
    return kMfMaxIterations;
  }
  mf_precondition(op, r.data(), z.data());
  double rho = dot(r, z);
  if (!std::isfinite(rho) || rho <= 0.0) return kMfNonPositiveCurvature;
  p = z;
  for (uint32_t it = 1; it <= o.max_iterations; ++it) {
    mf_apply(op, p.data(), q.data(), threads);
    const double curv = dot(p, q);
    if (!std::isfinite(curv) || curv <= 0.0) return kMfNonPositiveCurvature;
    const double alpha = rho / curv;
    if (!std::isfinite(alpha)) return kMfNonFinite;
    for (size_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    rn = std::sqrt(dot(r, r));
    *iterations = it;
    if (!all_finite(x.data(), n) || !std::isfinite(rn)) return kMfNonFinite;
    if (rn <= target) {
      const double t = true_norm();
      *residual = t;
      return t <= target ? kMfOk : kMfResidualCheckFailed;
    }
    if (it == o.max_iterations) {
      const double t = true_norm();
      *residual = t;
      return t <= target ? kMfOk : kMfMaxIterations;
    }
    mf_precondition(op, r.data(), z.data());
    const double next = dot(r, z);
    if (!std::isfinite(next) || next <= 0.0) return kMfNonPositiveCurvature;
    const double beta = next / rho;
    if (!std::isfinite(beta)) return kMfNonFinite;
    for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rho = next;
  }
  return kMfMaxIterations;
}

// complete_delta (implicit_schur.rs:789-828): dl = H^-1 (-b_l - sum A^T dp).
int mf_complete_delta(const MfOperator& op, const std::vector<double>& dp, int threads,
                      std::vector<double>& dl) {
  const Normal& N = *op.N;
  if (!all_finite(dp.data(), dp.size())) return kMfNonFinite;
  dl.assign(op.nl * 3, 0.0);
  bool bad = false;
#pragma omp parallel for schedule(static) num_threads(threads) reduction(|| : bad)
  for (long long ll = 0; ll < (long long)op.nl; ++ll) {
    const size_t l = (size_t)ll;
    if (!op.inv_ok[l]) continue;
    double acc[3] = {-N.b_l[l * 3], -N.b_l[l * 3 + 1], -N.b_l[l * 3 + 2]};
    for (const Cross& c : N.cross[l])
      for (int k = 0; k < 3; ++k) {
        double t = 0.0;
        for (int r = 0; r < 6; ++r) t += c.a[r * 3 + k] * dp[c.pose * 6 + r];
        acc[k] -= t;
      }
    const double* hi = &op.hinv[l * 9];
    for (int k = 0; k < 3; ++k) {
      dl[l * 3 + k] = hi[k * 3] * acc[0] + hi[k * 3 + 1] * acc[1] + hi[k * 3 + 2] * acc[2];
      if (!std::isfinite(dl[l * 3 + k])) bad = true;
    }
  }
  return bad ? kMfNonFinite : kMfOk;
}

// The reference LM loop (lm.rs:356-1009, Legacy or matrix-free backend): the
// linear solve is `step`, which returns false for BaError::SingularSystem.
using StepFn = std::function<bool(const Normal&, size_t, size_t, double, std::vector<double>&,
                                  std::vector<double>&)>;
int run_lm(vlba_problem* p, const vlba_config* cfg, int threads, vlba_result* res,
           vlba_iteration* its, uint32_t cap, const StepFn& step);

}  // namespace

extern "C" {

int vlba_oracle_check(const vlba_problem* p, const vlba_config* cfg, uint64_t* err_index) {
  Problem P;
  int status;
  if (!load_problem(p, cfg, &P, &status, err_index)) return status;
  Slots S;
  build_slots(p, &S);
  if (S.var_poses.empty() && S.var_lms.empty()) return VLBA_ERR_ALL_POSES_FIXED;
  return VLBA_OK;
}

int vlba_oracle_cost(const vlba_problem* p, const vlba_config* cfg, int threads, double* cost,
                     uint64_t* nonprojectable) {
  Problem P;
  int status;
  if (!load_problem(p, cfg, &P, &status, nullptr)) return status;
  cost_and_nonprojectable(P, threads_or_default(threads), cost, nonprojectable);
  return VLBA_OK;
}

// reprojection_squared_residuals (problem.rs:756-830): per observation, in
// its order, the squared reprojection residual, NaN when the observation is
// behind its sensor or does not project.
int vlba_oracle_squared_residuals(const vlba_problem* p, const vlba_config* cfg, double* out) {
  Problem P;
  int status;
  if (!load_problem(p, cfg, &P, &status, nullptr)) return status;
  for (uint64_t o = 0; o < p->num_observations; ++o) {
    if (p->obs_kind && p->obs_kind[o] != 0) {
      double r[4], jp[24], jl[12];
      const int m = obs_residual_jacobians(P, o, r, jp, jl);
      double ss = 0.0;
      for (int i = 0; i < m; ++i) ss += r[i] * r[i];
      out[o] = m ? ss : std::numeric_limits<double>::quiet_NaN();
      continue;
    }
    const Se3& T = P.poses[p->obs_pose[o]];
    const Cam& c = P.cam_of(o);
    V3 xc = se3_transform(T, P.points[p->obs_landmark[o]]);
    if (P.per_obs_camera) xc = se3_transform(c.sensor_from_rig, xc);
    double pred[2];
    if (xc.z <= 0.0 || !camera_project(c, xc, pred)) {
      out[o] = std::numeric_limits<double>::quiet_NaN();
      continue;
    }
    const double rx = pred[0] - p->obs_xy[2 * o], ry = pred[1] - p->obs_xy[2 * o + 1];
    out[o] = rx * rx + ry * ry;
  }
  return VLBA_OK;
}

// Camera::project of one camera-frame point; returns 0 when it does not project.
int vlba_oracle_camera_project(const vlba_camera* cam, const double xc[3], double out[2]) {
  Cam c;
  if (!resolve_camera(*cam, &c)) return -1;
  return camera_project(c, v3(xc[0], xc[1], xc[2]), out) ? 1 : 0;
}

// mono_project_with_jacobian; returns 0 when the point does not project.
int vlba_oracle_mono_project(const vlba_camera* cam, const double xc[3], double pred[2],
                             double jac[6]) {
  Cam c;
  if (!resolve_camera(*cam, &c)) return -1;
  return mono_project_with_jacobian(c, v3(xc[0], xc[1], xc[2]), pred, jac) ? 1 : 0;
}

// T <- T * Exp(xi) for a pose given as quaternion (w,i,j,k) + translation.
void vlba_oracle_pose_update(double q[4], double t[3], const double xi[6]) {
  Se3 T{Quat{q[0], q[1], q[2], q[3]}, v3(t[0], t[1], t[2])};
  const Se3 r = se3_compose(T, se3_exp(xi));
  q[0] = r.q.w; q[1] = r.q.i; q[2] = r.q.j; q[3] = r.q.k;
  t[0] = r.t.x; t[1] = r.t.y; t[2] = r.t.z;
}

// Normal equations at the current state: h_pp (36 per variable pose), b_p (6),
// h_ll (9 per variable landmark), b_l (3).  Arrays sized by the caller.
int vlba_oracle_normal_equations(const vlba_problem* p, const vlba_config* cfg, int threads,
                                 double* h_pp, double* b_p, double* h_ll, double* b_l) {
  Problem P;
  int status;
  if (!load_problem(p, cfg, &P, &status, nullptr)) return status;
  Slots S;
  build_slots(p, &S);
  Normal N;
  build_normal(P, S, threads_or_default(threads), &N);
  std::copy(N.h_pp.begin(), N.h_pp.end(), h_pp);
  std::copy(N.b_p.begin(), N.b_p.end(), b_p);
  std::copy(N.h_ll.begin(), N.h_ll.end(), h_ll);
  std::copy(N.b_l.begin(), N.b_l.end(), b_l);
  return VLBA_OK;
}

// Reduced camera system (dense (6P)^2, both triangles) and its rhs at lambda,
// plus the damped step (dp 6P, dl 3L) when dp/dl are non-NULL.
int vlba_oracle_reduced_system(const vlba_problem* p, const vlba_config* cfg, double lambda,
                               int threads, double* s_out, double* rhs_out, double* dp_out,
                               double* dl_out) {
  Problem P;
  int status;
  if (!load_problem(p, cfg, &P, &status, nullptr)) return status;
  Slots S;
  build_slots(p, &S);
  const int nt = threads_or_default(threads);
  Normal N;
  build_normal(P, S, nt, &N);
  const size_t np = S.var_poses.size(), nl = S.var_lms.size();
  std::vector<double> s, rhs, hinv;
  std::vector<uint8_t> ok;
  if (np > 0) {
    reduce(N, np, nl, lambda, nt, s, rhs, ok, hinv);
    if (s_out) std::copy(s.begin(), s.end(), s_out);
    if (rhs_out) std::copy(rhs.begin(), rhs.end(), rhs_out);
  }
  if (dp_out || dl_out) {
    std::vector<double> dp, dl;
    if (!solve_step(N, np, nl, lambda, 0, nt, dp, dl)) return VLBA_ERR_SINGULAR_SYSTEM;
    if (dp_out) std::copy(dp.begin(), dp.end(), dp_out);
    if (dl_out) std::copy(dl.begin(), dl.end(), dl_out);
  }
  return VLBA_OK;
}

}  // extern "C"

namespace {

int run_lm(vlba_problem* p, const vlba_config* cfg, int threads, vlba_result* res,
           vlba_iteration* its, uint32_t cap, const StepFn& step) {
  Problem P;
  int status;
  uint64_t err_index = 0;
  if (res) std::memset(res, 0, sizeof *res);
  if (!load_problem(p, cfg, &P, &status, &err_index)) {
    if (res) res->error_index = err_index;
    return status;
  }
  const int nt = threads_or_default(threads);
  Slots S;
  build_slots(p, &S);
  if (S.var_poses.empty() && S.var_lms.empty()) return VLBA_ERR_ALL_POSES_FIXED;
  const size_t np = S.var_poses.size(), nl = S.var_lms.size();

  double initial_cost;
  uint64_t current_nonproj;
  cost_and_nonprojectable(P, nt, &initial_cost, &current_nonproj);
  const uint64_t initial_nonproj = current_nonproj;
  double current_cost = initial_cost;
  double lambda = cfg->has_initial_lambda ? cfg->initial_lambda : 0.0;
  bool converged = false;
  uint32_t count = 0;
  auto push = [&](uint64_t it, double cb, double ca, double mps, double mls, double lam,
                  bool acc) {
    if (its && count < cap) {
      vlba_iteration& e = its[count];
      std::memset(&e, 0, sizeof e);
      e.iteration = it;
      e.cost_before = cb;
      e.cost_after = ca;
      e.max_pose_step = mps;
      e.max_landmark_step = mls;
      e.lambda = lam;
      e.step_accepted = acc ? 1u : 0u;
    }
    ++count;
  };
  uint64_t final_nonproj = current_nonproj;
  for (uint32_t iteration = 0; iteration < cfg->max_iterations; ++iteration) {
    Normal N;
    build_normal(P, S, nt, &N);
    const std::vector<Se3> saved_poses = P.poses;
    const std::vector<V3> saved_points = P.points;
    const double cost_before = current_cost;
    std::vector<double> dp, dl;
    if (!step(N, np, nl, lambda, dp, dl)) {
      lambda = std::min(lambda * cfg->lambda_increase_factor, cfg->max_lambda);
      push(iteration, cost_before, cost_before, 0.0, 0.0, lambda, false);
      if (lambda >= cfg->max_lambda) break;
      continue;
    }
    double max_pose_step = 0.0;
    for (size_t s = 0; s < np; ++s) {
      const double* xi = &dp[s * 6];
      double nn = 0.0;
      for (int k = 0; k < 6; ++k) nn += xi[k] * xi[k];
      max_pose_step = std::max(max_pose_step, std::sqrt(nn));
      Se3& T = P.poses[S.var_poses[s]];
      T = se3_compose(T, se3_exp(xi));
    }
    double max_lm_step = 0.0;
    for (size_t s = 0; s < nl; ++s) {
      const double* d = &dl[s * 3];
      max_lm_step = std::max(max_lm_step, std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
      V3& X = P.points[S.var_lms[s]];
      X = v3(X.x + d[0], X.y + d[1], X.z + d[2]);
    }
    double cost_after;
    uint64_t nonproj_after;
    cost_and_nonprojectable(P, nt, &cost_after, &nonproj_after);
    const bool cost_accepted = cfg->has_initial_lambda ? (cost_after < cost_before) : true;
    const bool accepted = cost_accepted && nonproj_after <= current_nonproj;
    if (!accepted) {
      P.poses = saved_poses;
      P.points = saved_points;
      lambda = std::min(lambda * cfg->lambda_increase_factor, cfg->max_lambda);
      push(iteration, cost_before, cost_after, max_pose_step, max_lm_step, lambda, false);
      if (!cfg->has_initial_lambda) break;
      if (lambda >= cfg->max_lambda) break;
      continue;
    }
    push(iteration, cost_before, cost_after, max_pose_step, max_lm_step, lambda, true);
    current_cost = cost_after;
    current_nonproj = nonproj_after;
    final_nonproj = nonproj_after;
    if (cfg->has_initial_lambda)
      lambda = std::max(lambda * cfg->lambda_decrease_factor, cfg->min_lambda);
    if (max_pose_step < cfg->step_tolerance && max_lm_step < cfg->step_tolerance) {
      converged = true;
      break;
    }
    if (std::fabs(cost_before - cost_after) < cfg->cost_tolerance) {
      converged = true;
      break;
    }
    if (cfg->has_relative_cost_tolerance) {
      const double tol = cfg->relative_cost_tolerance;
      if (std::isfinite(tol) && tol >= 0.0 &&
          (cost_before - cost_after) /
                  std::max(std::fabs(cost_before), std::numeric_limits<double>::epsilon()) <
              tol) {
        converged = true;
        break;
      }
    }
  }
  store_problem(P, p);
  if (res) {
    res->initial_cost = initial_cost;
    res->final_cost = current_cost;
    res->converged = converged ? 1u : 0u;
    res->num_iterations = count;
    res->initial_nonprojectable = initial_nonproj;
    res->final_nonprojectable = final_nonproj;
  }
  return VLBA_OK;
}

}  // namespace

extern "C" {

// BundleAdjustment::optimize (lm.rs:162-1017, Legacy backend).
// solver: 0 = LinearSolver::Dense (Cholesky, LU fallback), 1 = Sparse
// (Cholesky only), 2 = Sparse factored in band storage when the reduced
// system is banded in the capture or fold order (else as 1).  threads <= 0:
// all.
int vlba_oracle_optimize(vlba_problem* p, const vlba_config* cfg, int solver, int threads,
                         vlba_result* res, vlba_iteration* its, uint32_t cap) {
  const int nt = threads_or_default(threads);
  return run_lm(p, cfg, threads, res, its, cap,
                [&](const Normal& N, size_t np, size_t nl, double lambda, std::vector<double>& dp,
                    std::vector<double>& dl) {
                  return solve_step(N, np, nl, lambda, solver, nt, dp, dl);
                });
}

// BundleAdjustment::optimize_matrix_free (bundle/optimize.rs:105-139): the
// same LM loop with the landmark-eliminated system solved by bounded PCG on
// the implicit Schur operator (MatrixFreeBaOptions: max_pcg_iterations,
// pcg_relative_tolerance, pcg_absolute_tolerance; defaults 128, 1e-12,
// 1e-12, bundle/mod.rs:781-798), block-Jacobi preconditioned or, with
// cluster8, by the principal Schur blocks of groups of eight poses
// (optimize_matrix_free_cluster8, optimize.rs:192-208).  A failed solve (any
// ImplicitSchurError) rejects the step and raises lambda, as SingularSystem
// does (lm.rs:574-600).  pcg_iterations (may be NULL) receives the total PCG
// iterations, failures (may be NULL) the failed solves.  Requires at least
// one variable pose (validate_matrix_free_entry, optimize.rs:386-431).
int vlba_oracle_optimize_matrix_free(vlba_problem* p, const vlba_config* cfg,
                                     uint32_t max_pcg_iterations, double pcg_relative_tolerance,
                                     double pcg_absolute_tolerance, int cluster8, int threads,
                                     vlba_result* res, vlba_iteration* its, uint32_t cap,
                                     uint64_t* pcg_iterations, uint32_t* failures) {
  if (!cfg || cfg->max_iterations == 0) return VLBA_ERR_INVALID_ARGUMENT;
  if (cfg->has_initial_lambda && !(std::isfinite(cfg->initial_lambda) && cfg->initial_lambda > 0.0))
    return VLBA_ERR_INVALID_ARGUMENT;
  if (p) {
    bool any_var = false;
    for (uint64_t i = 0; i < p->num_poses && !any_var; ++i)
      any_var = !(p->pose_fixed && p->pose_fixed[i]);
    if (!any_var) return VLBA_DECLINED;  // MatrixFreeBaError::Ineligible
  }
  const int nt = threads_or_default(threads);
  uint64_t total = 0;
  uint32_t failed = 0;
  const MfPcgOptions opt{max_pcg_iterations, pcg_relative_tolerance, pcg_absolute_tolerance};
  const int st = run_lm(
      p, cfg, threads, res, its, cap,
      [&](const Normal& N, size_t np, size_t nl, double lambda, std::vector<double>& dp,
          std::vector<double>& dl) {
        MfOperator op;
        int e = mf_build(N, np, nl, lambda, nt, &op);
        if (e == kMfOk && cluster8) e = mf_cluster8(&op);
        uint32_t iters = 0;
        double resid = 0.0, target = 0.0;
        if (e == kMfOk) e = mf_solve_pcg(op, op.rhs, opt, nt, dp, &iters, &resid, &target);
        total += iters;
        if (e == kMfOk) e = mf_complete_delta(op, dp, nt, dl);
        if (e != kMfOk) ++failed;
        return e == kMfOk;
      });
  if (pcg_iterations) *pcg_iterations = total;
  if (failures) *failures = failed;
  return st;
}

// The implicit Schur operator on a normal-equation system given directly
// (NormalEquationsBa with a PoseDiagonal camera Hessian): np pose blocks
// diag[36 np] (row-major), b_p[6 np], nl landmarks h_ll[9 nl], b_l[3 nl],
// and per landmark cross_count[l] cross blocks (cross_pose, cross_block 6x3
// row-major) in order.  Outputs (each may be NULL): rhs[6 np]; apply_out =
// S x (x[6 np]); precond_out = M^-1 probe; with solve, the PCG solution
// solution[6 np] of S x = rhs_in (rhs_in NULL: the operator's rhs) under
// the options, its iterations, true residual and target, and the landmark
// step delta_l[3 nl] of that solution.  Returns the ImplicitSchurError code
// (0 = ok) of the first failing step.  Test hook for the reference's
// operator tests (implicit_schur.rs:952-1619).
int vlba_oracle_mf_system(uint32_t np, const double* diag, const double* b_p, uint32_t nl,
                          const double* h_ll, const double* b_l, const uint32_t* cross_count,
                          const uint32_t* cross_pose, const double* cross_block, double lambda,
                          int cluster8, const double* x, double* apply_out, const double* probe,
                          double* precond_out, double* rhs_out, int solve, const double* rhs_in,
                          uint32_t max_iterations, double relative_tolerance,
                          double absolute_tolerance, double* solution, uint32_t* iterations,
                          double* residual, double* target, double* delta_l) {
  Normal N;
  N.h_pp.assign(diag, diag + 36 * (size_t)np);
  N.b_p.assign(b_p, b_p + 6 * (size_t)np);
  N.h_ll.assign(h_ll, h_ll + 9 * (size_t)nl);
  N.b_l.assign(b_l, b_l + 3 * (size_t)nl);
  N.cross.assign(nl, {});
  size_t at = 0;
  for (uint32_t l = 0; l < nl; ++l)
    for (uint32_t k = 0; k < cross_count[l]; ++k, ++at) {
      Cross c;
      c.pose = cross_pose[at];
      if (c.pose >= np) return kMfNonFinite;
      std::memcpy(c.a, cross_block + 18 * at, sizeof c.a);
      N.cross[l].push_back(c);
    }
  MfOperator op;
  int e = mf_build(N, np, nl, lambda, 1, &op);
  if (e == kMfOk && cluster8) e = mf_cluster8(&op);
  if (e != kMfOk) return e;
  const size_t n = 6 * (size_t)np;
  if (rhs_out) std::copy(op.rhs.begin(), op.rhs.end(), rhs_out);
  if (x && apply_out) mf_apply(op, x, apply_out, 1);
  if (probe && precond_out) mf_precondition(op, probe, precond_out);
  if (!solve) return kMfOk;
  std::vector<double> b = rhs_in ? std::vector<double>(rhs_in, rhs_in + n) : op.rhs;
  std::vector<double> sol;
  uint32_t it = 0;
  double r = 0.0, t = 0.0;
  e = mf_solve_pcg(op, b, MfPcgOptions{max_iterations, relative_tolerance, absolute_tolerance}, 1,
                   sol, &it, &r, &t);
  if (iterations) *iterations = it;
  if (residual) *residual = r;
  if (target) *target = t;
  if (solution && sol.size() == n) std::copy(sol.begin(), sol.end(), solution);
  if (e != kMfOk) return e;
  if (delta_l) {
    std::vector<double> dl;
    e = mf_complete_delta(op, sol, 1, dl);
    std::copy(dl.begin(), dl.end(), delta_l);
  }
  return e;
}

// ---------------------------------------------------------------------------
// pcg_core (pipelines/slam/src/colmap_incremental/rig_ba_solver.rs:1406-1480)
// on a reduced camera system as ReducedCameraSystem hands it over
// (ba_accel.rs:50-72): damped diagonal blocks (column-major f64), sorted
// edges (a, b) with their (row b, column a) blocks (column-major f32, read in
// f64 with fused multiply-adds as edge_product does, :1314-1331), the run
// inverses (z over each run, block-Jacobi Cholesky inverses elsewhere) and
// the additive coarse level (CoarseCorrection::add_to, :1198-1213).  On
// `threads` OpenMP threads (0: all): each node's product sums its own
// diagonal, then its edges in edge order; dots add fixed chunks of nodes,
// then the chunks in order -- the result does not depend on the thread
// count.  Returns 0 (x and *iterations set), 1 (a non-positive or non-finite
// p.q: pcg_core's None) or 2 (a diagonal block that is not positive definite:
// pcg_core's None too).
int vlba_oracle_reduced_pcg(uint32_t n, uint64_t ne, const uint32_t* edges, const double* diag,
                            const float* offdiag, const double* rhs, double tol,
                            uint32_t max_iterations, uint32_t num_clusters,
                            const uint32_t* cluster_first, const uint32_t* cluster_size,
                            const double* cluster_inverse, uint32_t coarse_group,
                            uint32_t coarse_nodes, const double* coarse_inverse, int threads,
                            double* x, uint32_t* iterations) {
  if (threads > 0) omp_set_num_threads(threads);
  const size_t N = 6 * (size_t)n;
  // Per node its out-edges (a = i, contiguous: edges are sorted) and its
  // in-edges (b = i), each list in edge order.
  std::vector<uint64_t> out_off(n + 1, 0), in_off(n + 1, 0);
  for (uint64_t e = 0; e < ne; ++e) {
    ++out_off[edges[2 * e] + 1];
    ++in_off[edges[2 * e + 1] + 1];
  }
  for (uint32_t i = 0; i < n; ++i) {
    out_off[i + 1] += out_off[i];
    in_off[i + 1] += in_off[i];
  }
  std::vector<uint64_t> in_edge(ne), fill(in_off.begin(), in_off.end() - 1);
  for (uint64_t e = 0; e < ne; ++e) in_edge[fill[edges[2 * e + 1]]++] = e;
  std::vector<double> u(6 * ne);  // B p_a per edge, gathered by row b
  // Block-Jacobi inverses (pcg_core factors every diagonal block).
  std::vector<double> jac(36 * (size_t)n);
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    // d.cholesky().map(|c| c.inverse()): factor, then solve for each column.
    std::vector<double> a(36);
    for (int r = 0; r < 6; ++r)
      for (int c = 0; c < 6; ++c) a[r * 6 + c] = diag[36 * i + c * 6 + r];
    if (!cholesky(a, 6, 1)) {
      bad |= 1;
      continue;
    }
    for (int c = 0; c < 6; ++c) {
      std::vector<double> col(6, 0.0);
      col[c] = 1.0;
      cholesky_solve(a, 6, col);
      for (int r = 0; r < 6; ++r) jac[36 * i + r * 6 + c] = col[r];
    }
  }
  if (bad) return 2;
  std::vector<uint64_t> cl_off(num_clusters + 1, 0);
  for (uint32_t c = 0; c < num_clusters; ++c)
    cl_off[c + 1] = cl_off[c] + 36ull * cluster_size[c] * cluster_size[c];
  std::vector<uint8_t> in_run(n, 0);
  for (uint32_t c = 0; c < num_clusters; ++c)
    for (uint32_t k = 0; k < cluster_size[c]; ++k) in_run[cluster_first[c] + k] = 1;
  const uint32_t m = coarse_group && coarse_nodes ? (coarse_nodes + coarse_group - 1) / coarse_group
                                                   : 0;
  // Each block read once per product, as edge_product does: row a adds its
  // out-edges' B^T p_b and leaves B p_a per edge; row b then adds its
  // in-edges' in edge order.
  auto matvec = [&](const std::vector<double>& p, std::vector<double>& q) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      double y[6];
      for (int r = 0; r < 6; ++r) {
        double acc = 0.0;
        for (int c = 0; c < 6; ++c) acc = std::fma(diag[36 * i + c * 6 + r], p[6 * i + c], acc);
        y[r] = acc;
      }
      const double* pa = &p[6 * (size_t)i];
      for (uint64_t e = out_off[i]; e < out_off[i + 1]; ++e) {
        const float* B = offdiag + 36 * e;  // (row b, column a), column-major
        const double* pb = &p[6 * (size_t)edges[2 * e + 1]];
        double tb[6] = {0, 0, 0, 0, 0, 0};
        for (int c = 0; c < 6; ++c) {
          double d0 = 0.0;
          for (int r = 0; r < 6; ++r) {
            const double v = B[c * 6 + r];
            tb[r] = std::fma(v, pa[c], tb[r]);
            d0 = std::fma(v, pb[r], d0);
          }
          y[c] += d0;
        }
        for (int r = 0; r < 6; ++r) u[6 * e + r] = tb[r];
      }
      for (int r = 0; r < 6; ++r) q[6 * i + r] = y[r];
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; ++i)
      for (uint64_t k = in_off[i]; k < in_off[i + 1]; ++k)
        for (int r = 0; r < 6; ++r) q[6 * i + r] += u[6 * in_edge[k] + r];
  };
  constexpr size_t kChunk = 6 * 256;
  const size_t nchunks = (N + kChunk - 1) / kChunk;
  std::vector<double> part(nchunks);
  auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < (int64_t)nchunks; ++c) {
      double s = 0.0;
      for (size_t k = c * kChunk; k < std::min(N, (c + 1) * kChunk); ++k) s += a[k] * b[k];
      part[c] = s;
    }
    double s = 0.0;
    for (size_t c = 0; c < nchunks; ++c) s += part[c];
    return s;
  };
  std::vector<double> rc(6 * (size_t)m), yc(6 * (size_t)m);
  auto apply = [&](const std::vector<double>& r, std::vector<double>& z) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      if (in_run[i]) continue;
      for (int a = 0; a < 6; ++a) {
        double s = 0.0;
        for (int b = 0; b < 6; ++b) s += jac[36 * i + a * 6 + b] * r[6 * i + b];
        z[6 * i + a] = s;
      }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < (int64_t)num_clusters; ++c) {
      const size_t rows = 6 * (size_t)cluster_size[c], base = 6 * (size_t)cluster_first[c];
      const double* M = cluster_inverse + cl_off[c];
      for (size_t row = 0; row < rows; ++row) {
        double s = 0.0;
        for (size_t k = 0; k < rows; ++k) s += M[k * rows + row] * r[base + k];
        z[base + row] = s;
      }
    }
    if (m) {
      std::fill(rc.begin(), rc.end(), 0.0);
      for (uint32_t i = 0; i < coarse_nodes; ++i)
        for (int k = 0; k < 6; ++k) rc[6 * (i / coarse_group) + k] += r[6 * (size_t)i + k];
      const size_t M6 = 6 * (size_t)m;
#pragma omp parallel for schedule(static)
      for (int64_t row = 0; row < (int64_t)M6; ++row) {
        double s = 0.0;
        for (size_t k = 0; k < M6; ++k) s += coarse_inverse[k * M6 + row] * rc[k];
        yc[row] = s;
      }
      for (uint32_t i = 0; i < coarse_nodes; ++i)
        for (int k = 0; k < 6; ++k) z[6 * (size_t)i + k] += yc[6 * (i / coarse_group) + k];
    }
  };
  std::vector<double> b(rhs, rhs + N), r(b), z(N), p(N), q(N), xs(N, 0.0);
  const double bnorm = std::sqrt(dot(b, b));
  uint32_t it = 0;
  if (bnorm == 0.0) {
    std::memset(x, 0, N * sizeof(double));
    *iterations = 0;
    return 0;
  }
  apply(r, z);
  p = z;
  double rz = dot(r, z);
  for (uint32_t k = 0; k < max_iterations; ++k) {
    ++it;
    matvec(p, q);
    const double pq = dot(p, q);
    if (!std::isfinite(pq) || pq <= 0.0) return 1;
    const double alpha = rz / pq;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)N; ++i) {
      xs[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    if (std::sqrt(dot(r, r)) <= tol * bnorm) break;
    apply(r, z);
    const double rz_next = dot(r, z);
    const double beta = rz_next / rz;
    rz = rz_next;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)N; ++i) p[i] = z[i] + beta * p[i];
  }
  std::memcpy(x, xs.data(), N * sizeof(double));
  *iterations = it;
  return 0;
}

}  // extern "C"
