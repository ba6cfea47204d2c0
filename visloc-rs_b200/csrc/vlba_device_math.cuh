// vlba_device_math.cuh -- FP64 camera and robust-kernel arithmetic shared by
// the kernel files: quaternion rotation, projection through the radial
// pinhole family with its analytic Jacobian, and the robust kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "vlba_common.cuh"

namespace vlba {
namespace {

// ----------------------------------------------------------------- algebra
// nalgebra UnitQuaternion::to_rotation_matrix (row-major).
__device__ __forceinline__ void quat_to_matrix(const double* q, double* m) {
  const double w = q[0], i = q[1], j = q[2], k = q[3];
  const double ww = w * w, ii = i * i, jj = j * j, kk = k * k;
  const double ij = i * j * 2.0, wk = w * k * 2.0, wj = w * j * 2.0;
  const double ik = i * k * 2.0, jk = j * k * 2.0, wi = w * i * 2.0;
  m[0] = ww + ii - jj - kk;
  m[1] = ij - wk;
  m[2] = wj + ik;
  m[3] = wk + ij;
  m[4] = ww - ii + jj - kk;
  m[5] = jk - wi;
  m[6] = ik - wj;
  m[7] = wi + jk;
  m[8] = ww - ii - jj + kk;
}

// nalgebra UnitQuaternion * Vector3.
__device__ __forceinline__ void quat_rotate(const double* q, const double* p, double* out) {
  const double tx = 2.0 * (q[2] * p[2] - q[3] * p[1]);
  const double ty = 2.0 * (q[3] * p[0] - q[1] * p[2]);
  const double tz = 2.0 * (q[1] * p[1] - q[2] * p[0]);
  const double cx = q[2] * tz - q[3] * ty;
  const double cy = q[3] * tx - q[1] * tz;
  const double cz = q[1] * ty - q[2] * tx;
  out[0] = tx * q[0] + cx + p[0];
  out[1] = ty * q[0] + cy + p[1];
  out[2] = tz * q[0] + cz + p[2];
}

__device__ __forceinline__ double robust_weight(uint32_t kind, double p, double s) {
  if (kind == VLBA_KERNEL_HUBER) return s <= p * p ? 1.0 : p / sqrt(s);
  if (kind == VLBA_KERNEL_CAUCHY) return 1.0 / (1.0 + s / (p * p));
  return 1.0;
}

__device__ __forceinline__ double robust_cost(uint32_t kind, double p, double s) {
  if (kind == VLBA_KERNEL_HUBER) return s <= p * p ? s : 2.0 * p * sqrt(s) - p * p;
  if (kind == VLBA_KERNEL_CAUCHY) return p * p * log(1.0 + s / (p * p));
  return s;
}

// World point -> sensor frame through pose (R, t) and the camera extrinsic.
__device__ __forceinline__ void to_sensor(const double* rt, const DevCamera& cam,
                                          const double* X, double* xs) {
  double xc[3];
  for (int a = 0; a < 3; ++a)
    xc[a] = rt[a * 3] * X[0] + rt[a * 3 + 1] * X[1] + rt[a * 3 + 2] * X[2] + rt[9 + a];
  if (cam.rig) {
    for (int a = 0; a < 3; ++a)
      xs[a] = cam.R[a * 3] * xc[0] + cam.R[a * 3 + 1] * xc[1] + cam.R[a * 3 + 2] * xc[2] +
              cam.t[a];
  } else {
    xs[0] = xc[0];
    xs[1] = xc[1];
    xs[2] = xc[2];
  }
}

// Camera::project for the radial pinhole family (camera.rs:351-432).
__device__ __forceinline__ bool camera_project(const DevCamera& c, const double* p,
                                               double* out) {
  if (!(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]))) return false;
  if (p[2] <= 0.0) return false;
  double x = p[0] / p[2];
  double y = p[1] / p[2];
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

// mono_project_with_jacobian (jacobians.rs:63-113); j row-major 2x3.
__device__ __forceinline__ bool project_jacobian(const DevCamera& c, const double* xc,
                                                 double* pred, double* j) {
  if (!(xc[2] > 0.0)) return false;
  const double z_inv = 1.0 / xc[2];
  if (!c.radial) {
    pred[0] = c.fx * xc[0] / xc[2] + c.cx;
    pred[1] = c.fy * xc[1] / xc[2] + c.cy;
    j[0] = c.fx * z_inv;
    j[1] = 0.0;
    j[2] = -c.fx * xc[0] * z_inv * z_inv;
    j[3] = 0.0;
    j[4] = c.fy * z_inv;
    j[5] = -c.fy * xc[1] * z_inv * z_inv;
    return isfinite(pred[0]) && isfinite(pred[1]);
  }
  const double x = xc[0] / xc[2];
  const double y = xc[1] / xc[2];
  const double r2 = x * x + y * y;
  const double d = 1.0 + c.k1 * r2 + c.k2 * r2 * r2;
  pred[0] = c.fx * (x * d) + c.cx;
  pred[1] = c.fy * (y * d) + c.cy;
  const double g = c.k1 + 2.0 * c.k2 * r2;
  const double d11 = d + 2.0 * x * x * g;
  const double d12 = 2.0 * x * y * g;
  const double d22 = d + 2.0 * y * y * g;
  j[0] = c.fx * d11 * z_inv;
  j[1] = c.fx * d12 * z_inv;
  j[2] = -c.fx * (d11 * x + d12 * y) * z_inv;
  j[3] = c.fy * d12 * z_inv;
  j[4] = c.fy * d22 * z_inv;
  j[5] = -c.fy * (d12 * x + d22 * y) * z_inv;
  bool ok = isfinite(pred[0]) && isfinite(pred[1]);
#pragma unroll
  for (int e = 0; e < 6; ++e) ok = ok && isfinite(j[e]);
  return ok;
}

// d(pinhole pixel)/d(sensor point) rows of camera c at p (z > 0), appended
// as two rows of j (row-major, 3 wide), and the pixel (project_pinhole,
// jacobians.rs:115-124, and pinhole_projection_jacobian, sqrt_qr.rs:445-463:
// no distortion).
__device__ __forceinline__ void pinhole_rows(const DevCamera& c, const double* p, double* pix,
                                             double* j) {
  const double z_inv = 1.0 / p[2];
  pix[0] = c.fx * p[0] * z_inv + c.cx;
  pix[1] = c.fy * p[1] * z_inv + c.cy;
  if (j) {
    j[0] = c.fx * z_inv;
    j[1] = 0.0;
    j[2] = -c.fx * p[0] * z_inv * z_inv;
    j[3] = 0.0;
    j[4] = c.fy * z_inv;
    j[5] = -c.fy * p[1] * z_inv * z_inv;
  }
}

// Residual rows of a stereo observation at its left-sensor point xs and,
// when jl is not null, d r / d X (m x 3, row-major) for the world -> left
// sensor rotation Re.  Returns m (3 or 4), or 0 when a camera sees the point
// at z <= 0 (the observation does not count).
//   kind 1, rectified (normal_equations.rs:496-570): r = (u_l, v_l, u_r)
//     predicted minus observed with u_r = u_l - fx b / z; st = (u_r observed,
//     baseline b).
//   kind 2, general (sqrt_qr.rs:465-518): r = (u_l, v_l, u_r, v_r) with the
//     right point camR.R xs + camR.t (T_right<-left) through camR's pinhole
//     intrinsics; st = the right pixel.
__device__ __forceinline__ int stereo_rows(uint32_t kind, const DevCamera& camL,
                                           const DevCamera& camR, double2 xy, double2 st,
                                           const double* xs, const double* Re, double* r,
                                           double* jl) {
  if (!(xs[2] > 0.0)) return 0;
  double pix[2], jp[6];
  pinhole_rows(camL, xs, pix, jl ? jp : nullptr);
  r[0] = pix[0] - xy.x;
  r[1] = pix[1] - xy.y;
  if (kind == kObsStereo) {
    const double z_inv = 1.0 / xs[2];
    r[2] = (pix[0] - camL.fx * st.y * z_inv) - st.x;
    if (jl) {
      const double j3[3] = {camL.fx * z_inv, 0.0, -camL.fx * (xs[0] - st.y) * z_inv * z_inv};
      for (int b = 0; b < 3; ++b) {
        jl[b] = jp[0] * Re[b] + jp[1] * Re[3 + b] + jp[2] * Re[6 + b];
        jl[3 + b] = jp[3] * Re[b] + jp[4] * Re[3 + b] + jp[5] * Re[6 + b];
        jl[6 + b] = j3[0] * Re[b] + j3[1] * Re[3 + b] + j3[2] * Re[6 + b];
      }
    }
    return 3;
  }
  double xr[3];
  for (int a = 0; a < 3; ++a)
    xr[a] = camR.R[a * 3] * xs[0] + camR.R[a * 3 + 1] * xs[1] + camR.R[a * 3 + 2] * xs[2] + camR.t[a];
  if (!(xr[2] > 0.0)) return 0;
  double pr[2], jr[6];
  pinhole_rows(camR, xr, pr, jl ? jr : nullptr);
  r[2] = pr[0] - st.x;
  r[3] = pr[1] - st.y;
  if (jl) {
    double RR[9];  // world -> right sensor rotation: camR.R Re
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        RR[a * 3 + b] = camR.R[a * 3] * Re[b] + camR.R[a * 3 + 1] * Re[3 + b] + camR.R[a * 3 + 2] * Re[6 + b];
    for (int b = 0; b < 3; ++b) {
      jl[b] = jp[0] * Re[b] + jp[1] * Re[3 + b] + jp[2] * Re[6 + b];
      jl[3 + b] = jp[3] * Re[b] + jp[4] * Re[3 + b] + jp[5] * Re[6 + b];
      jl[6 + b] = jr[0] * RR[b] + jr[1] * RR[3 + b] + jr[2] * RR[6 + b];
      jl[9 + b] = jr[3] * RR[b] + jr[4] * RR[3 + b] + jr[5] * RR[6 + b];
    }
  }
  return 4;
}

}  // namespace
}  // namespace vlba
