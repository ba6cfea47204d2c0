// vlba_kernels.cu -- the Levenberg-Marquardt step on sm_100a.
//
// One LM iteration (trial) of the reference (pipelines/slam/src/bundle/
// lm.rs:356-1009, GPU twin crates/ba-gpu/src/solver.rs:552-690 with the
// shaders of crates/ba-gpu/src/shaders/ba.wgsl) is the kernel sequence
//
//   k_linearize     per observation, after an accepted step: residual,
//                   analytic Jacobian, robust weight; H_o, e_o
//                                                      (ba.wgsl:63-135)
//   k_point_prep    per point: H_ll and g_l from its observations' records
//                   (after an accepted step), damped 3x3 inverse in FP64,
//                   v = H^-1 g; the point's records for the assembly
//                                                      (ba.wgsl:185-243)
//   k_offdiag       per camera pair: S_ij = -sum W_i H^-1 W_j^T, a segmented
//                   reduction over the pair's points (no atomics)
//   k_cam_diag      per camera: S_ii = H_pp + lambda I - sum W H^-1 W^T, the
//                   reduced rhs and the FP64 6x6 Cholesky block-Jacobi inverse
//                                                      (ba.wgsl:141-183, 263-387)
//   k_pcg           persistent: block-Jacobi PCG on S, tiles of S streamed
//                   HBM -> shared memory by TMA bulk copies (ba.wgsl:420-562)
//   k_pose_update   T <- T Exp(xi) in FP64             (solver.rs:599-607)
//   k_cost<true>    back-substitution dl = -H^-1 (g + sum W^T dc), then the
//                   FP64 robust cost and non-projectable count of the trial
//                                                      (ba.wgsl:565-586,
//                                                       solver.rs:696-727)
//   k_decide        LM accept / reject, lambda schedule and convergence tests
//                   in FP64 on the device              (solver.rs:629-682,
//                                                       lm.rs:804-1008)
//
// Precision: Jacobians, H_o, Schur blocks and PCG vectors in FP32 (the Schur
// off-diagonal blocks with compensated FP32 sums); FP64 for the residual, the
// cost, the 3x3 and 6x6 inverses, the diagonal blocks and the PCG scalars.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "vlba_device_math.cuh"
#include "vlba_kernels.cuh"

namespace vlba {
namespace {

// Upper-triangle index of (r, c), r <= c, in a symmetric 6x6.
__host__ __device__ constexpr int ut6(int r, int c) { return r * 6 - (r * (r + 1)) / 2 + c; }

// A pose's 12 derived doubles (R row-major, t; 96 bytes at a 32-byte
// aligned offset) as three 32-byte loads: a warp gathers the poses of 32
// observations, so each load instruction costs one L1 wavefront per pose.
// The table is read-only while the gathering kernels run.
__device__ __forceinline__ void load_rt(const double* rt, double* out) {
#pragma unroll
  for (int q = 0; q < 3; ++q)
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
        : "=d"(out[4 * q]), "=d"(out[4 * q + 1]), "=d"(out[4 * q + 2]), "=d"(out[4 * q + 3])
        : "l"(rt + 4 * q));
}

// S += sign * B^T K B for symmetric or general 3x3 K and B = [I | -[X]x]:
// B^T K B = [[K, -K[X]x], [[X]x K, -[X]x K [X]x]]; full 6x6 row-major.
template <typename T>
__device__ __forceinline__ void btkb(const T* K, T x, T y, T z, T* out) {
  // C = K [X]x : row r of C is K_r x X.
  T C[9];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const T k0 = K[r * 3], k1 = K[r * 3 + 1], k2 = K[r * 3 + 2];
    C[r * 3 + 0] = k1 * z - k2 * y;
    C[r * 3 + 1] = k2 * x - k0 * z;
    C[r * 3 + 2] = k0 * y - k1 * x;
  }
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      out[r * 6 + c] = K[r * 3 + c];
      out[r * 6 + 3 + c] = -C[r * 3 + c];
    }
  // [X]x K (column c is X x K_c) and [X]x C.
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T k0 = K[c], k1 = K[3 + c], k2 = K[6 + c];
    out[18 + c] = y * k2 - z * k1;
    out[24 + c] = z * k0 - x * k2;
    out[30 + c] = x * k1 - y * k0;
    const T c0 = C[c], c1 = C[3 + c], c2 = C[6 + c];
    out[18 + 3 + c] = -(y * c2 - z * c1);
    out[24 + 3 + c] = -(z * c0 - x * c2);
    out[30 + 3 + c] = -(x * c1 - y * c0);
  }
}

// Fixed-order block reductions (deterministic for a given block size).
template <typename T, int N>
__device__ __forceinline__ T block_sum(T v, T* red) {
  red[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = N / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  const T out = red[0];
  __syncthreads();
  return out;
}

template <int N>
__device__ __forceinline__ double block_max(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = N / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const double out = red[0];
  __syncthreads();
  return out;
}

// 6x6 SPD inverse by Cholesky in FP64; false if not positive definite.
__device__ bool chol_inverse6(const double* a, double* inv) {
  double L[36];
#pragma unroll
  for (int e = 0; e < 36; ++e) L[e] = a[e];
  for (int j = 0; j < 6; ++j) {
    double s = L[j * 6 + j];
    for (int q = 0; q < j; ++q) s -= L[j * 6 + q] * L[j * 6 + q];
    if (!(s > 0.0) || !isfinite(s)) return false;
    const double ljj = sqrt(s);
    L[j * 6 + j] = ljj;
    for (int i = j + 1; i < 6; ++i) {
      double t = L[i * 6 + j];
      for (int q = 0; q < j; ++q) t -= L[i * 6 + q] * L[j * 6 + q];
      L[i * 6 + j] = t / ljj;
    }
  }
  for (int c = 0; c < 6; ++c) {
    double y[6];
    for (int i = 0; i < 6; ++i) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int q = 0; q < i; ++q) s -= L[i * 6 + q] * y[q];
      y[i] = s / L[i * 6 + i];
    }
    for (int ii = 5; ii >= 0; --ii) {
      double s = y[ii];
      for (int q = ii + 1; q < 6; ++q) s -= L[q * 6 + ii] * inv[q * 6 + c];
      inv[ii * 6 + c] = s / L[ii * 6 + ii];
    }
  }
  return true;
}

// 32-byte vector load (read-only path) and store: one request per 32-byte
// sector on sm_100.  The address must be 32-byte aligned.
__device__ __forceinline__ void ld8(const float4* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}
__device__ __forceinline__ void st8(float4* p, float4 a, float4 b) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(a.x), "f"(a.y),
               "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
               : "memory");
}

// ------------------------------------------------------------ pose table
__global__ void __launch_bounds__(256) k_pose_table(Dev d) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < d.num_poses;
       p += gridDim.x * blockDim.x) {
    const uint32_t cur = d.ctrl[d.pose_prob[p]].cur;
    double q[4], m[9];
#pragma unroll
    for (int a = 0; a < 4; ++a) q[a] = d.pose_q[cur][4 * p + a];
    quat_to_matrix(q, m);
    double* rt = d.pose_rt[cur] + 12 * (size_t)p;
#pragma unroll
    for (int a = 0; a < 9; ++a) rt[a] = m[a];
#pragma unroll
    for (int a = 0; a < 3; ++a) rt[9 + a] = d.pose_t[cur][3 * p + a];
  }
}

// 32-byte load and store of four doubles (the point records are 32-byte
// aligned and read-only while the kernels that read them run).
__device__ __forceinline__ void ld4d(const double* p, double* o) {
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
      : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3])
      : "l"(p));
}
__device__ __forceinline__ void st4d(double* p, double a, double b, double c, double e) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(e)
               : "memory");
}
// Two f32 values in one double's bits (low word first).
__device__ __forceinline__ double pack2f(float lo, float hi) {
  return __longlong_as_double(((long long)__float_as_uint(hi) << 32) | (long long)__float_as_uint(lo));
}
__device__ __forceinline__ float2 unpack2f(double v) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  return make_float2(__uint_as_float((uint32_t)u), __uint_as_float((uint32_t)(u >> 32)));
}

// ------------------------------------------------------------- linearize
// One thread per observation (point-major order): the residual and analytic
// Jacobian in FP64, the IRLS weight, and the observation's H_o and e_o.  The
// point sums H_ll and g_l are formed by k_point_prep from these records.
__global__ void __launch_bounds__(256, 3) k_linearize(Dev d) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < d.num_obs;
       k += gridDim.x * blockDim.x) {
    const uint32_t l = d.obs_point[k];
    const uint32_t P = d.num_problems == 1 ? 0u : d.point_prob[l];
    const Ctrl& c = d.ctrl[P];
    if (c.done || !c.relinearize) continue;
    const uint32_t cur = c.cur;
    const LmParams& lp = d.params[P];
    double X[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[a] = d.points[cur][3 * (size_t)l + a];
    {
      const uint32_t pose = d.obs_pose[k];
      const DevCamera& cam = d.cameras[d.obs_cam[k]];
      double rt[12];
      load_rt(d.pose_rt[cur] + 12 * (size_t)pose, rt);
      double xs[3], pred[2], jpi[6];
      to_sensor(rt, cam, X, xs);
      float h[6] = {0, 0, 0, 0, 0, 0}, e[3] = {0, 0, 0};
      float wf = 0.0f;
      const uint32_t kind = d.obs_kind ? d.obs_kind[k] : kObsMono;
      if (kind != kObsMono) {
        // Stereo: 3 or 4 residual rows through the same J_l factor.
        double Re[9];
        if (cam.rig) {
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
              Re[a * 3 + b] = cam.R[a * 3] * rt[b] + cam.R[a * 3 + 1] * rt[3 + b] +
                              cam.R[a * 3 + 2] * rt[6 + b];
        } else {
#pragma unroll
          for (int a = 0; a < 9; ++a) Re[a] = rt[a];
        }
        double r[4], jl[12];
        const int m = stereo_rows(kind, cam, d.cameras[d.obs_rcam[k]], d.obs_xy[k], d.obs_st[k], xs,
                                  Re, r, jl);
        if (m) {
          double ss = 0.0;
          for (int i = 0; i < m; ++i) ss += r[i] * r[i];
          double w = robust_weight(lp.robust_kernel, lp.robust_parameter, ss);
          if (d.obs_w) w *= d.obs_w[k];
          wf = (float)w;
          float jf[12], rf[4];
          for (int i = 0; i < 3 * m; ++i) jf[i] = (float)jl[i];
          for (int i = 0; i < m; ++i) rf[i] = (float)r[i];
          const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
          for (int q = 0; q < 6; ++q) {
            float acc = 0.0f;
            for (int i = 0; i < m; ++i) acc += jf[3 * i + ab[q][0]] * jf[3 * i + ab[q][1]];
            h[q] = wf * acc;
          }
          for (int a = 0; a < 3; ++a) {
            float acc = 0.0f;
            for (int i = 0; i < m; ++i) acc += jf[3 * i + a] * rf[i];
            e[a] = wf * acc;
          }
        }
      } else if (project_jacobian(cam, xs, pred, jpi)) {
        const double2 xy = d.obs_xy[k];
        const double rx = pred[0] - xy.x, ry = pred[1] - xy.y;
        // The robust IRLS weight times the external weight
        // (normal_equations.rs:458).
        double w = robust_weight(lp.robust_kernel, lp.robust_parameter, rx * rx + ry * ry);
        if (d.obs_w) w *= d.obs_w[k];
        // Effective rotation world -> sensor.
        double Re[9];
        if (cam.rig) {
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
              Re[a * 3 + b] = cam.R[a * 3] * rt[b] + cam.R[a * 3 + 1] * rt[3 + b] +
                              cam.R[a * 3 + 2] * rt[6 + b];
        } else {
#pragma unroll
          for (int a = 0; a < 9; ++a) Re[a] = rt[a];
        }
        // J_l = J_pi R (2x3), FP32.
        float jl[6];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b)
            jl[a * 3 + b] = (float)(jpi[a * 3] * Re[b] + jpi[a * 3 + 1] * Re[3 + b] +
                                    jpi[a * 3 + 2] * Re[6 + b]);
        wf = (float)w;
        const float r0 = (float)rx, r1 = (float)ry;
        h[0] = wf * (jl[0] * jl[0] + jl[3] * jl[3]);
        h[1] = wf * (jl[0] * jl[1] + jl[3] * jl[4]);
        h[2] = wf * (jl[0] * jl[2] + jl[3] * jl[5]);
        h[3] = wf * (jl[1] * jl[1] + jl[4] * jl[4]);
        h[4] = wf * (jl[1] * jl[2] + jl[4] * jl[5]);
        h[5] = wf * (jl[2] * jl[2] + jl[5] * jl[5]);
        e[0] = wf * (jl[0] * r0 + jl[3] * r1);
        e[1] = wf * (jl[1] * r0 + jl[4] * r1);
        e[2] = wf * (jl[2] * r0 + jl[5] * r1);
      }
      d.obs_h[2 * (size_t)k] = make_float4(h[0], h[1], h[2], h[3]);
      d.obs_h[2 * (size_t)k + 1] = make_float4(h[4], h[5], __uint_as_float(l), (float)X[2]);
      d.obs_e[k] = make_float4(e[0], e[1], e[2], wf);
    }
  }
}

// ------------------------------------------------------------ point prep
// Observations a chunked kernel stages through shared memory per pass.
constexpr uint32_t kObsStage = 1024;

// Damped landmark inverse (FP64 cofactors, nalgebra Matrix3::try_inverse:
// singular iff det == 0) and v = H^-1 g.  A singular or fixed point gets a
// zero inverse, which drops it from the reduced system and back-substitution
// exactly as the reference's `continue` does (normal_equations.rs:1662-1668).
__global__ void __launch_bounds__(256) k_point_prep(Dev d) {
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < d.num_points;
       l += gridDim.x * blockDim.x) {
    const uint32_t P = d.num_problems == 1 ? 0u : d.point_prob[l];
    const Ctrl& c = d.ctrl[P];
    if (c.done) continue;
    const uint32_t cur = c.cur;
    const double lambda = c.lambda;
    const float X0 = (float)d.points[cur][3 * (size_t)l];
    const float X1 = (float)d.points[cur][3 * (size_t)l + 1];
    const float X2 = (float)d.points[cur][3 * (size_t)l + 2];
    double inv[6] = {0, 0, 0, 0, 0, 0}, v[3] = {0, 0, 0}, g[3] = {0, 0, 0};
    double ci[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // the FP64 record's inverse and v
    float ok = 0.0f;
    if (d.point_var[l] && c.relinearize) {
      // H_ll and g_l of the new linearisation: the observations' records
      // summed in observation order (FP64 sums, stored FP32).
      double hl[6] = {0, 0, 0, 0, 0, 0}, gl[3] = {0, 0, 0};
      for (uint32_t k = d.pt_off[l]; k < d.pt_off[l + 1]; ++k) {
        const float4 h0 = d.obs_h[2 * (size_t)k], h1 = d.obs_h[2 * (size_t)k + 1];
        const float4 e = d.obs_e[k];
        hl[0] += h0.x;
        hl[1] += h0.y;
        hl[2] += h0.z;
        hl[3] += h0.w;
        hl[4] += h1.x;
        hl[5] += h1.y;
        gl[0] += e.x;
        gl[1] += e.y;
        gl[2] += e.z;
      }
      float* ph = d.pt_h + 9 * (size_t)l;
#pragma unroll
      for (int a = 0; a < 6; ++a) ph[a] = (float)hl[a];
#pragma unroll
      for (int a = 0; a < 3; ++a) ph[6 + a] = (float)gl[a];
    }
    if (d.point_var[l]) {
      const float* ph = d.pt_h + 9 * (size_t)l;
      double a = ph[0], b = ph[1], cc = ph[2], dd = ph[3], e = ph[4], f = ph[5];
      g[0] = ph[6];
      g[1] = ph[7];
      g[2] = ph[8];
      if (lambda > 0.0) {
        a += lambda;
        dd += lambda;
        f += lambda;
      }
      // Symmetric [[a b c] [b d e] [c e f]].
      const double m22 = dd * f - e * e;   // minor (1,1)-(2,2)
      const double m12 = b * f - e * cc;   // minor rows 1,2 cols 0,2
      const double m11 = b * e - dd * cc;  // minor rows 1,2 cols 0,1
      const double det = a * m22 - b * m12 + cc * m11;
      if (det != 0.0 && isfinite(det)) {
        inv[0] = m22 / det;
        inv[1] = (cc * e - f * b) / det;
        inv[2] = (b * e - dd * cc) / det;
        inv[3] = (a * f - cc * cc) / det;
        inv[4] = (cc * b - e * a) / det;
        inv[5] = (a * dd - b * b) / det;
        v[0] = inv[0] * g[0] + inv[1] * g[1] + inv[2] * g[2];
        v[1] = inv[1] * g[0] + inv[3] * g[1] + inv[4] * g[2];
        v[2] = inv[2] * g[0] + inv[4] * g[1] + inv[5] * g[2];
        ok = 1.0f;
        // The FP64 copy the camera diagonal and the back-substitution read
        // (point_inverse64): the same cofactors over one reciprocal of the
        // determinant, formed once per point instead of per observation.
        const double rdet = 1.0 / det;
        const double i0 = m22 * rdet, i1 = (cc * e - f * b) * rdet, i2 = (b * e - dd * cc) * rdet,
                     i3 = (a * f - cc * cc) * rdet, i4 = (cc * b - e * a) * rdet,
                     i5 = (a * dd - b * b) * rdet;
        ci[0] = i0;
        ci[1] = i1;
        ci[2] = i2;
        ci[3] = i3;
        ci[4] = i4;
        ci[5] = i5;
        ci[6] = i0 * g[0] + i1 * g[1] + i2 * g[2];
        ci[7] = i1 * g[0] + i3 * g[1] + i4 * g[2];
        ci[8] = i2 * g[0] + i4 * g[1] + i5 * g[2];
      }
    }
    {
      double* pc = d.pt_c + 12 * (size_t)l;
      st4d(pc, ci[0], ci[1], ci[2], ci[3]);
      st4d(pc + 4, ci[4], ci[5], ci[6], ci[7]);
      st4d(pc + 8, ci[8], pack2f(X0, X1), pack2f(X2, ok), 0.0);
    }
    float4* ps = d.pt_s + 4 * (size_t)l;
    const float4 p0 = make_float4((float)inv[0], (float)inv[1], (float)inv[2], (float)inv[3]);
    const float4 p1 = make_float4((float)inv[4], (float)inv[5], X0, X1);
    ps[0] = p0;
    ps[1] = p1;
    // The same 32 bytes as one record for the off-diagonal assembly.
    st8(d.pt_p + 2 * (size_t)l, p0, p1);
    ps[2] = make_float4(X2, (float)v[0], (float)v[1], (float)v[2]);
    ps[3] = make_float4((float)g[0], (float)g[1], (float)g[2], ok);
  }
}

// The damped inverse of point l's H_ll and v = H^-1 g in FP64, as
// k_point_prep formed them this trial from the FP64 sums it stores as FP32
// (its cofactor formulas over one reciprocal of the determinant; it rounds
// its own inverse to FP32 for the other kernels).  Read only for points
// whose determinant is nonzero.  The camera diagonal needs this precision:
// when a point has one contributing observation (its others weighted 0, or
// observed twice by one camera), H_ll is H_o of rank 2 and
// H_o - H_o (H_ll + lambda I)^-1 H_o cancels down to O(lambda), far below
// what an FP32 inverse with entries near 1/lambda resolves.
__device__ __forceinline__ void point_inverse64(const Dev& d, uint32_t l, double* M, double* v) {
  double c[12];
  const double* pc = d.pt_c + 12 * (size_t)l;
  ld4d(pc, c);
  ld4d(pc + 4, c + 4);
  ld4d(pc + 8, c + 8);
  M[0] = c[0]; M[1] = c[1]; M[2] = c[2];
  M[3] = c[1]; M[4] = c[3]; M[5] = c[4];
  M[6] = c[2]; M[7] = c[4]; M[8] = c[5];
  v[0] = c[6];
  v[1] = c[7];
  v[2] = c[8];
}

// ------------------------------------------------- off-diagonal Schur blocks
// One group of G lanes per camera pair (i, j), i > j: lanes stride the pair's
// points in order, each accumulating -B^T H_i H^-1 H_j B with compensated
// (Kahan) FP32 sums, then a fixed butterfly over the group.  Deterministic,
// no atomics; the destination is the block's slot in its dense tile (and the
// mirrored slot inside a diagonal tile).
//
// A term reads three 32-byte records with one request each -- H_i (with the
// point's z), the point's record (damped inverse and x, y), and H_j --
// addressed by the pair entry and the term's point stored beside it, whose
// successors are fetched while the current term is computed.  Warps take the blocks in the order of
// ord_range / ord_dst (plan order, sorted by length within windows of 256
// blocks, each block's range and destination stored at its place): the groups of
// a warp then loop about as many times (lane-pass efficiency 0.82 -> 0.99 on
// ring-4m) while the blocks running at one time stay those of nearby rows.
// LONG: the blocks of the long list (at least kLongBlockTerms terms) on G
// lanes each; otherwise the other blocks in the length-sorted order.
template <int G, bool LONG>
__global__ void __launch_bounds__(256, 2) k_offdiag(Dev d) {
  constexpr int kPerWarp = 32 / G;
  const uint32_t lane = threadIdx.x % G;
  const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const uint32_t warps_total = gridDim.x * blockDim.x / 32;
  const uint32_t tile_floats = d.tb * d.tb * kBlock;
  const uint32_t nblocks = LONG ? d.num_long_blocks : d.num_offdiag_blocks;
  const uint32_t nwb = (nblocks + kPerWarp - 1) / kPerWarp;
  for (uint32_t wb = warp_global; wb < nwb; wb += warps_total) {
    const uint32_t q = wb * kPerWarp + (threadIdx.x % 32) / G;
    bool valid = q < nblocks;
    uint2 dst = make_uint2(kNone, kNone), pr = make_uint2(0u, 0u);
    uint32_t c0 = 0, c1 = 0, pt = 0;
    if (valid) {
      // The block's range and first pair go out beside its problem's status
      // (a single problem's is the same for every block): the pair loads do
      // not wait for the lookup of the problem.
      const uint2 range = LONG ? d.long_range[q] : d.ord_range[q];
      dst = LONG ? d.long_dst[q] : d.ord_dst[q];
      c0 = range.x;
      c1 = range.y;
      if (!LONG && c1 - c0 >= kLongBlockTerms) c1 = c0;  // the long kernel's block
      if (c0 + lane < c1) {
        pr = d.pairs[c0 + lane];
        pt = d.pair_pt[c0 + lane];
      }
      const uint32_t P =
          d.num_problems == 1 ? 0u : d.tr_prob[d.tile_ij[dst.x / tile_floats] >> 16];
      valid = !d.ctrl[P].done && (LONG || range.y - range.x < kLongBlockTerms);
    }
    float acc[36], cmp[36];
#pragma unroll
    for (int e = 0; e < 36; ++e) {
      acc[e] = 0.0f;
      cmp[e] = 0.0f;
    }
    if (valid && c0 + lane < c1) {
      for (uint32_t cidx = c0 + lane; cidx < c1; cidx += G) {
        float4 a0, a1, p0, p1, b0, b1;
        ld8(d.obs_h + 2 * (size_t)pr.x, a0, a1);
        ld8(d.pt_p + 2 * (size_t)pt, p0, p1);
        ld8(d.obs_h + 2 * (size_t)pr.y, b0, b1);
        if (cidx + G < c1) {
          pr = d.pairs[cidx + G];
          pt = d.pair_pt[cidx + G];
        }
        const float Hi[9] = {a0.x, a0.y, a0.z, a0.y, a0.w, a1.x, a0.z, a1.x, a1.y};
        const float Hj[9] = {b0.x, b0.y, b0.z, b0.y, b0.w, b1.x, b0.z, b1.x, b1.y};
        const float Mi[9] = {p0.x, p0.y, p0.z, p0.y, p0.w, p1.x, p0.z, p1.x, p1.y};
        float M[9], K[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc)
            M[r * 3 + cc] = Mi[r * 3] * Hj[cc] + Mi[r * 3 + 1] * Hj[3 + cc] +
                            Mi[r * 3 + 2] * Hj[6 + cc];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc)
            K[r * 3 + cc] = Hi[r * 3] * M[cc] + Hi[r * 3 + 1] * M[3 + cc] +
                            Hi[r * 3 + 2] * M[6 + cc];
        float blk[36];
        btkb<float>(K, p1.z, p1.w, a1.w, blk);
#pragma unroll
        for (int e = 0; e < 36; ++e) {  // acc -= blk, Kahan compensated
          const float y = -blk[e] - cmp[e];
          const float t = acc[e] + y;
          cmp[e] = (t - acc[e]) - y;
          acc[e] = t;
        }
      }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
      for (int e = 0; e < 36; ++e) acc[e] += __shfl_xor_sync(0xffffffffu, acc[e], off, G);
    if (valid) {
#pragma unroll
      for (int e = 0; e < 36; ++e) {
        if ((uint32_t)(e % G) == lane) {
          d.tiles[dst.x + e] = acc[e];
          if (dst.y != kNone) d.tiles[dst.y + (e % 6) * 6 + e / 6] = acc[e];
        }
      }
    }
  }
}

// acc[ut6(r,c)] += sign * (B^T K B)[r][c] for r <= c (K general 3x3).
__device__ __forceinline__ void add_btkb_upper(const double* K, double x, double y, double z,
                                               double* acc, double sign) {
  double C[9];  // C = K [X]x, row r = K_r x X
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const double k0 = K[r * 3], k1 = K[r * 3 + 1], k2 = K[r * 3 + 2];
    C[r * 3 + 0] = k1 * z - k2 * y;
    C[r * 3 + 1] = k2 * x - k0 * z;
    C[r * 3 + 2] = k0 * y - k1 * x;
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
#pragma unroll
    for (int c = r; c < 3; ++c) acc[ut6(r, c)] += sign * K[r * 3 + c];
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[ut6(r, 3 + c)] -= sign * C[r * 3 + c];
  }
  // Bottom-right -[X]x C: column c is -(X x C_c).
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double c0 = C[c], c1 = C[3 + c], c2 = C[6 + c];
    const double b0 = -(y * c2 - z * c1), b1 = -(z * c0 - x * c2), b2 = -(x * c1 - y * c0);
    if (0 <= c) acc[ut6(3, 3 + c)] += sign * b0;
    if (1 <= c) acc[ut6(4, 3 + c)] += sign * b1;
    if (2 <= c) acc[ut6(5, 3 + c)] += sign * b2;
  }
}

__device__ __forceinline__ double quad3(const double* H, double a, double b, double c) {
  return a * (H[0] * a + H[1] * b + H[2] * c) + b * (H[3] * a + H[4] * b + H[5] * c) +
         c * (H[6] * a + H[7] * b + H[8] * c);
}

// --------------------------------------------------- camera diagonal blocks
// One block of 128 threads per variable camera: FP64 sums of
//   S_ii = sum_o B^T (H_o - H_o H^-1 H_o) B + lambda I   (H_pp minus Schur)
//   b_i  = sum_o B^T (H_o v - e_o)                        (-g_p + sum W v)
// then the FP64 Cholesky inverse of S_ii as the block-Jacobi preconditioner
// (ba.wgsl:263-387; fallback to the inverse damped diagonal, ba.wgsl:375-383).
// Thread t adds the camera's observations t, t + 128, ... in list (= point)
// order, so the blocks running at one time read the records of nearby
// points.  An observation's records and its point's 96-byte FP64 record are
// one gather away (the point stored beside the list, cam_pt), five loads of
// 16 and 32 bytes issued together; the next observation's indices are loaded
// while this one is summed (measured on ring-4m: 270 -> 210 us against the
// records read through the observation's own point index; the point's data
// in one record instead of three took another 36 us off the assembly).
// Warps sum by a butterfly, then in warp order: fixed order throughout.
constexpr int kDiagThreads = 128;
constexpr int kDiagAcc = 27;  // 21 upper S, 6 rhs

// Fixed-order block sum of n per-thread values: butterfly within each warp,
// then the warps' sums in warp order; the totals land in tot[0, n).
template <int N>
__device__ __forceinline__ void diag_block_sum(double* acc, double* red, double* tot) {
#pragma unroll
  for (int e = 0; e < N; ++e) {
    double v = acc[e];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    acc[e] = v;
  }
  const int warp = threadIdx.x / 32;
  if ((threadIdx.x % 32) == 0) {
#pragma unroll
    for (int e = 0; e < N; ++e) red[warp * N + e] = acc[e];
  }
  __syncthreads();
  if (threadIdx.x < (unsigned)N) {
    double t = 0.0;
    for (int w = 0; w < kDiagThreads / 32; ++w) t += red[w * N + threadIdx.x];
    tot[threadIdx.x] = t;
  }
  __syncthreads();
}

// Observation k (of point l)'s terms of S_ii and b_i.
__device__ __forceinline__ void cam_diag_obs(const Dev& d, uint32_t k, uint32_t l, double* acc) {
  float4 h0, h1;
  ld8(d.obs_h + 2 * (size_t)k, h0, h1);
  const float4 ev = __ldg(d.obs_e + k);
  // The point's 96-byte record: FP64 damped inverse and v, X and the ok flag.
  double c[12];
  const double* pc = d.pt_c + 12 * (size_t)l;
  ld4d(pc, c);
  ld4d(pc + 4, c + 4);
  ld4d(pc + 8, c + 8);
  const float2 xy = unpack2f(c[9]), zo = unpack2f(c[10]);
  const double H[9] = {h0.x, h0.y, h0.z, h0.y, h0.w, h1.x, h0.z, h1.x, h1.y};
  const double X = xy.x, Y = xy.y, Z = zo.x;
  double K[9], w[3];
  if (zo.y != 0.0f) {
    const double Mi[9] = {c[0], c[1], c[2], c[1], c[3], c[4], c[2], c[4], c[5]};
    double M[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
        M[r * 3 + cc] = Mi[r * 3] * H[cc] + Mi[r * 3 + 1] * H[3 + cc] + Mi[r * 3 + 2] * H[6 + cc];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
        K[r * 3 + cc] = H[r * 3 + cc] - (H[r * 3] * M[cc] + H[r * 3 + 1] * M[3 + cc] +
                                         H[r * 3 + 2] * M[6 + cc]);
    const double v0 = c[6], v1 = c[7], v2 = c[8];
    w[0] = H[0] * v0 + H[1] * v1 + H[2] * v2 - ev.x;
    w[1] = H[3] * v0 + H[4] * v1 + H[5] * v2 - ev.y;
    w[2] = H[6] * v0 + H[7] * v1 + H[8] * v2 - ev.z;
  } else {
#pragma unroll
    for (int q = 0; q < 9; ++q) K[q] = H[q];
    w[0] = -(double)ev.x;
    w[1] = -(double)ev.y;
    w[2] = -(double)ev.z;
  }
  add_btkb_upper(K, X, Y, Z, acc, 1.0);
  acc[21] += w[0];
  acc[22] += w[1];
  acc[23] += w[2];
  acc[24] += Y * w[2] - Z * w[1];
  acc[25] += Z * w[0] - X * w[2];
  acc[26] += X * w[1] - Y * w[0];
}

__global__ void __launch_bounds__(kDiagThreads) k_cam_diag(Dev d) {
  __shared__ double red[(kDiagThreads / 32) * kDiagAcc];
  __shared__ double tot[kDiagAcc];
  __shared__ int s_fail;
  const uint32_t t = threadIdx.x;
  for (uint32_t s = blockIdx.x; s < d.num_var_cams; s += gridDim.x) {
    const uint32_t P = d.num_problems == 1 ? 0u : d.slot_prob[s];
    if (d.ctrl[P].done) continue;
    const uint32_t o0 = d.cam_off[s], o1 = d.cam_off[s + 1];
    double acc[kDiagAcc];
#pragma unroll
    for (int e = 0; e < kDiagAcc; ++e) acc[e] = 0.0;
    uint32_t idx = o0 + t, k = kNone, l = 0u;
    if (idx < o1) {
      k = d.cam_obs[idx];
      l = d.cam_pt[idx];
    }
    while (k != kNone) {
      const uint32_t nidx = idx + kDiagThreads;
      uint32_t nk = kNone, nl = 0u;
      if (nidx < o1) {
        nk = d.cam_obs[nidx];
        nl = d.cam_pt[nidx];
      }
      cam_diag_obs(d, k, l, acc);
      idx = nidx;
      k = nk;
      l = nl;
    }
    // Same-camera pairs k != k' of one point (a point observed twice by a
    // camera): -B^T H_k H^-1 H_k' B, both orders listed.
    for (uint32_t i = d.dup_off[s] + t; i < d.dup_off[s + 1]; i += kDiagThreads) {
      const uint2 pr = d.dup_pairs[i];
      const float4 a0 = d.obs_h[2 * (size_t)pr.x], a1 = d.obs_h[2 * (size_t)pr.x + 1];
      const float4 b0 = d.obs_h[2 * (size_t)pr.y], b1 = d.obs_h[2 * (size_t)pr.y + 1];
      const uint32_t pl = __float_as_uint(a1.z);
      const float4 s1 = d.pt_s[4 * (size_t)pl + 1], s2 = d.pt_s[4 * (size_t)pl + 2];
      if (d.pt_s[4 * (size_t)pl + 3].w == 0.0f) continue;  // no inverse: no Schur term
      const double Hi[9] = {a0.x, a0.y, a0.z, a0.y, a0.w, a1.x, a0.z, a1.x, a1.y};
      const double Hj[9] = {b0.x, b0.y, b0.z, b0.y, b0.w, b1.x, b0.z, b1.x, b1.y};
      double Mi[9], vv[3];
      point_inverse64(d, pl, Mi, vv);
      double M[9], K[9];
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc)
          M[r * 3 + cc] = Mi[r * 3] * Hj[cc] + Mi[r * 3 + 1] * Hj[3 + cc] + Mi[r * 3 + 2] * Hj[6 + cc];
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc)
          K[r * 3 + cc] = Hi[r * 3] * M[cc] + Hi[r * 3 + 1] * M[3 + cc] + Hi[r * 3 + 2] * M[6 + cc];
      add_btkb_upper(K, (double)s1.z, (double)s1.w, (double)s2.x, acc, -1.0);
    }
    diag_block_sum<kDiagAcc>(acc, red, tot);
    const double lambda = d.ctrl[P].lambda;
    if (t == 0) {
      double S[36], inv[36];
      for (int r = 0; r < 6; ++r)
        for (int cc = 0; cc < 6; ++cc) {
          double v = r <= cc ? tot[ut6(r, cc)] : tot[ut6(cc, r)];
          if (r == cc && lambda > 0.0) v += lambda;
          S[r * 6 + cc] = v;
        }
      float* blk = d.tiles + d.diag_dst[s];
      for (int e = 0; e < 36; ++e) blk[e] = (float)S[e];
      for (int a = 0; a < 6; ++a) d.rhs[6 * (size_t)s + a] = (float)tot[21 + a];
      const bool ok = chol_inverse6(S, inv);
      if (ok)
        for (int e = 0; e < 36; ++e) d.minv[36 * (size_t)s + e] = (float)inv[e];
      s_fail = ok ? 0 : 1;
    }
    __syncthreads();
    if (s_fail) {
      // Not positive definite: the inverse damped diagonal of B^T H B over
      // the camera's observations (H_aa, then the quadratic forms
      // (X x e_a)^T H (X x e_a)), summed only for such a camera.
      double g[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      for (uint32_t i = o0 + t; i < o1; i += kDiagThreads) {
        const uint32_t kk = d.cam_obs[i], pl = d.cam_pt[i];
        const float4 h0 = d.obs_h[2 * (size_t)kk], h1 = d.obs_h[2 * (size_t)kk + 1];
        const float4 s1 = d.pt_s[4 * (size_t)pl + 1], s2 = d.pt_s[4 * (size_t)pl + 2];
        const double H[9] = {h0.x, h0.y, h0.z, h0.y, h0.w, h1.x, h0.z, h1.x, h1.y};
        const double X = s1.z, Y = s1.w, Z = s2.x;
        g[0] += H[0];
        g[1] += H[4];
        g[2] += H[8];
        g[3] += quad3(H, 0.0, Z, -Y);
        g[4] += quad3(H, -Z, 0.0, X);
        g[5] += quad3(H, Y, -X, 0.0);
      }
      diag_block_sum<6>(g, red, tot);
      if (t == 0) {
        for (int e = 0; e < 36; ++e) d.minv[36 * (size_t)s + e] = 0.0f;
        for (int a = 0; a < 6; ++a)
          d.minv[36 * (size_t)s + a * 7] = (float)(1.0 / fmax(tot[a] + lambda, 1e-20));
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------- pose update
// T' = T * Exp(xi) in FP64 (SE3::exp + compose, se3.rs:32-37,72-82,109-121).
__global__ void __launch_bounds__(256) k_pose_update(Dev d) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < d.num_poses;
       p += gridDim.x * blockDim.x) {
    const uint32_t P = d.pose_prob[p];
    Ctrl& c = d.ctrl[P];
    if (c.done) continue;
    const uint32_t cur = c.cur, nxt = cur ^ 1u;
    double q[4], t[3];
#pragma unroll
    for (int a = 0; a < 4; ++a) q[a] = d.pose_q[cur][4 * (size_t)p + a];
#pragma unroll
    for (int a = 0; a < 3; ++a) t[a] = d.pose_t[cur][3 * (size_t)p + a];
    double step = 0.0;
    const uint32_t slot = d.pose_slot[p];
    if (slot != kNone) {
      double xi[6];
      double nn = 0.0;
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        xi[a] = (double)d.x[6 * (size_t)slot + a];
        nn += xi[a] * xi[a];
      }
      step = sqrt(nn);
      if (!isfinite(step)) c.nonfinite = 1u;
      // Exp: rotation = exp(omega / 2) as a quaternion (nalgebra
      // from_scaled_axis), translation = V(omega) rho.
      const double hx = xi[3] / 2.0, hy = xi[4] / 2.0, hz = xi[5] / 2.0;
      const double hn = hx * hx + hy * hy + hz * hz;
      double qe[4] = {1.0, 0.0, 0.0, 0.0};
      const double eps = 2.220446049250313e-16;
      if (hn > eps * eps) {
        const double n = sqrt(hn);
        const double sn = sin(n) / n;
        qe[0] = cos(n);
        qe[1] = hx * sn;
        qe[2] = hy * sn;
        qe[3] = hz * sn;
      }
      const double wx = xi[3], wy = xi[4], wz = xi[5];
      const double th2 = wx * wx + wy * wy + wz * wz;
      double ca, cb;
      if (th2 < 1e-10) {
        ca = 0.5;
        cb = 1.0 / 6.0;
      } else {
        const double th = sqrt(th2);
        ca = (1.0 - cos(th)) / th2;
        cb = (th - sin(th)) / (th * th2);
      }
      const double S[9] = {0.0, -wz, wy, wz, 0.0, -wx, -wy, wx, 0.0};
      double te[3];
      for (int a = 0; a < 3; ++a) {
        double v = 0.0;
        for (int b = 0; b < 3; ++b) {
          double s2 = 0.0;
          for (int k = 0; k < 3; ++k) s2 += S[a * 3 + k] * S[k * 3 + b];
          const double vab = (a == b ? 1.0 : 0.0) + ca * S[a * 3 + b] + cb * s2;
          v += vab * xi[b];
        }
        te[a] = v;
      }
      const double nq[4] = {q[0] * qe[0] - q[1] * qe[1] - q[2] * qe[2] - q[3] * qe[3],
                            q[0] * qe[1] + q[1] * qe[0] + q[2] * qe[3] - q[3] * qe[2],
                            q[0] * qe[2] - q[1] * qe[3] + q[2] * qe[0] + q[3] * qe[1],
                            q[0] * qe[3] + q[1] * qe[2] - q[2] * qe[1] + q[3] * qe[0]};
      double rte[3];
      quat_rotate(q, te, rte);
      for (int a = 0; a < 3; ++a) t[a] = rte[a] + t[a];
      for (int a = 0; a < 4; ++a) q[a] = nq[a];
    }
    d.pose_step[p] = step;
    double m[9];
    quat_to_matrix(q, m);
    double* rt = d.pose_rt[nxt] + 12 * (size_t)p;
#pragma unroll
    for (int a = 0; a < 9; ++a) rt[a] = m[a];
#pragma unroll
    for (int a = 0; a < 4; ++a) d.pose_q[nxt][4 * (size_t)p + a] = q[a];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      d.pose_t[nxt][3 * (size_t)p + a] = t[a];
      rt[9 + a] = t[a];
    }
  }
}

// ------------------------------------------------- back-substitution + cost
// One block of 256 threads per chunk of (at most 256) points of one problem,
// in two steps.  With TRIAL, first the landmark step
//   dl = -H^-1 (g + sum_o H_o (rho + omega x X))
// of every variable point (W_o^T dc = H_o B dc) and the candidate point
// X + dl: the chunk's observations (contiguous) each form their term
// H_o (rho + omega x X) on one thread, kObsStage per pass, into shared
// memory, and each point's thread adds its own terms from there in
// observation order.  Then one thread per observation of the chunk for the
// cost at the candidate poses/points (the current state without TRIAL).
// Sums in a fixed order per chunk.
template <bool TRIAL>
__global__ void __launch_bounds__(256) k_cost(Dev d) {
  __shared__ double red[256];
  __shared__ unsigned long long redu[256];
  __shared__ double sX[3 * 256];                      // the chunk's (candidate) points
  __shared__ float sXf[TRIAL ? 3 * 256 : 1];          // the points as FP32 (pt_s)
  __shared__ double sC[TRIAL ? 3 * kObsStage : 1];    // staged observation terms
  __shared__ unsigned char sAct[TRIAL ? 256 : 1];     // point takes a step
  for (uint32_t ch = blockIdx.x; ch < d.num_point_chunks; ch += gridDim.x) {
    const uint32_t lo = d.chunk_point_begin[ch], hi = d.chunk_point_begin[ch + 1];
    const uint32_t P = d.num_problems == 1 ? 0u : d.point_prob[lo];
    const Ctrl& c = d.ctrl[P];
    if (c.done) continue;  // uniform: a chunk lies inside one problem
    const uint32_t cur = c.cur;
    const uint32_t pose_buf = TRIAL ? (cur ^ 1u) : cur;
    const LmParams& lp = d.params[P];
    double cost = 0.0, step = 0.0;
    unsigned long long bad = 0;
    const uint32_t l = lo + threadIdx.x;
    const bool mine = l < hi;
    double X[3] = {0.0, 0.0, 0.0};
    if (mine) {
#pragma unroll
      for (int a = 0; a < 3; ++a) X[a] = d.points[cur][3 * (size_t)l + a];
    }
    if (TRIAL) {
      const uint32_t o0 = d.pt_off[lo], o1 = d.pt_off[hi];
      bool act = false;
      if (mine) {
        const float4 s1 = d.pt_s[4 * (size_t)l + 1], s2 = d.pt_s[4 * (size_t)l + 2],
                     s3 = d.pt_s[4 * (size_t)l + 3];
        act = d.point_var[l] && s3.w != 0.0f;
        sXf[3 * threadIdx.x] = s1.z;
        sXf[3 * threadIdx.x + 1] = s1.w;
        sXf[3 * threadIdx.x + 2] = s2.x;
        sAct[threadIdx.x] = act ? 1 : 0;
      }
      __syncthreads();
      // In FP64 with the point's FP64 damped inverse: a point whose depth one
      // observation alone constrains has an inverse with entries near
      // 1/lambda along its ray, which FP32 would turn into a large spurious
      // step along the ray.
      double u0 = 0.0, u1 = 0.0, u2 = 0.0;
      if (act) {
        const float* ph = d.pt_h + 9 * (size_t)l;
        u0 = ph[6];
        u1 = ph[7];
        u2 = ph[8];
      }
      const uint32_t k0 = mine ? d.pt_off[l] : 0u, k1 = mine ? d.pt_off[l + 1] : 0u;
      for (uint32_t base = o0; base < o1; base += kObsStage) {
        const uint32_t end = min(o1, base + kObsStage);
        for (uint32_t k = base + threadIdx.x; k < end; k += blockDim.x) {
          double t0 = 0.0, t1 = 0.0, t2 = 0.0;
          const uint32_t pl = d.obs_point[k] - lo;
          const uint32_t slot = d.obs_slot[k];
          if (sAct[pl] && slot != kNone) {
            const double x = sXf[3 * pl], y = sXf[3 * pl + 1], z = sXf[3 * pl + 2];
            // The slot's step as three 8-byte loads.
            const float2* dc = reinterpret_cast<const float2*>(d.x + 6 * (size_t)slot);
            const float2 c01 = dc[0], c23 = dc[1], c45 = dc[2];
            const double w0 = c23.y, w1 = c45.x, w2 = c45.y;
            const double b0 = c01.x + (w1 * z - w2 * y);
            const double b1 = c01.y + (w2 * x - w0 * z);
            const double b2 = c23.x + (w0 * y - w1 * x);
            const float4 h0 = d.obs_h[2 * (size_t)k], h1 = d.obs_h[2 * (size_t)k + 1];
            t0 = h0.x * b0 + h0.y * b1 + h0.z * b2;
            t1 = h0.y * b0 + h0.w * b1 + h1.x * b2;
            t2 = h0.z * b0 + h1.x * b1 + h1.y * b2;
          }
          double* q = sC + 3 * (k - base);
          q[0] = t0;
          q[1] = t1;
          q[2] = t2;
        }
        __syncthreads();
        if (act) {
          const uint32_t a = max(k0, base), b = min(k1, end);
          for (uint32_t k = a; k < b; ++k) {
            const double* q = sC + 3 * (k - base);
            u0 += q[0];
            u1 += q[1];
            u2 += q[2];
          }
        }
        __syncthreads();
      }
      if (act) {
        double Mi[9], vv[3];
        point_inverse64(d, l, Mi, vv);
        const double e0 = -(Mi[0] * u0 + Mi[1] * u1 + Mi[2] * u2);
        const double e1 = -(Mi[3] * u0 + Mi[4] * u1 + Mi[5] * u2);
        const double e2 = -(Mi[6] * u0 + Mi[7] * u1 + Mi[8] * u2);
        step = fmax(step, sqrt(e0 * e0 + e1 * e1 + e2 * e2));
        X[0] += e0;
        X[1] += e1;
        X[2] += e2;
      }
      if (mine) {
#pragma unroll
        for (int a = 0; a < 3; ++a) d.points[cur ^ 1u][3 * (size_t)l + a] = X[a];
      }
    }
    if (mine) {
#pragma unroll
      for (int a = 0; a < 3; ++a) sX[3 * threadIdx.x + a] = X[a];
    }
    __syncthreads();
    // The chunk's observations, one thread each (stride 256), at the points
    // just placed in shared memory.
    const uint32_t o0 = d.pt_off[lo], o1 = d.pt_off[hi];
    for (uint32_t k = o0 + threadIdx.x; k < o1; k += blockDim.x) {
      const double* Xk = sX + 3 * (d.obs_point[k] - lo);
      const DevCamera& cam = d.cameras[d.obs_cam[k]];
      double rt[12];
      load_rt(d.pose_rt[pose_buf] + 12 * (size_t)d.obs_pose[k], rt);
      double xs[3], pred[2];
      to_sensor(rt, cam, Xk, xs);
      double ss;
      const uint32_t kind = d.obs_kind ? d.obs_kind[k] : kObsMono;
      if (kind != kObsMono) {
        double r[4];
        const int m = stereo_rows(kind, cam, d.cameras[d.obs_rcam[k]], d.obs_xy[k], d.obs_st[k], xs,
                                  nullptr, r, nullptr);
        if (!m) {
          ++bad;
          continue;
        }
        ss = 0.0;
        for (int i = 0; i < m; ++i) ss += r[i] * r[i];
      } else {
        if (!(xs[2] > 0.0) || !camera_project(cam, xs, pred)) {
          ++bad;
          continue;
        }
        const double2 xy = d.obs_xy[k];
        const double rx = pred[0] - xy.x, ry = pred[1] - xy.y;
        ss = rx * rx + ry * ry;
      }
      const double rc = robust_cost(lp.robust_kernel, lp.robust_parameter, ss);
      cost += d.obs_w ? d.obs_w[k] * rc : rc;  // w * rho(s) (problem.rs:497-560)
    }
    const double tc = block_sum<double, 256>(cost, red);
    const unsigned long long tb = block_sum<unsigned long long, 256>(bad, redu);
    const double ts = block_max<256>(step, red);
    if (threadIdx.x == 0) {
      d.chunk_cost[ch] = tc;
      d.chunk_bad[ch] = tb;
      d.chunk_step[ch] = ts;
    }
  }
}

// ------------------------------------------------------------------ decide
// The reference LM control per problem (solver.rs:629-682 / lm.rs:
// 608-663, 804-1008): accept iff the cost decreased (or unconditionally
// without initial_lambda) and the non-projectable count did not grow; lambda
// x10 / x0.1 clamped; convergence on step, absolute and relative cost change.
// A non-finite step is the reference's SingularSystem: lambda up, no step.
template <bool INIT>
__global__ void __launch_bounds__(256) k_decide(Dev d) {
  __shared__ double red[256];
  __shared__ unsigned long long redu[256];
  const uint32_t P = blockIdx.x;
  if (P >= d.num_problems) return;
  Ctrl& c = d.ctrl[P];
  if (c.done) return;
  const LmParams& lp = d.params[P];
  double cost = 0.0, lstep = 0.0, pstep = 0.0;
  unsigned long long bad = 0;
  for (uint32_t ch = d.prob_chunk_begin[P] + threadIdx.x; ch < d.prob_chunk_begin[P + 1];
       ch += blockDim.x) {
    cost += d.chunk_cost[ch];
    bad += d.chunk_bad[ch];
    lstep = fmax(lstep, d.chunk_step[ch]);
  }
  if (!INIT)
    for (uint32_t p = d.prob_pose_begin[P] + threadIdx.x; p < d.prob_pose_begin[P + 1];
         p += blockDim.x)
      pstep = fmax(pstep, d.pose_step[p]);
  cost = block_sum<double, 256>(cost, red);
  bad = block_sum<unsigned long long, 256>(bad, redu);
  lstep = block_max<256>(lstep, red);
  pstep = block_max<256>(pstep, red);
  if (threadIdx.x != 0) return;
  if (INIT) {
    c.initial_cost = cost;
    c.current_cost = cost;
    c.initial_nonproj = bad;
    c.current_nonproj = bad;
    c.lambda = lp.has_initial_lambda ? lp.initial_lambda : 0.0;
    c.relinearize = 1u;
    c.iteration = 0u;
    c.converged = 0u;
    c.nonfinite = 0u;
    c.total_pcg = 0ull;
    if (lp.max_iterations == 0) c.done = 1u;
    return;
  }
  const uint32_t it = c.iteration;
  const PcgState& pg = d.pcg[P];
  vlba_iteration rec;
  rec.iteration = it;
  rec.cost_before = c.current_cost;
  rec.pcg_iterations = pg.iters;
  rec.pcg_relative_residual = pg.bnorm > 0.0 ? pg.rnorm / pg.bnorm : 0.0;
  rec.linearize_ms = 0.0;
  rec.assemble_ms = 0.0;
  rec.pcg_ms = 0.0;
  rec.update_ms = 0.0;
  c.total_pcg += pg.iters;
  c.pcg_iters = pg.iters;
  c.pcg_status = pg.status;
  bool accepted = false;
  bool stop = false;
  if (c.nonfinite || !isfinite(pstep) || !isfinite(lstep)) {
    // SingularSystem (lm.rs:608-663): lambda up, cost unchanged, no step.
    c.lambda = fmin(c.lambda * lp.lambda_increase_factor, lp.max_lambda);
    rec.cost_after = c.current_cost;
    rec.max_pose_step = 0.0;
    rec.max_landmark_step = 0.0;
    rec.lambda = c.lambda;
    rec.step_accepted = 0u;
    if (c.lambda >= lp.max_lambda) stop = true;
  } else {
    const bool cost_ok = lp.has_initial_lambda ? (cost < c.current_cost) : true;
    accepted = cost_ok && bad <= c.current_nonproj;
    rec.cost_after = cost;
    rec.max_pose_step = pstep;
    rec.max_landmark_step = lstep;
    if (!accepted) {
      c.lambda = fmin(c.lambda * lp.lambda_increase_factor, lp.max_lambda);
      rec.lambda = c.lambda;
      rec.step_accepted = 0u;
      if (!lp.has_initial_lambda || c.lambda >= lp.max_lambda) stop = true;
    } else {
      rec.lambda = c.lambda;
      rec.step_accepted = 1u;
      const double before = c.current_cost;
      c.current_cost = cost;
      c.current_nonproj = bad;
      c.cur ^= 1u;
      if (lp.has_initial_lambda)
        c.lambda = fmax(c.lambda * lp.lambda_decrease_factor, lp.min_lambda);
      if (pstep < lp.step_tolerance && lstep < lp.step_tolerance) {
        c.converged = 1u;
        stop = true;
      } else if (fabs(before - cost) < lp.cost_tolerance) {
        c.converged = 1u;
        stop = true;
      } else if (lp.has_relative_cost_tolerance) {
        const double tol = lp.relative_cost_tolerance;
        if (isfinite(tol) && tol >= 0.0 &&
            (before - cost) / fmax(fabs(before), 2.220446049250313e-16) < tol) {
          c.converged = 1u;
          stop = true;
        }
      }
    }
  }
  c.cost_after = rec.cost_after;
  c.nonproj_after = bad;
  c.max_pose_step = rec.max_pose_step;
  c.max_landmark_step = rec.max_landmark_step;
  if (it < d.max_records) d.records[(size_t)P * d.max_records + it] = rec;
  c.iteration = it + 1;
  c.relinearize = accepted ? 1u : 0u;
  c.nonfinite = 0u;
  if (stop || c.iteration >= lp.max_iterations) c.done = 1u;
}

// -------------------------------------------------------------------- PCG
// Block-Jacobi PCG on the reduced camera system (the reference's pcg_init /
// apply_lm / apply_pose / pcg_step, ba.wgsl:420-562, with the explicit S in
// place of the implicit Schur operator): stop when |r| <= tol |b|, on
// non-positive curvature, or at the iteration cap.
//
// One cooperative launch runs every iteration; two grid barriers each.
//   A  every warp streams its own tiles of S (8 x 8 blocks of 6x6, 9.2 KB)
//      HBM/L2 -> shared memory with cp.async.bulk (TMA) through a private
//      two-stage ring, and writes per tile (I,J) the row-side partial
//      S_IJ p_J and the column-side partial S_IJ^T p_I, with p = z + beta p
//      formed on the fly; no block-wide synchronisation per tile.  Partials
//      of a tile row are contiguous slots that hold an empty marker until
//      their tile stores them; the owner block of a row (row mod grid) reads
//      each slot as soon as it is filled (bounded), reduces the row in a
//      fixed order into q, the new p and the partial p.q, and empties the
//      slots again.
//   -- grid barrier --
//   C  the owner of a tile row: x += alpha p, r -= alpha q, z = M^-1 r and
//      the partial dots r.z and r.r.
//   -- grid barrier --
// The first tiles of the next iteration are prefetched before the barriers.
// The leading tiles (a byte budget set from the L2 size) are loaded with an
// L2 evict_last policy and the rest with evict_first; at exit the resident
// lines are returned to the normal eviction priority.
// All scalars are per problem, summed over the problem's tile rows in a fixed
// order, so every block derives bit-identical alphas and betas and a
// problem's solve does not depend on what else is in the batch.  The grid
// barrier and every mbarrier wait are bounded; a timeout sets an error flag
// and every block leaves.
struct Pcg {
  static constexpr int kTB = 8;              // tile edge in 6x6 blocks
  static constexpr int kWarps = 8;           // one block per SM (shared memory)
  static constexpr int kThreads = 32 * kWarps;
  static constexpr int kStages = 2;          // per-warp TMA ring
  static constexpr int kTileFloats = kTB * kTB * kBlock;
  static constexpr uint32_t kTileBytes = kTileFloats * 4u;
  static constexpr int kRow = kTB * 6;       // floats of a tile-row vector segment
  static constexpr size_t kWarpBytes = (size_t)kStages * kTileBytes + 2 * kRow * 4;
  // Owned tile rows per block and their state in shared memory: p, z, q, x,
  // r (kRow floats each) and the kRow x 6 rows of M^-1, kept for the launch.
  static constexpr int kOwnMax = 32;
  static constexpr int kOwnFloats = 5 * kRow + 6 * kRow;
  static constexpr size_t kSmem = kWarps * kWarpBytes + (size_t)kWarps * kRow * 4 +
                                  (size_t)kWarps * 8 + (size_t)kOwnMax * kOwnFloats * 4 + 64;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ uint64_t l2_policy(bool keep) {
  uint64_t p;
  if (keep)
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  else
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// One bulk copy global -> shared completing on `bar`, with an L2 policy.
// The destination stage is reused only after every thread's reads of it have
// completed (their values consumed, then a warp or block barrier), so the
// copy needs no proxy fence -- the reuse rule of TMA pipelines.
__device__ __forceinline__ void tma_load(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar, uint64_t policy) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; false (and the error flag) once kWaitLimitNs have passed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t_end = now_ns() + kWaitLimitNs;
  while (!mbar_try_wait(bar, parity)) {
    if (now_ns() > t_end) {
      atomicOr(err, (unsigned int)kErrTmaTimeout);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void red_add_release(unsigned int* a, unsigned int v) {
  asm volatile("red.add.release.gpu.u32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* a) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

// Grid barrier on one arrival counter, bar[0], zeroed by k_pcg_setup before
// every launch: each block's arrival is a release reduction (no round trip),
// then its thread 0 polls with acquire loads, bounded in time, until the
// count reaches nblocks times the block's generation `gen` (the barriers it
// has passed, counted from the launch).  Returns false when any block has
// flagged an error (every thread of the block sees the same value).
__device__ bool grid_barrier(unsigned int* bar, unsigned int nblocks, unsigned int* err,
                             unsigned int* s_flag, unsigned int& gen) {
  __syncthreads();
  ++gen;
  if (threadIdx.x == 0) {
    red_add_release(bar, 1u);
    const unsigned int target = gen * nblocks;
    if ((int)(ld_acquire(bar) - target) < 0) {
      const unsigned long long t_end = now_ns() + kWaitLimitNs;
      while ((int)(ld_acquire(bar) - target) < 0) {
        if (now_ns() > t_end) {
          atomicOr(err, (unsigned int)kErrBarrierTimeout);
          break;
        }
      }
    }
    *s_flag = *(volatile unsigned int*)err;
  }
  __syncthreads();
  return *s_flag == 0u;
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Per-tile marks (first kTraceTiles tiles of each warp): [iteration][warp][tile][4].
constexpr int kTraceTiles = 8;
__device__ __forceinline__ void trace_tile(const Dev& d, int k, uint32_t gw, uint32_t tw, uint32_t m,
                                           int which) {
  if (d.trace && (threadIdx.x & 31u) == 0 && k < kTraceIters && m < (uint32_t)kTraceTiles) {
    unsigned long long* w = d.trace + (size_t)kTraceIters * gridDim.x * kTracePhases +
                            (size_t)kTraceIters * tw * 2;
    w[(((size_t)k * tw + gw) * kTraceTiles + m) * 4 + which] = globaltimer();
  }
}

// Per-warp marks after the block marks: [iteration][warp of grid][2].
__device__ __forceinline__ void trace_warp(const Dev& d, int k, uint32_t gw, uint32_t tw, int which) {
  if (d.trace && (threadIdx.x & 31u) == 0 && k < kTraceIters) {
    unsigned long long* w = d.trace + (size_t)kTraceIters * gridDim.x * kTracePhases;
    w[((size_t)k * tw + gw) * 2 + which] = globaltimer();
  }
}

__device__ __forceinline__ void trace_mark(const Dev& d, int k, int phase) {
  if (d.trace && threadIdx.x == 0 && k < kTraceIters) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    d.trace[((size_t)k * gridDim.x + blockIdx.x) * kTracePhases + phase] = t;
  }
}

// Per-problem PCG scalars from the tile-row dots, summed by warp 0 in a
// fixed order (lane-strided partial sums, then a butterfly).
struct ProbScal {
  int active;
  int status;   // when inactive: 0 converged, 1 cap, 2 breakdown
  uint32_t iters;
  uint32_t pad;
  double beta;
  double rz;    // rz(k-1)
  double rr;
  double bnorm;
};

// Tile-row dots, one contiguous array per quantity (coalesced per-problem
// sums): slot q of tile row tr at dots[q * num_tile_rows + tr].  rz and rr
// rotate over three slots (iteration k mod 3), p.q over two.
__device__ __forceinline__ int mod3(int k) { return ((k % 3) + 3) % 3; }
constexpr int kDotRz = 0, kDotRr = 3, kDotPq = 6, kDotB2 = 8;
__device__ __forceinline__ double* dot_at(const Dev& d, int slot, uint32_t tr) {
  return d.dots + (size_t)slot * d.num_tile_rows + tr;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Sums of a problem's tile-row dots (rz(k-1), rz(k-2), rr(k-1), pq(k-1), b2)
// in one fixed order: the rows are dealt to kSumSlots slots -- row
// t0 + 32 (w + kSumSlots i) + l to lane l of slot w -- each lane adds its rows
// in ascending order (two rows' loads ahead of their adds), a butterfly sums
// the slot, and the slots are added in order.  A block computes the slots on
// its warps at once (the block's scalars), one warp computes them in turn:
// the same sums, so every block takes the same decisions.
constexpr int kSumSlots = 8;
__device__ __forceinline__ void dot_sums_slot(const Dev& d, int k, uint32_t t0, uint32_t t1,
                                              uint32_t w, double (&v)[5]) {
  const uint32_t lane = threadIdx.x & 31u;
  const double* q0 = dot_at(d, kDotRz + mod3(k - 1), 0);
  const double* q1 = dot_at(d, kDotRz + mod3(k - 2), 0);
  const double* q2 = dot_at(d, kDotRr + mod3(k - 1), 0);
  const double* q3 = dot_at(d, kDotPq + ((k - 1) & 1), 0);
  const double* q4 = dot_at(d, kDotB2, 0);
  constexpr uint32_t kStep = 32 * kSumSlots;
  double a[5] = {0, 0, 0, 0, 0};
  uint32_t tr = t0 + 32 * w + lane;
  for (; tr + kStep < t1; tr += 2 * kStep) {
    const double x0 = __ldcg(q0 + tr), x1 = __ldcg(q1 + tr), x2 = __ldcg(q2 + tr),
                 x3 = __ldcg(q3 + tr), x4 = __ldcg(q4 + tr);
    const double y0 = __ldcg(q0 + tr + kStep), y1 = __ldcg(q1 + tr + kStep),
                 y2 = __ldcg(q2 + tr + kStep), y3 = __ldcg(q3 + tr + kStep),
                 y4 = __ldcg(q4 + tr + kStep);
    a[0] += x0;
    a[1] += x1;
    a[2] += x2;
    a[3] += x3;
    a[4] += x4;
    a[0] += y0;
    a[1] += y1;
    a[2] += y2;
    a[3] += y3;
    a[4] += y4;
  }
  if (tr < t1) {
    a[0] += __ldcg(q0 + tr);
    a[1] += __ldcg(q1 + tr);
    a[2] += __ldcg(q2 + tr);
    a[3] += __ldcg(q3 + tr);
    a[4] += __ldcg(q4 + tr);
  }
#pragma unroll
  for (int e = 0; e < 5; ++e) v[e] = warp_sum(a[e]);
}

// Per-problem scalars from the sums of dot_sums_slot (every lane of the
// calling warp returns the same values); the sticky flag is read once and
// broadcast.
__device__ ProbScal prob_scalars_from(const Dev& d, uint32_t P, int k, const double (&v)[5]) {
  const uint32_t lane = threadIdx.x & 31u;
  int sticky = 0;
  if (lane == 0) sticky = (int)*(volatile uint32_t*)&d.pcg[P].active;
  sticky = __shfl_sync(0xffffffffu, sticky, 0);
  const LmParams& lp = d.params[P];
  ProbScal s;
  s.active = sticky;
  s.status = 0;
  s.iters = (uint32_t)k;
  s.pad = 0;
  s.beta = 0.0;
  s.rz = v[0];
  s.rr = v[2];
  s.bnorm = sqrt(v[4]);
  if (sticky) {
    if (k == 0) {
      // pcg_init (ba.wgsl:420-439): done when |b| = 0 or r.z <= 0.
      if (!(v[4] > 0.0) || !(v[0] > 0.0) || lp.max_pcg_iterations == 0) s.active = 0;
    } else if (!(v[3] > 0.0) || !isfinite(v[3])) {
      s.active = 0;  // non-positive curvature in iteration k-1: x unchanged
      s.status = 2;
      s.iters = (uint32_t)(k - 1);
    } else if (sqrt(v[2]) <= lp.pcg_relative_tolerance * s.bnorm || !(v[0] > 0.0)) {
      s.active = 0;
    } else if ((uint32_t)k >= lp.max_pcg_iterations) {
      s.active = 0;
      s.status = 1;
    } else {
      s.beta = v[0] / v[1];
    }
  }
  return s;
}

// The same scalars computed by one warp alone, the slots in turn.
__device__ ProbScal prob_scalars_warp(const Dev& d, uint32_t P, int k) {
  const uint32_t t0 = d.prob_tr_begin[P], t1 = d.prob_tr_begin[P + 1];
  double tot[5] = {0, 0, 0, 0, 0};
  // Slots past the problem's last row hold no rows: left out (as the block
  // form leaves them out), so a problem of few rows costs one slot.
  for (uint32_t w = 0; w < (uint32_t)kSumSlots && t0 + 32 * w < t1; ++w) {
    double v[5];
    dot_sums_slot(d, k, t0, t1, w, v);
#pragma unroll
    for (int e = 0; e < 5; ++e) tot[e] += v[e];
  }
  return prob_scalars_from(d, P, k, tot);
}

// p.q(k) of a problem in the same slot order as dot_sums_slot: slot w's
// lane-strided sum (two rows' loads ahead of their adds) and butterfly.
__device__ __forceinline__ double pq_slot(const Dev& d, int k, uint32_t t0, uint32_t t1,
                                          uint32_t w) {
  const double* q = dot_at(d, kDotPq + (k & 1), 0);
  constexpr uint32_t kStep = 32 * kSumSlots;
  double a = 0.0;
  uint32_t tr = t0 + 32 * w + (threadIdx.x & 31u);
  for (; tr + kStep < t1; tr += 2 * kStep) {
    const double x = __ldcg(q + tr), y = __ldcg(q + tr + kStep);
    a += x;
    a += y;
  }
  if (tr < t1) a += __ldcg(q + tr);
  return warp_sum(a);
}

// The same p.q computed by one warp alone, the slots in turn.
__device__ double pq_warp(const Dev& d, uint32_t P, int k) {
  const uint32_t t0 = d.prob_tr_begin[P], t1 = d.prob_tr_begin[P + 1];
  double pq = 0.0;
  for (uint32_t w = 0; w < (uint32_t)kSumSlots && t0 + 32 * w < t1; ++w)
    pq += pq_slot(d, k, t0, t1, w);
  return pq;
}

// Fixed-order sum of a double over the block: butterfly per warp, then the
// warps in order (result valid in every thread).
template <int NW>
__device__ __forceinline__ double block_sum_fast(double v, double* red) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < NW; ++w) t += red[w];
  __syncthreads();
  return t;
}

// A partial slot holds kSlotEmpty -- a NaN bit pattern that FP32 arithmetic
// never produces (it returns the canonical NaN) -- in every entry until the
// warp of its tile stores the partial.  The owner of the slot's tile row
// reads it once no entry is empty and empties it again for the next
// iteration; the grid barriers between that store and the next iteration's
// partial stores order the two.
constexpr uint32_t kSlotEmpty = 0xFFC0DEADu;

// Wait (bounded) until the U x 2 entries v[u][e] -- loaded from src(u) + 32 e
// where valid(u, e) -- are all filled, reloading the empty ones; then empty
// the slots' entries.  Warp-collective.
template <int U, typename Src, typename Valid>
__device__ __forceinline__ void take_slots(float (&v)[U][2], Src src, Valid valid,
                                           unsigned int* err) {
  auto missing = [&]() {
    bool miss = false;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int e = 0; e < 2; ++e)
        if (valid(u, e) && __float_as_uint(v[u][e]) == kSlotEmpty) miss = true;
    return miss;
  };
  if (__any_sync(0xffffffffu, missing())) {
    const unsigned long long t_end = now_ns() + kWaitLimitNs;
    do {
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (valid(u, e) && __float_as_uint(v[u][e]) == kSlotEmpty) v[u][e] = __ldcg(src(u) + 32 * e);
      if (__any_sync(0xffffffffu, now_ns() > t_end)) {
        if ((threadIdx.x & 31u) == 0) atomicOr(err, (unsigned int)kErrBarrierTimeout);
        break;
      }
    } while (__any_sync(0xffffffffu, missing()));
  }
#pragma unroll
  for (int u = 0; u < U; ++u)
#pragma unroll
    for (int e = 0; e < 2; ++e)
      if (valid(u, e)) __stcg(src(u) + 32 * e, __uint_as_float(kSlotEmpty));
}

__global__ void __launch_bounds__(Pcg::kThreads, 1) k_pcg(Dev d) {
  using C = Pcg;
  constexpr int NW = C::kWarps;
  extern __shared__ __align__(128) unsigned char smem[];
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  // Per-warp region: kStages tile buffers, then the warp's p segments.
  unsigned char* wbase = smem + (size_t)warp * C::kWarpBytes;
  float* const ring = reinterpret_cast<float*>(wbase);
  float* const wPI = reinterpret_cast<float*>(wbase + (size_t)C::kStages * C::kTileBytes);
  float* const wPJ = wPI + C::kRow;
  float* const colw = reinterpret_cast<float*>(smem + (size_t)NW * C::kWarpBytes);  // [NW kRow]
  double* const red = reinterpret_cast<double*>(colw + NW * C::kRow);             // [NW]
  float* const own = reinterpret_cast<float*>(red + NW);  // [kOwnMax][kOwnFloats]
  __shared__ uint64_t mbar[NW][C::kStages];
  __shared__ ProbScal sc;
  __shared__ uint32_t sc_prob;
  __shared__ int sc_k;
  __shared__ unsigned int s_flag;

  const uint32_t G = gridDim.x;
  const uint32_t TW = G * NW;  // warps in the grid
  // Warps are numbered from the last block down, so the blocks that own one
  // tile row more than others (the first ones) get the warps with one tile
  // fewer.
  const uint32_t gw0 = (G - 1u - blockIdx.x) * NW;
  const uint32_t gw = gw0 + warp;
  const uint32_t ntiles = d.num_tiles;
  // This warp's tiles: gw + m TW, m < Mw, in the same order each iteration.
  const uint32_t Mw = gw < ntiles ? (ntiles - 1 - gw) / TW + 1 : 0u;
  const uint64_t keep = l2_policy(true), stream = l2_policy(false);
  if (lane == 0) {
    for (int st = 0; st < C::kStages; ++st) mbar_init(&mbar[warp][st]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid == 0) {
    sc_prob = kNone;
    sc_k = -2;
  }
  __syncthreads();
  // Warp tile sequence s = k Mw + m: stage s % kStages, phase (s / kStages) & 1,
  // both kept by increments: (cst, cph) for the next tile to consume, ist for
  // the next copy.  `issued` (sequence number of the next copy), `iss_m` (its
  // tile index m, kept modulo Mw) and ist are tracked by lane 0 alone.
  uint64_t issued = 0, consumed = 0;
  uint32_t iss_m = 0, ist = 0, cst = 0, cph = 0;
  auto issue = [&]() {  // lane 0 only
    const uint32_t t = gw + iss_m * TW;
    const int st = (int)ist;
    tma_load(ring + (size_t)st * C::kTileFloats, d.tiles + (size_t)t * C::kTileFloats,
             C::kTileBytes, &mbar[warp][st], t < d.l2_resident_tiles ? keep : stream);
    ++issued;
    ist = ist + 1u == (uint32_t)C::kStages ? 0u : ist + 1u;
    iss_m = (iss_m + 1u == Mw) ? 0u : iss_m + 1u;
  };
  bool ok = true;

  // Block-level per-problem scalars (cached per problem and iteration).
  // The block's scalars of problem P: each warp sums one slot of the rows'
  // dots, warp 0 adds the slots in order (the sums of prob_scalars_warp).
  static_assert(NW >= kSumSlots, "a warp per slot of the scalar sums");
  __shared__ double s_slot[kSumSlots][5];
  auto scal = [&](uint32_t P, int k) {
    if (sc_prob == P && sc_k == k) return;  // uniform: shared values
    __syncthreads();
    if (warp < (uint32_t)kSumSlots) {
      double v[5];
      dot_sums_slot(d, k, d.prob_tr_begin[P], d.prob_tr_begin[P + 1], warp, v);
      if (lane == 0)
        for (int e = 0; e < 5; ++e) s_slot[warp][e] = v[e];
    }
    __syncthreads();
    if (warp == 0) {
      double tot[5] = {0, 0, 0, 0, 0};
      const uint32_t t0 = d.prob_tr_begin[P], t1 = d.prob_tr_begin[P + 1];
      for (uint32_t w = 0; w < (uint32_t)kSumSlots && t0 + 32 * w < t1; ++w)
#pragma unroll
        for (int e = 0; e < 5; ++e) tot[e] += s_slot[w][e];
      const ProbScal s = prob_scalars_from(d, P, k, tot);
      if (lane == 0) {
        sc = s;
        sc_prob = P;
        sc_k = k;
      }
    }
    __syncthreads();
  };

  // Rows this block owns (row R belongs to block R mod G), kOwnMax at most
  // (the host never launches a grid with rows > G kOwnMax): list bounds and
  // problem, constant for the launch.  The owner alone writes its rows' p, z,
  // x and r, so their shared-memory copies stay current for the whole solve.
  constexpr int kOwn = C::kOwnMax;
  constexpr uint32_t kBigRow = 32;  // rows of this many tiles reduce over the whole block
  constexpr int kOP = 0, kOZ = C::kRow, kOQ = 2 * C::kRow, kOX = 3 * C::kRow, kOR = 4 * C::kRow,
                kOM = 5 * C::kRow;
  __shared__ uint32_t own_m0[kOwn], own_m1[kOwn], own_prob[kOwn];
  const uint32_t nown = blockIdx.x < d.num_tile_rows
                            ? min((uint32_t)kOwn, (d.num_tile_rows - 1 - blockIdx.x) / G + 1)
                            : 0u;
  if (tid < nown) {
    const uint32_t R = blockIdx.x + tid * G;
    own_m0[tid] = d.tr_list_off[R];
    own_m1[tid] = d.tr_list_off[R + 1];
    own_prob[tid] = d.tr_prob[R];
  }
  auto ownrow = [&](uint32_t j) -> float* { return own + (size_t)j * C::kOwnFloats; };
  unsigned int bar_gen = 0u;  // barriers passed in this launch (the counter starts at 0)

  // Fixed-order reduction of tile row R: warp w sums slots m0 + w + j NW
  // (contiguous kRow floats, coalesced, kBatch in flight), in slot order;
  // then the warps' sums in warp order.  Gives q_R, the new p_R and the
  // partial p.q of iteration k.
  auto reduce_row = [&](int j, int k, double beta) {
    const uint32_t R = blockIdx.x + (uint32_t)j * G;
    const uint32_t m0 = own_m0[j], m1 = own_m1[j];
    constexpr int kPer = (C::kRow + 31) / 32;
    constexpr int kBatch = 20;  // 20 slots per warp in flight: one round for 160 slots
    float acc[kPer];
#pragma unroll
    for (int e = 0; e < kPer; ++e) acc[e] = 0.0f;
    static_assert(kPer == 2, "two entries per lane");
    for (uint32_t m = m0 + warp; m < m1; m += kBatch * NW) {
      float v[kBatch][kPer];
      float* const base = d.partial + (size_t)m * C::kRow + lane;
      auto src = [&](int u) { return base + (size_t)u * NW * C::kRow; };
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const uint32_t slot = m + u * NW;
#pragma unroll
        for (int e = 0; e < kPer; ++e)
          v[u][e] = (slot < m1 && lane + 32 * e < (uint32_t)C::kRow) ? __ldcg(src(u) + 32 * e) : 0.0f;
      }
      take_slots<kBatch>(v, src, [&](int u, int e) {
        return m + u * NW < m1 && lane + 32 * e < (uint32_t)C::kRow;
      }, d.error);
#pragma unroll
      for (int u = 0; u < kBatch; ++u)
#pragma unroll
        for (int e = 0; e < kPer; ++e) acc[e] += v[u][e];
    }
#pragma unroll
    for (int e = 0; e < kPer; ++e)
      if (lane + 32 * e < (uint32_t)C::kRow) colw[warp * C::kRow + lane + 32 * e] = acc[e];
    __syncthreads();
    double pq = 0.0;
    if (tid < (uint32_t)C::kRow) {
      const size_t at = (size_t)R * C::kRow + tid;
      float q = 0.0f;
#pragma unroll
      for (int w2 = 0; w2 < NW; ++w2) q += colw[w2 * C::kRow + tid];
      float* o = ownrow((uint32_t)j);
      float pv = o[kOP + tid];
      if (k > 0) pv = __fmaf_rn((float)beta, pv, o[kOZ + tid]);
      o[kOP + tid] = pv;
      o[kOQ + tid] = q;
      d.p[at] = pv;
      d.q[at] = q;
      pq = (double)pv * (double)q;
    }
    pq = block_sum_fast<NW>(pq, red);
    if (tid == 0) *dot_at(d, kDotPq + (k & 1), R) = pq;
  };

  // Row-local steps run one warp per owned row (row j on warp j mod NW),
  // entries e = lane and lane + 32 of the row's kRow, with the warp's segment
  // buffer as scratch; their dots are butterflies over the warp.
  static_assert(C::kRow > 32 && C::kRow <= 64, "two entries per lane");
  const bool e1 = lane + 32u < (uint32_t)C::kRow;  // this lane has a second entry
  float* const sPI = wPI;  // warp scratch of kRow floats (init / C)

  // ---- init: x = 0, r = b, z = M^-1 r, p = z; dots rz, b2 of "iteration -1".
  for (uint32_t j = warp; j < nown; j += NW) {
    const uint32_t tr = blockIdx.x + j * G;
    const uint32_t P = d.tr_prob[tr];
    if (!*(volatile uint32_t*)&d.pcg[P].active) continue;
    const size_t base = (size_t)tr * C::kRow;
    float* o = ownrow(j);
    for (uint32_t e = lane; e < (uint32_t)C::kRow; e += 32) {
      const float b = d.rhs[base + e];
      d.x[base + e] = 0.0f;
      d.r[base + e] = b;
      o[kOX + e] = 0.0f;
      o[kOR + e] = b;
      sPI[e] = b;
    }
    __syncwarp();
    double rz = 0.0, bb = 0.0;
    for (uint32_t e = lane; e < (uint32_t)C::kRow; e += 32) {
      const uint32_t cam = e / 6, a = e % 6;
      const float* m = d.minv + 36 * (base / 6 + cam) + a * 6;
      float z = 0.0f;
#pragma unroll
      for (int b = 0; b < 6; ++b) {
        const float mb = m[b];
        o[kOM + e * 6 + b] = mb;
        z += mb * sPI[cam * 6 + b];
      }
      d.z[base + e] = z;
      d.p[base + e] = z;
      o[kOZ + e] = z;
      o[kOP + e] = z;
      rz += (double)sPI[e] * (double)z;
      bb += (double)sPI[e] * (double)sPI[e];
    }
    rz = warp_sum(rz);
    bb = warp_sum(bb);
    if (lane == 0) {
      *dot_at(d, kDotRz + mod3(-1), tr) = rz;
      *dot_at(d, kDotRr + mod3(-1), tr) = bb;
      *dot_at(d, kDotPq + 1, tr) = 1.0;
      *dot_at(d, kDotB2, tr) = bb;
    }
    __syncwarp();
  }
  // Every partial slot starts empty.
  {
    const size_t n = (size_t)d.tr_list_off[d.num_tile_rows] * C::kRow;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + tid; i < n; i += (size_t)G * blockDim.x)
      __stcg(d.partial + i, __uint_as_float(kSlotEmpty));
  }
  // The metadata of the warp's first three tiles (the same every iteration).
  const uint4 meta0 = Mw > 0 ? d.tile_meta[gw] : make_uint4(0u, 0u, 0u, 0u);
  const uint4 meta1 = Mw > 1 ? d.tile_meta[gw + TW] : make_uint4(0u, 0u, 0u, 0u);
  const uint4 meta2 = Mw > 2 ? d.tile_meta[gw + 2 * TW] : make_uint4(0u, 0u, 0u, 0u);
  // The first tiles of every warp go out before the barrier.
  if (lane == 0)
    while (issued < (uint64_t)C::kStages && issued < Mw) issue();
  ok = grid_barrier(d.barrier, G, d.error, &s_flag, bar_gen);

  for (int k = 0; ok; ++k) {
    trace_mark(d, k, 0);
    // ---- A: status of the problems whose first tile row this block owns
    // (by that row's warp), then the warps' tiles.
    // The block's scalars of its first tile's problem first: the owner of
    // that problem (the single-problem case) reads them from there.
    if (NW > 0) {
      if (gw0 < ntiles) scal(d.tile_meta[gw0].w, k);
    }
    for (uint32_t j = warp; j < nown; j += NW) {
      const uint32_t tr = blockIdx.x + j * G;
      const uint32_t P = own_prob[j];
      if (d.prob_tr_begin[P] != tr) continue;  // owner = first tile row
      if (!*(volatile uint32_t*)&d.pcg[P].active) continue;
      const ProbScal ps = (sc_prob == P && sc_k == k) ? sc : prob_scalars_warp(d, P, k);
      if (!ps.active && lane == 0) {
        PcgState& st = d.pcg[P];
        st.iters = ps.iters;
        st.status = (uint32_t)ps.status;
        st.bnorm = ps.bnorm;
        st.rnorm = sqrt(ps.rr);
        st.rz = ps.rz;
        __threadfence();
        st.active = 0u;
        atomicSub(d.barrier + 2, 1u);
      }
      __syncwarp();
    }
    trace_mark(d, k, 1);
    {
      // Software pipeline per warp: tile metadata three tiles ahead, the p/z
      // segments (entries e = lane + 32 j of [0, 2 kRow): row I's, then row
      // J's) two tiles ahead in two register sets that alternate (the loop
      // is unrolled by two, so neither set is indexed at run time), the tile
      // itself kStages ahead (TMA ring).
      constexpr int kPre = (2 * C::kRow + 31) / 32;
      float pa_p[kPre], pa_z[kPre], pb_p[kPre], pb_z[kPre];
      auto prefetch_seg = [&](float (&pp)[kPre], float (&pz)[kPre], uint32_t ij) {
#pragma unroll
        for (int j = 0; j < kPre; ++j) {
          const uint32_t e = lane + 32u * j;
          if (e < 2u * C::kRow) {
            const uint32_t row = e < (uint32_t)C::kRow ? (ij >> 16) : (ij & 0xFFFFu);
            const size_t at = (size_t)row * C::kRow + (e % C::kRow);
            pp[j] = __ldcg(d.p + at);
            pz[j] = __ldcg(d.z + at);
          }
        }
      };
      uint32_t wprob = kNone;
      ProbScal ws;
      ws.active = 0;
      ws.beta = 0.0;
      uint4 meta_cur = meta0, meta_n1 = meta1, meta_n2 = meta2;
      if (Mw > 0) prefetch_seg(pa_p, pa_z, meta0.x);
      if (Mw > 1) prefetch_seg(pb_p, pb_z, meta1.x);
      trace_warp(d, k, gw, TW, 0);
      // Tile m with its segments in (pre_p, pre_z); they are refilled with
      // tile m + 2's once copied out.  A tile's segments are read before its
      // partials are stored, so before the owners of its rows can reduce
      // them and write the next p.
      auto step = [&](uint32_t m, float (&pre_p)[kPre], float (&pre_z)[kPre]) {
        const uint64_t s = (uint64_t)k * Mw + m;
        trace_tile(d, k, gw, TW, m, 0);
        const uint4 meta = meta_cur;
        uint4 meta_n3 = make_uint4(0u, 0u, 0u, 0u);
        if (m + 3 < Mw) meta_n3 = d.tile_meta[gw + (m + 3) * TW];
        const uint32_t I = meta.x >> 16, J = meta.x & 0xFFFFu;
        const uint32_t P = meta.w;
        if (P != wprob) {
          if (sc_prob == P && sc_k == k) ws = sc;  // the block's scalars
          else ws = prob_scalars_warp(d, P, k);
          wprob = P;
        }
        const bool active = ws.active != 0;
        if (active) {
#pragma unroll
          for (int j = 0; j < kPre; ++j) {
            const uint32_t e = lane + 32u * j;
            if (e < 2u * C::kRow) {
              const float v = k > 0 ? __fmaf_rn((float)ws.beta, pre_p[j], pre_z[j]) : pre_p[j];
              if (e < (uint32_t)C::kRow) wPI[e] = v;
              else wPJ[e - C::kRow] = v;
            }
          }
        }
        if (m + 2 < Mw) prefetch_seg(pre_p, pre_z, meta_n2.x);
        const int st = (int)cst;
        trace_tile(d, k, gw, TW, m, 1);
        const bool arrived =
            __all_sync(0xffffffffu, mbar_wait(&mbar[warp][st], cph, d.error));
        consumed = s + 1;
        if (++cst == (uint32_t)C::kStages) {
          cst = 0u;
          cph ^= 1u;
        }
        __syncwarp();  // the segments are visible to the whole warp
        trace_tile(d, k, gw, TW, m, 2);
        if (!arrived) ok = false;
        if (active && arrived) {
          // Lane l takes blocks l and l + 32: (li, lj) = (l / 8, l % 8) and
          // (l / 8 + 4, l % 8); 16-byte reads at a 144-byte stride are free
          // of bank conflicts within each quarter warp.
          const float* tile = ring + (size_t)st * C::kTileFloats;
          const int li = (int)(lane >> 3), lj = (int)(lane & 7);
          float row[2][6], col[6];
#pragma unroll
          for (int c = 0; c < 6; ++c) col[c] = 0.0f;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float4* blk = reinterpret_cast<const float4*>(tile + (lane + 32 * h) * kBlock);
            float sv[36];
#pragma unroll
            for (int q = 0; q < 9; ++q) {
              const float4 v = blk[q];
              sv[4 * q] = v.x;
              sv[4 * q + 1] = v.y;
              sv[4 * q + 2] = v.z;
              sv[4 * q + 3] = v.w;
            }
            // The segments' six entries as three 8-byte shared loads.
            float pj[6], pi[6];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const float2 vj = reinterpret_cast<const float2*>(wPJ + lj * 6)[c];
              const float2 vi = reinterpret_cast<const float2*>(wPI + (li + 4 * h) * 6)[c];
              pj[2 * c] = vj.x;
              pj[2 * c + 1] = vj.y;
              pi[2 * c] = vi.x;
              pi[2 * c + 1] = vi.y;
            }
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
          // Row sides: sums over lj (lane bits 0-2) by a reduce-scatter
          // butterfly -- offsets 4, 2, 1, each lane keeping the half its bit
          // selects -- so every lane ends with one or two finished entries
          // (the sums of an all-reduce butterfly, in the same order).
          // Lane bit 2 picks h, bit 1 the entries a = 0-2 or 3-5, bit 0 the
          // first two of those or the third.
          const bool b2 = (lane >> 2) & 1u, b1 = (lane >> 1) & 1u, b0 = lane & 1u;
          float rs[6];
#pragma unroll
          for (int a = 0; a < 6; ++a) {
            const float keep = b2 ? row[1][a] : row[0][a];
            const float send = b2 ? row[0][a] : row[1][a];
            rs[a] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
          }
          float r3[3];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const float keep = b1 ? rs[a + 3] : rs[a];
            const float send = b1 ? rs[a] : rs[a + 3];
            r3[a] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
          }
          // Bit 0: the even lane keeps entries 0 and 1 of the three, the odd
          // lane entry 2.
          const float x0 = __shfl_xor_sync(0xffffffffu, b0 ? r3[0] : r3[2], 1);
          const float x1 = __shfl_xor_sync(0xffffffffu, r3[1], 1);
          float* part = d.partial + (size_t)meta.y * C::kRow;
          {
            const int base = (li + 4 * (int)b2) * 6 + 3 * (int)b1;
            if (b0) {
              part[base + 2] = r3[2] + x0;
            } else {
              part[base] = r3[0] + x0;
              part[base + 1] = r3[1] + x1;
            }
          }
          if (I != J) {
            // Column side: sums over li (lane bits 3-4), offsets 8 then 16:
            // bit 3 picks the entries c = 0-2 or 3-5, bit 4 the first two
            // of those or the third.
            const bool b3 = (lane >> 3) & 1u, b4 = (lane >> 4) & 1u;
            float c3[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const float keep = b3 ? col[c + 3] : col[c];
              const float send = b3 ? col[c] : col[c + 3];
              c3[c] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
            }
            const float y0 = __shfl_xor_sync(0xffffffffu, b4 ? c3[0] : c3[2], 16);
            const float y1 = __shfl_xor_sync(0xffffffffu, c3[1], 16);
            float* partc = d.partial + (size_t)meta.z * C::kRow + lj * 6 + 3 * (int)b3;
            if (b4) {
              partc[2] = c3[2] + y0;
            } else {
              partc[0] = c3[0] + y0;
              partc[1] = c3[1] + y1;
            }
          }
        }
        __syncwarp();  // the stage and the segments are free again
        trace_tile(d, k, gw, TW, m, 3);
        // Refill the stage with the tile kStages ahead (possibly the next
        // iteration's; S does not change during the solve).
        if (lane == 0 && issued < s + 1 + C::kStages) issue();
        meta_cur = meta_n1;
        meta_n1 = meta_n2;
        meta_n2 = meta_n3;
      };
      for (uint32_t m = 0; m < Mw; m += 2) {
        step(m, pa_p, pa_z);
        if (m + 1 < Mw) step(m + 1, pb_p, pb_z);
      }
      trace_warp(d, k, gw, TW, 1);
    }
    // Row reductions by their owners, each slot read as soon as it is
    // filled: a row of many tiles by the whole block (its slots spread over
    // the warps), the others one warp per row.
    for (uint32_t j = 0; j < nown; ++j) {
      if (own_m1[j] - own_m0[j] < kBigRow) continue;
      scal(own_prob[j], k);
      if (!sc.active) continue;
      reduce_row((int)j, k, sc.beta);
    }
    uint32_t oprob = kNone;
    ProbScal os;
    os.active = 0;
    os.beta = 0.0;
    for (uint32_t j = warp; j < nown; j += NW) {
      if (own_m1[j] - own_m0[j] >= kBigRow) continue;
      const uint32_t P = own_prob[j];
      if (P != oprob) {
        os = (sc_prob == P && sc_k == k) ? sc : prob_scalars_warp(d, P, k);
        oprob = P;
      }
      if (!os.active) continue;
      // Slots in order, eight loads in flight per lane.
      const uint32_t R = blockIdx.x + j * G;
      const uint32_t m0 = own_m0[j], m1 = own_m1[j];
      float q0 = 0.0f, q1 = 0.0f;
      for (uint32_t m = m0; m < m1; m += 8) {
        float v[8][2];
        float* const base = d.partial + (size_t)m * C::kRow + lane;
        auto src = [&](int u) { return base + u * C::kRow; };
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          v[u][0] = m + u < m1 ? __ldcg(src(u)) : 0.0f;
          v[u][1] = (m + u < m1 && e1) ? __ldcg(src(u) + 32) : 0.0f;
        }
        take_slots<8>(v, src, [&](int u, int e) { return m + u < m1 && (e == 0 || e1); }, d.error);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          q0 += v[u][0];
          q1 += v[u][1];
        }
      }
      float* o = ownrow(j);
      const size_t at = (size_t)R * C::kRow;
      double pq = 0.0;
      {
        float pv = o[kOP + lane];
        if (k > 0) pv = __fmaf_rn((float)os.beta, pv, o[kOZ + lane]);
        o[kOP + lane] = pv;
        o[kOQ + lane] = q0;
        d.p[at + lane] = pv;
        d.q[at + lane] = q0;
        pq = (double)pv * (double)q0;
      }
      if (e1) {
        const uint32_t e = 32 + lane;
        float pv = o[kOP + e];
        if (k > 0) pv = __fmaf_rn((float)os.beta, pv, o[kOZ + e]);
        o[kOP + e] = pv;
        o[kOQ + e] = q1;
        d.p[at + e] = pv;
        d.q[at + e] = q1;
        pq += (double)pv * (double)q1;
      }
      pq = warp_sum(pq);
      if (lane == 0) *dot_at(d, kDotPq + (k & 1), R) = pq;
      __syncwarp();
    }
    trace_mark(d, k, 2);
    ok = grid_barrier(d.barrier, G, d.error, &s_flag, bar_gen) && ok;
    trace_mark(d, k, 3);
    if (!ok) break;
    if (*(volatile unsigned int*)(d.barrier + 2) == 0u) break;  // every problem done

    // ---- C, one warp per owned row: alpha = rz / p.q of the row's
    // problem; x, r, z updates; the row's r.z and r.r.  The p.q of the
    // block's own problem is summed by the block's warps, one slot each
    // (the sums of pq_warp, which the warps use for other problems).
    const bool own_sc = sc_k == k && sc_prob != kNone;
    if (own_sc) {
      __syncthreads();
      if (warp < (uint32_t)kSumSlots) {
        const double v = pq_slot(d, k, d.prob_tr_begin[sc_prob], d.prob_tr_begin[sc_prob + 1],
                                 warp);
        if (lane == 0) s_slot[warp][0] = v;
      }
      __syncthreads();
    }
    uint32_t cprob = kNone;
    double alpha = 0.0;
    for (uint32_t j = warp; j < nown; j += NW) {
      const uint32_t tr = blockIdx.x + j * G;
      const uint32_t P = own_prob[j];
      if (P != cprob) {
        // The block's scalars of this iteration when they are this problem's
        // (the single-problem case), else this warp's own.
        const bool mine = own_sc && sc_prob == P;
        const ProbScal ps = mine ? sc : prob_scalars_warp(d, P, k);
        double pq = 0.0;
        if (mine) {
          const uint32_t t0 = d.prob_tr_begin[P], t1 = d.prob_tr_begin[P + 1];
          for (uint32_t w = 0; w < (uint32_t)kSumSlots && t0 + 32 * w < t1; ++w)
            pq += s_slot[w][0];
        } else {
          pq = pq_warp(d, P, k);
        }
        alpha = (ps.active && pq > 0.0 && isfinite(pq)) ? ps.rz / pq : 0.0;
        cprob = P;
      }
      if (alpha == 0.0) continue;  // inactive, or breakdown: x frozen, flagged at A(k+1)
      const size_t base = (size_t)tr * C::kRow;
      const float af = (float)alpha;
      float* o = ownrow(j);
      for (uint32_t e = lane; e < (uint32_t)C::kRow; e += 32) {
        const float xv = o[kOX + e] + af * o[kOP + e];
        o[kOX + e] = xv;
        d.x[base + e] = xv;
        const float rv = o[kOR + e] - af * o[kOQ + e];
        o[kOR + e] = rv;
        d.r[base + e] = rv;
        sPI[e] = rv;
      }
      __syncwarp();
      double rz = 0.0, rr = 0.0;
      for (uint32_t e = lane; e < (uint32_t)C::kRow; e += 32) {
        const uint32_t cam = e / 6;
        float z = 0.0f;
#pragma unroll
        for (int b = 0; b < 6; ++b) z += o[kOM + e * 6 + b] * sPI[cam * 6 + b];
        o[kOZ + e] = z;
        d.z[base + e] = z;
        rz += (double)sPI[e] * (double)z;
        rr += (double)sPI[e] * (double)sPI[e];
      }
      rz = warp_sum(rz);
      rr = warp_sum(rr);
      if (lane == 0) {
        *dot_at(d, kDotRz + mod3(k), tr) = rz;
        *dot_at(d, kDotRr + mod3(k), tr) = rr;
      }
      __syncwarp();
    }
    trace_mark(d, k, 4);
    ok = grid_barrier(d.barrier, G, d.error, &s_flag, bar_gen);
    trace_mark(d, k, 5);
  }
  // Drain the copies still in flight (prefetched tiles), bounded.
  if (lane == 0) {
    for (uint64_t s = consumed; s < issued; ++s) {
      const unsigned long long t_end = now_ns() + kWaitLimitNs;
      while (!mbar_try_wait(&mbar[warp][cst], cph) && now_ns() <= t_end) {
      }
      if (++cst == (uint32_t)C::kStages) {
        cst = 0u;
        cph ^= 1u;
      }
    }
  }
  // Return this warp's L2-resident tiles to the normal eviction priority.
  for (uint32_t m = 0; m < Mw; ++m) {
    const uint32_t t = gw + m * TW;
    if (t >= d.l2_resident_tiles) break;
    const char* base = reinterpret_cast<const char*>(d.tiles + (size_t)t * C::kTileFloats);
    for (uint32_t off = lane * 128u; off < C::kTileBytes; off += 32u * 128u)
      asm volatile("applypriority.global.L2::evict_normal [%0], 128;" ::"l"(base + off) : "memory");
  }
}

// A reduced camera system given by the caller (ReducedCameraSystem,
// pipelines/slam/src/ba_accel.rs:50-72) into the tiles: edge e's (row b,
// column a) block, column-major (f32, or the f64 blocks of a device
// elimination), to its row-major slot (and the mirrored slot in a diagonal
// tile); node i's damped diagonal block, column-major
// f64, to its diagonal slot, its FP64 Cholesky inverse (the block-Jacobi
// preconditioner; the diagonal's inverse if not positive definite) and its
// rhs.  Padding slots keep zero blocks, preconditioner and rhs.
__global__ void __launch_bounds__(256) k_reduced_fill(Dev d, uint32_t n, uint64_t ne,
                                                      const double* diag, const float* offdiag,
                                                      const double* offdiag64,
                                                      const double* rhs) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < ne; e += stride) {
    const uint2 dst = d.blk_dst[e];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const float v = offdiag ? offdiag[36 * e + c * 6 + r] : (float)offdiag64[36 * e + c * 6 + r];
        d.tiles[dst.x + r * 6 + c] = v;
        if (dst.y != kNone) d.tiles[dst.y + c * 6 + r] = v;
      }
  }
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < d.num_var_cams;
       i += stride) {
    double a[36], inv[36];
    if (i < n) {
      for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) a[r * 6 + c] = diag[36 * i + c * 6 + r];
      float* blk = d.tiles + d.diag_dst[i];
      for (int e2 = 0; e2 < 36; ++e2) blk[e2] = (float)a[e2];
      if (!chol_inverse6(a, inv)) {
        for (int e2 = 0; e2 < 36; ++e2) inv[e2] = 0.0;
        for (int q = 0; q < 6; ++q) inv[q * 7] = 1.0 / fmax(a[q * 7], 1e-20);
      }
      for (int q = 0; q < 6; ++q) d.rhs[6 * i + q] = (float)rhs[6 * i + q];
    } else {
      for (int e2 = 0; e2 < 36; ++e2) inv[e2] = 0.0;
      for (int q = 0; q < 6; ++q) d.rhs[6 * i + q] = 0.0f;
    }
    for (int e2 = 0; e2 < 36; ++e2) d.minv[36 * i + e2] = (float)inv[e2];
  }
}

// Self-test of the bounded waits: thread 0 waits on a flag that nothing
// sets, with the wait primitive the kernels use, until `limit_ns` has
// passed; it then sets the timeout bit and returns, recording how long it
// waited.
__global__ void k_wait_probe(const unsigned int* flag, unsigned long long limit_ns,
                             unsigned int* err, unsigned long long* waited) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const unsigned long long t0 = now_ns(), t_end = t0 + limit_ns;
  while (ld_acquire(flag) == 0u) {
    if (now_ns() > t_end) {
      atomicOr(err, (unsigned int)kErrBarrierTimeout);
      break;
    }
    __nanosleep(1000);
  }
  *waited = now_ns() - t0;
}

// Current state (buffer Ctrl::cur) of every problem into buffer 0.
// The off-diagonal assembly's block order: each window of 256 blocks in plan
// order sorted by the loop passes its blocks take at g lanes, longest first,
// ties in plan order (a block's rank is the count of blocks of its window
// before it in that order); each block's term range and destination are
// written at its place in that order.
__global__ void __launch_bounds__(256) k_block_order(const uint32_t* blk_off, const uint2* blk_dst,
                                                     uint32_t nb, uint32_t g, uint2* ord_range,
                                                     uint2* ord_dst, uint2* long_range,
                                                     uint2* long_dst, uint32_t* num_long) {
  __shared__ uint32_t key[256];
  const uint32_t b0 = blockIdx.x * 256u, t = threadIdx.x;
  const uint32_t n = min(256u, nb - b0);
  uint32_t k = 0;
  if (t < n) k = (blk_off[b0 + t + 1] - blk_off[b0 + t] + g - 1) / g;
  key[t] = k;
  __syncthreads();
  if (t < n) {
    uint32_t rank = 0;
    for (uint32_t j = 0; j < n; ++j) {
      const uint32_t kj = key[j];
      rank += (kj > k || (kj == k && j < t)) ? 1u : 0u;
    }
    const uint2 range = make_uint2(blk_off[b0 + t], blk_off[b0 + t + 1]);
    ord_range[b0 + rank] = range;
    ord_dst[b0 + rank] = blk_dst[b0 + t];
    if (range.y - range.x >= kLongBlockTerms) {
      const uint32_t at = atomicAdd(num_long, 1u);  // any order: a block's sums do not depend on it
      long_range[at] = range;
      long_dst[at] = blk_dst[b0 + t];
    }
  }
}

// The point of every Schur term, beside the term list (read by the
// off-diagonal assembly with the term, both coalesced).
__global__ void __launch_bounds__(256) k_pair_points(const uint2* pairs, const uint32_t* obs_point,
                                                     uint64_t n, uint32_t* pair_pt) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
       q += (uint64_t)gridDim.x * blockDim.x)
    pair_pt[q] = obs_point[pairs[q].x];
}

// The point of every listed observation, beside the per-slot lists (read
// by the camera-diagonal sums with the observation index, both coalesced).
__global__ void __launch_bounds__(256) k_cam_points(Dev d, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    d.cam_pt[i] = d.obs_point[d.cam_obs[i]];
}

__global__ void __launch_bounds__(256) k_state_to_front(Dev d) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < d.num_poses; p += stride) {
    if (d.ctrl[d.pose_prob[p]].cur == 0u) continue;
#pragma unroll
    for (int a = 0; a < 4; ++a) d.pose_q[0][4 * (size_t)p + a] = d.pose_q[1][4 * (size_t)p + a];
#pragma unroll
    for (int a = 0; a < 3; ++a) d.pose_t[0][3 * (size_t)p + a] = d.pose_t[1][3 * (size_t)p + a];
  }
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < d.num_points; l += stride) {
    if (d.ctrl[d.point_prob[l]].cur == 0u) continue;
#pragma unroll
    for (int a = 0; a < 3; ++a) d.points[0][3 * (size_t)l + a] = d.points[1][3 * (size_t)l + a];
  }
}

__global__ void __launch_bounds__(1024) k_pcg_setup(Dev d) {
  // Per-problem PCG state, grid-barrier words and the active count (one
  // block; problems and rows strided over its threads).
  __shared__ unsigned int active;
  if (threadIdx.x == 0) active = 0u;
  __syncthreads();
  unsigned int mine = 0;
  for (uint32_t P = threadIdx.x; P < d.num_problems; P += blockDim.x) {
    const bool on = !d.ctrl[P].done && d.prob_tr_begin[P + 1] > d.prob_tr_begin[P];
    PcgState& s = d.pcg[P];
    s.active = on ? 1u : 0u;
    s.iters = 0u;
    s.status = 0u;
    s.rz = 0.0;
    s.bnorm = 0.0;
    s.rnorm = 0.0;
    mine += on ? 1u : 0u;
  }
  if (mine) atomicAdd(&active, mine);
  __syncthreads();
  for (int w = threadIdx.x; w < kBarrierWords; w += blockDim.x) d.barrier[w] = w == 2 ? active : 0u;
}

}  // namespace

// ------------------------------------------------------------- launchers
static int grid1d(size_t n, int threads, int cap = 148 * 32) {
  size_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > (size_t)cap) g = cap;
  return (int)g;
}

cudaError_t launch_pose_table(const Dev& d, cudaStream_t s) {
  k_pose_table<<<grid1d(d.num_poses, 256), 256, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_cost(const Dev& d, bool trial, cudaStream_t s) {
  const int g = grid1d((size_t)d.num_point_chunks * 256, 256, 148 * 16);
  if (trial)
    k_cost<true><<<g, 256, 0, s>>>(d);
  else
    k_cost<false><<<g, 256, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_decide(const Dev& d, bool init, cudaStream_t s) {
  if (init)
    k_decide<true><<<d.num_problems, 256, 0, s>>>(d);
  else
    k_decide<false><<<d.num_problems, 256, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_linearize(const Dev& d, cudaStream_t s) {
  k_linearize<<<grid1d(d.num_obs, 256), 256, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_point_prep(const Dev& d, cudaStream_t s) {
  k_point_prep<<<grid1d(d.num_points, 256), 256, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_offdiag(const Dev& d, cudaStream_t s) {
  if (d.num_offdiag_blocks == 0) return cudaSuccess;
  const size_t threads_needed = (size_t)d.num_offdiag_blocks * d.group;
  const int g = grid1d(threads_needed, 256, 148 * 16);
  switch (d.group) {
    case 1: k_offdiag<1, false><<<g, 256, 0, s>>>(d); break;
    case 2: k_offdiag<2, false><<<g, 256, 0, s>>>(d); break;
    case 4: k_offdiag<4, false><<<g, 256, 0, s>>>(d); break;
    case 8: k_offdiag<8, false><<<g, 256, 0, s>>>(d); break;
    case 16: k_offdiag<16, false><<<g, 256, 0, s>>>(d); break;
    default: k_offdiag<32, false><<<g, 256, 0, s>>>(d); break;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (d.num_long_blocks == 0) return cudaSuccess;
  const int gl = grid1d((size_t)d.num_long_blocks * kLongLanes, 256, 148 * 16);
  k_offdiag<kLongLanes, true><<<gl, 256, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_cam_diag(const Dev& d, cudaStream_t s) {
  if (d.num_var_cams == 0) return cudaSuccess;
  const int g = d.num_var_cams < 148u * 16u ? (int)d.num_var_cams : 148 * 16;
  k_cam_diag<<<g, kDiagThreads, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_pose_update(const Dev& d, cudaStream_t s) {
  k_pose_update<<<grid1d(d.num_poses, 256), 256, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_pcg_setup(const Dev& d, cudaStream_t s) {
  k_pcg_setup<<<1, 1024, 0, s>>>(d);
  return cudaGetLastError();
}

size_t pcg_smem_bytes(int) { return Pcg::kSmem; }
int pcg_rows_per_block() { return Pcg::kOwnMax; }

cudaError_t launch_reduced_fill(const Dev& d, uint32_t n, uint64_t ne, const double* diag,
                                const float* offdiag, const double* offdiag64, const double* rhs,
                                cudaStream_t s) {
  const size_t work = std::max<size_t>((size_t)ne, d.num_var_cams);
  k_reduced_fill<<<grid1d(work, 256), 256, 0, s>>>(d, n, ne, diag, offdiag, offdiag64, rhs);
  return cudaGetLastError();
}

cudaError_t launch_wait_probe(const unsigned int* flag, unsigned long long limit_ns,
                              unsigned int* err, unsigned long long* waited, cudaStream_t s) {
  k_wait_probe<<<1, 32, 0, s>>>(flag, limit_ns, err, waited);
  return cudaGetLastError();
}

// Squared reprojection residual of every observation at the state in
// buffer 0 (after k_state_to_front), in plan order; NaN where the
// observation cannot be evaluated (behind the sensor or outside the
// projection's domain): reprojection_squared_residuals (bundle/problem.rs:
// 756-830), the input of the GNC weights.
__global__ void __launch_bounds__(256) k_sq_residuals(Dev d, double* out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < d.num_obs;
       k += gridDim.x * blockDim.x) {
    const uint32_t p = d.obs_pose[k], l = d.obs_point[k];
    double q[4], rt[12], X[3], xs[3], pred[2];
#pragma unroll
    for (int a = 0; a < 4; ++a) q[a] = d.pose_q[0][4 * (size_t)p + a];
    quat_to_matrix(q, rt);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      rt[9 + a] = d.pose_t[0][3 * (size_t)p + a];
      X[a] = d.points[0][3 * (size_t)l + a];
    }
    const DevCamera& cam = d.cameras[d.obs_cam[k]];
    to_sensor(rt, cam, X, xs);
    double s = __longlong_as_double(0x7ff8000000000000ll);  // NaN
    const uint32_t kind = d.obs_kind ? d.obs_kind[k] : kObsMono;
    if (kind != kObsMono) {
      double r[4];
      const int m = stereo_rows(kind, cam, d.cameras[d.obs_rcam[k]], d.obs_xy[k], d.obs_st[k], xs,
                                nullptr, r, nullptr);
      if (m) {
        s = 0.0;
        for (int i = 0; i < m; ++i) s += r[i] * r[i];
      }
    } else if (xs[2] > 0.0 && camera_project(cam, xs, pred)) {
      const double2 xy = d.obs_xy[k];
      const double rx = pred[0] - xy.x, ry = pred[1] - xy.y;
      s = rx * rx + ry * ry;
    }
    out[k] = s;
  }
}

cudaError_t launch_sq_residuals(const Dev& d, double* out, cudaStream_t s) {
  k_sq_residuals<<<grid1d(d.num_obs, 256), 256, 0, s>>>(d, out);
  return cudaGetLastError();
}

cudaError_t launch_pair_points(const Dev& d, uint64_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_pair_points<<<grid1d(n, 256), 256, 0, s>>>(d.pairs, d.obs_point, n, d.pair_pt);
  return cudaGetLastError();
}

cudaError_t launch_block_order(const Dev& d, cudaStream_t s) {
  if (d.num_offdiag_blocks == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(d.num_long, 0, 4, s);
  if (e != cudaSuccess) return e;
  k_block_order<<<(d.num_offdiag_blocks + 255) / 256, 256, 0, s>>>(
      d.blk_off, d.blk_dst, d.num_offdiag_blocks, d.group, const_cast<uint2*>(d.ord_range),
      const_cast<uint2*>(d.ord_dst), const_cast<uint2*>(d.long_range),
      const_cast<uint2*>(d.long_dst), d.num_long);
  return cudaGetLastError();
}

cudaError_t launch_cam_points(const Dev& d, uint32_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_cam_points<<<grid1d(n, 256), 256, 0, s>>>(d, n);
  return cudaGetLastError();
}

cudaError_t launch_state_to_front(const Dev& d, cudaStream_t s) {
  const size_t n = std::max<size_t>(d.num_poses, d.num_points);
  k_state_to_front<<<grid1d(n, 256), 256, 0, s>>>(d);
  return cudaGetLastError();
}

int pcg_grid_size(int, int sm_count) {
  int per_sm = 0;
  cudaFuncSetAttribute(k_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Pcg::kSmem);
  const cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg, Pcg::kThreads, Pcg::kSmem);
  if (e != cudaSuccess || per_sm <= 0) return 0;
  return per_sm * sm_count;
}

cudaError_t launch_pcg(const Dev& d, int grid, cudaStream_t s) {
  if (d.num_tile_rows == 0) return cudaSuccess;
  void* args[] = {const_cast<Dev*>(&d)};
  return cudaLaunchCooperativeKernel((const void*)k_pcg, grid, Pcg::kThreads, args, Pcg::kSmem, s);
}

}  // namespace vlba
