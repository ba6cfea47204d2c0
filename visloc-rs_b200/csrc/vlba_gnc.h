// vlba_gnc.h -- graduated non-convexity (the reference's crate gnc,
// pipelines/slam/src/gnc.rs): the Black-Rangarajan weights of the
// Geman-McClure and truncated-least-squares surrogates, the mu schedule that
// anneals them from least squares to the robust cost, and the MAD estimate of
// the inlier scale.  Host code, FP64; the driver (BundleAdjustment::
// optimize_gnc, bundle/lm.rs:28-142) is in vlba_solver.cu.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/visloc_ba_cuda.h"

namespace vlba {

// mu past which the truncated-least-squares transition band is under 1% of
// c^2 (gnc.rs:146-149): the surrogate is the hard truncated quadratic.
constexpr double kTlsTerminalMu = 200.0;

struct GncState {
  uint32_t kernel = VLBA_GNC_GEMAN_MCCLURE;
  double c2 = 1.0;
  double factor = 1.4;
  double mu = 1.0;

  // The first surrogate convex over residuals up to max_residual_sq
  // (GncState::new, gnc.rs:160-185).
  static GncState start(uint32_t kernel, double c, double factor, double max_residual_sq) {
    GncState g;
    g.kernel = kernel;
    g.c2 = c * c;
    g.factor = factor;
    const double s_max = std::max(max_residual_sq, 0.0);
    if (kernel == VLBA_GNC_TRUNCATED_LEAST_SQUARES) {
      const double denom = 2.0 * s_max - g.c2;
      g.mu = denom <= 0.0 ? kTlsTerminalMu : std::clamp(g.c2 / denom, DBL_MIN, kTlsTerminalMu);
    } else {
      g.mu = std::max(2.0 * s_max / g.c2, 1.0);
    }
    return g;
  }

  void set_inlier_scale(double c) { c2 = c * c; }

  // Weight in [0, 1] of a squared residual s (GncState::weight, gnc.rs:200-230).
  double weight(double s) const {
    s = std::max(s, 0.0);
    if (kernel == VLBA_GNC_TRUNCATED_LEAST_SQUARES) {
      const double lo = (mu / (mu + 1.0)) * c2, hi = ((mu + 1.0) / mu) * c2;
      if (s <= lo) return 1.0;
      if (s >= hi) return 0.0;
      return std::sqrt(c2 * mu * (mu + 1.0) / s) - mu;
    }
    const double m = mu * c2, r = m / (s + m);
    return r * r;
  }

  bool terminal() const {
    return kernel == VLBA_GNC_TRUNCATED_LEAST_SQUARES ? mu >= kTlsTerminalMu : mu <= 1.0;
  }

  // One geometric step of mu toward the robust cost (GncState::anneal,
  // gnc.rs:233-243).
  bool anneal() {
    if (kernel == VLBA_GNC_TRUNCATED_LEAST_SQUARES) mu = std::min(mu * factor, kTlsTerminalMu);
    else mu = std::max(mu / factor, 1.0);
    return terminal();
  }
};

// median(rho) + k 1.4826 MAD(rho) over rho = sqrt(s) of the finite,
// non-negative squared residuals (estimate_scale_mad, gnc.rs:250-270);
// false with fewer than two of them.
inline double median_sorted_in_place(std::vector<double>& v) {
  std::sort(v.begin(), v.end());
  const size_t n = v.size();
  return n % 2 ? v[n / 2] : 0.5 * (v[n / 2 - 1] + v[n / 2]);
}

inline bool estimate_scale_mad(const std::vector<double>& squared, double k, double* scale) {
  std::vector<double> rho;
  rho.reserve(squared.size());
  for (double s : squared)
    if (std::isfinite(s) && s >= 0.0) rho.push_back(std::sqrt(s));
  if (rho.size() < 2) return false;
  const double med = median_sorted_in_place(rho);
  for (double& r : rho) r = std::fabs(r - med);
  const double mad = median_sorted_in_place(rho);
  *scale = med + k * 1.4826 * mad;
  return true;
}

}  // namespace vlba
