"""Graduated non-convexity (BundleAdjustment::optimize_gnc, bundle/lm.rs:
28-142; surrogate math of pipelines/slam/src/gnc.rs).

CPU: the oracle's GNC restatement -- the surrogate weights, the mu schedule
and the MAD scale against their closed forms, and the whole loop rejecting
planted outliers.  GPU: the library's GNC (C++ driver over the device's
weighted LM) against the oracle's, level for level: the same outer levels,
the same inlier/outlier verdicts, the final estimate within the solver's
parity tolerance."""

from __future__ import annotations

import math

import numpy as np
import pytest

from _scenes import drifted_bundle
from oracle import oracle
from visloc_ba import AUTO_SCALE_K, BaConfig, GncConfig, PackedProblem, synth
from visloc_ba import _abi
from visloc_ba.solver import GpuBaSettings, GpuBundleAdjuster

GM, TLS = _abi.GNC_GEMAN_MCCLURE, _abi.GNC_TRUNCATED_LEAST_SQUARES
COST_RTOL = 1e-5
CENTER_TOL = 1e-5  # of the scene extent


def outlier_scene(num_cameras=12, num_points=500, seed=5, fraction=0.08, px=(25.0, 60.0)):
    """A ring with 0.5 px noise and a planted set of gross outliers (shifted
    by 25-60 px in a random direction): (problem, outlier mask)."""
    p = synth.ring_problem(num_cameras, num_points, seed=seed, sigma=0.5, outlier_fraction=0.0,
                           k1=(0.0, 0.0), track=("uniform", 3, 8))
    rng = np.random.default_rng(seed + 100)
    out = rng.random(p.num_observations) < fraction
    ang = rng.uniform(0.0, 2.0 * math.pi, int(out.sum()))
    mag = rng.uniform(px[0], px[1], int(out.sum()))
    xy = p.obs_xy.copy()
    xy[out, 0] += mag * np.cos(ang)
    xy[out, 1] += mag * np.sin(ang)
    q = PackedProblem(p.pose_q, p.pose_t, p.landmarks, p.obs_pose, p.obs_landmark, xy, p.cameras,
                      p.pose_fixed, p.landmark_fixed, p.obs_camera)
    return q, out


def inner_cfg() -> BaConfig:
    return BaConfig(max_pcg_iterations=300, pcg_relative_tolerance=1e-8)


# ------------------------------------------------------------------ CPU side
def test_geman_mcclure_schedule():
    s_max, c = 400.0, 2.0
    g = oracle.GncSurrogate(GM, c, 1.4, s_max)
    assert g.mu == pytest.approx(2.0 * s_max / (c * c))
    # The first surrogate keeps every residual at a substantial weight.
    assert g.weight(s_max) == pytest.approx(4.0 / 9.0)
    assert g.weight(0.0) == 1.0
    levels = 0
    while not g.anneal():
        levels += 1
    assert g.mu == 1.0 and levels == math.ceil(math.log(200.0) / math.log(1.4)) - 1
    for s in (0.0, 1.0, 4.0, 50.0):
        assert g.weight(s) == pytest.approx((4.0 / (s + 4.0)) ** 2)
    assert oracle.GncSurrogate(GM, 1.0, 1.4, 0.1).mu == 1.0  # never below 1


def test_truncated_least_squares_bands():
    c = 1.5
    g = oracle.GncSurrogate(TLS, c, 1.4, 10.0)
    assert g.mu == pytest.approx(c * c / (20.0 - c * c))
    for _ in range(6):
        lo = g.mu / (g.mu + 1.0) * g.c2
        hi = (g.mu + 1.0) / g.mu * g.c2
        assert g.weight(lo) == 1.0 and g.weight(0.5 * lo) == 1.0
        assert g.weight(hi) == 0.0 and g.weight(2.0 * hi) == 0.0
        mid = [g.weight(lo + (hi - lo) * t) for t in (0.1, 0.5, 0.9)]
        assert 1.0 > mid[0] > mid[1] > mid[2] > 0.0
        # Continuous at both band edges.
        assert g.weight(lo * (1 + 1e-12)) == pytest.approx(1.0, abs=1e-6)
        assert g.weight(hi * (1 - 1e-12)) == pytest.approx(0.0, abs=1e-6)
        g.anneal()
    assert oracle.GncSurrogate(TLS, 2.0, 1.4, 1.0).terminal()  # all inliers from the start
    while not g.anneal():
        pass
    assert g.mu == oracle.TLS_TERMINAL_MU


def test_mad_scale():
    assert oracle.estimate_scale_mad([4.0], 3.5) is None
    assert oracle.estimate_scale_mad([float("nan"), -1.0, 9.0], 3.5) is None
    sq = [r * r for r in (1.0, 2.0, 3.0, 4.0, 100.0)]  # norms 1..4 and one outlier
    # median 3, deviations (2,1,0,1,97) -> MAD 1.
    assert oracle.estimate_scale_mad(sq, 3.5) == pytest.approx(3.0 + 3.5 * 1.4826)
    assert oracle.estimate_scale_mad(sq + [float("nan")], 0.0) == pytest.approx(3.0)


def test_oracle_gnc_rejects_planted_outliers():
    p, out = outlier_scene()
    res, w = oracle.optimize_gnc(p, inner_cfg(), GncConfig(c=3.0))
    assert res["converged"] and res["outer_iterations"] >= 10
    rejected = w < 0.5
    assert (rejected & out).sum() >= 0.95 * out.sum()
    assert (rejected & ~out).sum() <= 0.01 * (~out).sum()
    assert res["inlier_cost"] < res["initial_cost"]


# ------------------------------------------------------------------ GPU side
@pytest.mark.gpu
@pytest.mark.parametrize("gnc", [
    GncConfig(c=3.0),
    GncConfig(kernel=TLS, c=3.0),
    GncConfig(c=1.0, auto_scale=AUTO_SCALE_K, auto_scale_readapt=True, inner_iterations=3),
])
def test_gnc_matches_the_oracle(solver, gnc):
    p, out = outlier_scene()
    gpu, ref = p.copy(), p.copy()
    st, res = solver.optimize_gnc(gpu, inner_cfg(), gnc)
    assert st == _abi.OK, solver.last_error()
    want, w_ref = oracle.optimize_gnc(ref, inner_cfg(), gnc)
    assert res.outer_iterations == want["outer_iterations"]
    assert res.converged == want["converged"]
    assert res.initial_cost == pytest.approx(want["initial_cost"], rel=1e-12)
    # Re-estimated from the residuals at each level's estimate, so it carries
    # the estimate's tolerance; fixed (or estimated once, at the input) it is
    # exact.
    tol = COST_RTOL if gnc.auto_scale_readapt else 1e-12
    assert res.inlier_scale == pytest.approx(want["inlier_scale"], rel=tol)
    assert np.array_equal(res.observation_weights >= 0.5, w_ref >= 0.5)
    assert res.final_cost == pytest.approx(want["final_cost"], rel=COST_RTOL)
    assert res.inlier_cost == pytest.approx(want["inlier_cost"], rel=COST_RTOL)
    extent = synth.scene_extent(ref)
    assert np.abs(gpu.camera_centers() - ref.camera_centers()).max() <= CENTER_TOL * extent
    rejected = res.observation_weights < 0.5
    assert (rejected & out).sum() >= 0.9 * out.sum()


@pytest.mark.gpu
def test_gnc_refuses_caller_weights(solver):
    p, _ = outlier_scene(num_cameras=8, num_points=200)
    p.obs_weight = np.ones(p.num_observations)
    st, res = solver.optimize_gnc(p, inner_cfg(), GncConfig())
    assert st == _abi.ERR_INVALID_ARGUMENT and res is None


@pytest.mark.gpu
def test_accelerator_gnc():
    acc = GpuBundleAdjuster(0, GpuBaSettings(300, 1e-8, True))
    ba = drifted_bundle()
    res = acc.optimize_gnc(ba, BaConfig(), GncConfig(c=3.0))
    assert res.converged
    assert res.observation_weights.shape == (len(ba.observations),)
    assert res.final_cost <= res.initial_cost
