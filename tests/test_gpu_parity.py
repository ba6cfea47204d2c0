"""CUDA solver against the FP64 oracle, through the C ABI.

Tolerances (stated by the solver's precision contract): final cost within
1e-5 relative of the oracle's FP64 solve and camera centres within 1e-5 of
the scene extent; the bit-exact cases are marked."""

from __future__ import annotations

import numpy as np
import pytest

from _scenes import center_error, drifted_bundle, pinhole
from oracle import oracle
from visloc_ba import BaConfig, Camera, CameraModel, RobustKernel, synth
from visloc_ba import _abi
from visloc_ba.solver import GpuBundleAdjuster, GpuBaSettings

pytestmark = pytest.mark.gpu

COST_RTOL = 1e-5
CENTER_TOL = 1e-5  # of the scene extent


def tight(cfg: BaConfig) -> BaConfig:
    cfg.max_pcg_iterations = 300
    cfg.pcg_relative_tolerance = 1e-8
    return cfg


def compare(solver, problem, cfg, cost_rtol=COST_RTOL, center_tol=CENTER_TOL):
    gpu, ref = problem.copy(), problem.copy()
    st, res = solver.optimize(gpu, cfg)
    assert st == _abi.OK, solver.last_error()
    st_ref, res_ref = oracle.optimize(ref, cfg)
    assert st_ref == _abi.OK
    assert res.initial_cost == pytest.approx(res_ref.initial_cost, rel=1e-12)
    rel = abs(res.final_cost - res_ref.final_cost) / max(abs(res_ref.final_cost), 1e-300)
    extent = synth.scene_extent(ref)
    dc = np.abs(gpu.camera_centers() - ref.camera_centers()).max() / extent
    assert rel <= cost_rtol, (res.final_cost, res_ref.final_cost, rel)
    assert dc <= center_tol, dc
    return res, res_ref, gpu, ref


def test_initial_cost_matches_the_oracle(solver):
    p = synth.ring_problem(30, 3000, seed=11)
    for k in (RobustKernel.none(), RobustKernel.huber(1.0), RobustKernel.cauchy(2.0)):
        cfg = BaConfig(robust_kernel=k)
        c, n = solver.cost(p, cfg)
        c_ref, n_ref = oracle.cost(p, cfg)
        assert n == n_ref
        assert c == pytest.approx(c_ref, rel=1e-12)


def test_drifted_pose_returns_to_truth(solver):
    """The reference's bundle_optimize_pulls_drifted_pose_back_to_truth
    (tests/bundle_adjustment.rs:367-402) through the accelerator."""
    ba = drifted_bundle()
    acc = GpuBundleAdjuster(0, GpuBaSettings(100, 1e-4, True))
    res = acc.solve(ba, BaConfig())
    assert res.final_cost < 1e-12
    assert res.final_cost < res.initial_cost
    assert res.converged
    assert center_error(ba, 30, (1.0, 0.0, 0.0)) < 1e-6


@pytest.mark.parametrize("model,params", [
    (CameraModel.PINHOLE, [500.0, 500.0, 320.0, 240.0, -0.15, 0.05]),
    (CameraModel.SIMPLE_RADIAL, [500.0, 320.0, 240.0, -0.1]),
    (CameraModel.RADIAL, [500.0, 320.0, 240.0, -0.1, 0.03]),
])
def test_distorted_bundle_converges(model, params):
    """pose_structure_ba_uses_radial_distortion_in_residual_and_jacobian (:455)."""
    ba = drifted_bundle(Camera(model, 640, 480, params))
    acc = GpuBundleAdjuster(0, GpuBaSettings(100, 1e-6, True))
    res = acc.solve(ba, BaConfig())
    assert res.final_cost < 1e-10
    assert center_error(ba, 30, (1.0, 0.0, 0.0)) < 1e-5


def test_ring_50_simple_radial_matches_the_oracle(solver):
    """The 50-camera SIMPLE_RADIAL ring (per-camera intrinsics, Huber 1 px,
    20 LM iterations)."""
    p = synth.ring_problem(50, 5000, seed=1001)
    cfg = tight(BaConfig(max_iterations=20, robust_kernel=RobustKernel.huber(1.0)))
    compare(solver, p, cfg)


@pytest.mark.parametrize("seed,kernel", [(1, RobustKernel.none()),
                                         (2, RobustKernel.huber(1.0)),
                                         (3, RobustKernel.cauchy(2.0))])
def test_shared_pinhole_ring_matches_the_oracle(solver, seed, kernel):
    p = synth.ring_problem(40, 4000, seed=seed, width=2000, height=1500, focal=(1500, 1500),
                           k1=(0.0, 0.0), per_camera_intrinsics=False,
                           track=("geometric", 8.0, 2, 40))
    cfg = tight(BaConfig(max_iterations=12, robust_kernel=kernel))
    compare(solver, p, cfg)


def test_street_loop_matches_the_oracle(solver):
    """A closed loop of forward-facing cameras with facade points seen by runs
    of consecutive views: a banded reduced system closed at the loop.  Forward
    motion with short tracks leaves a flat cost valley that LM crosses slowly
    (the camera centres still move 5e-4 of the extent between iterations 30
    and 60 in the oracle), where two solvers' states cannot be compared; this
    case has anchor poses around the loop and longer tracks, and enough
    iterations for both to settle (near the end an FP32 step can be rejected
    where the FP64 one is accepted, which the next iterations make up); the
    default street geometry is compared through its reduced system and one
    step."""
    p = synth.street_loop(240, 15000, seed=17, fixed=(0, 1, 120), track=(12.0, 4, 40),
                          outlier_fraction=0.0)
    cfg = tight(BaConfig(max_iterations=20, robust_kernel=RobustKernel.huber(1.0)))
    compare(solver, p, cfg)


def test_street_loop_reduced_system_and_step(solver):
    """The default street geometry at lambda = 0.1.  (At lambda = 1e-3 the
    points' nearly singular depth makes S_ii = H_pp - sum W H^-1 W^T cancel to
    about 1e-3 of H_pp, so the FP32 Jacobian records leave ~1e-4 relative
    error there and the step differs along the flat directions: the FP32
    contract cannot resolve that system, only its damped neighbours.)"""
    p = synth.street_loop(240, 15000, seed=18)
    cfg = BaConfig(robust_kernel=RobustKernel.huber(1.0), max_pcg_iterations=1000,
                   pcg_relative_tolerance=1e-7)
    lam = 0.1
    s, rhs = solver.reduced_system(p, cfg, lam)
    st, s_ref, rhs_ref, dp_ref, dl_ref = oracle.reduced_system(p, lam, cfg)
    assert st == 0
    assert np.abs(s - s_ref).max() <= 2e-5 * np.abs(s_ref).max()
    assert np.abs(rhs - rhs_ref).max() <= 2e-5 * np.abs(rhs_ref).max()
    dp, dl, iters, rr = solver.linear_step(p, cfg, lam)
    assert rr <= 1e-7
    assert np.abs(dp - dp_ref).max() <= 1e-2 * np.abs(dp_ref).max()


def test_stereo_window_matches_the_oracle(solver):
    """Rig observations (right camera as sensor_from_rig), 10% poses fixed."""
    p = synth.stereo_window(20, 1500, seed=6)
    # 20 iterations: the FP32 and FP64 solves take the same accept/reject and
    # lambda sequence, but mid-way their costs differ by up to 2e-4 before
    # meeting again (1.7e-5 at iteration 10, 9e-8 at 20).
    cfg = tight(BaConfig(max_iterations=20, robust_kernel=RobustKernel.huber(1.0)))
    compare(solver, p, cfg)


def test_pose_only_refinement_matches_the_oracle(solver):
    """One free camera, fixed landmarks, 30% outliers, Cauchy kernel."""
    p = synth.pose_only(800, seed=4)
    cfg = tight(BaConfig(max_iterations=10, robust_kernel=RobustKernel.cauchy(2.0)))
    compare(solver, p, cfg)


def test_landmark_only_matches_the_oracle(solver):
    """Every pose fixed: the landmark-only step (normal_equations.rs:1332-1371)."""
    p = synth.ring_problem(10, 500, seed=8)
    p.pose_fixed[:] = 1
    cfg = BaConfig(max_iterations=8, robust_kernel=RobustKernel.huber(1.0))
    res, res_ref, gpu, ref = compare(solver, p, cfg)
    assert np.abs(gpu.landmarks - ref.landmarks).max() < 1e-6 * synth.scene_extent(ref)


def test_pure_gauss_newton_matches_the_oracle(solver):
    """initial_lambda = None: every solved step is accepted (lm.rs:804-808)."""
    # Every point seen by >= 3 cameras: the undamped system is well posed.
    p = synth.ring_problem(12, 600, seed=12, outlier_fraction=0.0, track=("uniform", 3, 6))
    cfg = tight(BaConfig(max_iterations=6, initial_lambda=None))
    res, res_ref, _, _ = compare(solver, p, cfg)
    assert [i.step_accepted for i in res.iterations] == [i.step_accepted for i in res_ref.iterations]


def test_iteration_trace_matches_the_oracle(solver):
    p = synth.ring_problem(20, 1500, seed=21)
    cfg = tight(BaConfig(max_iterations=10, robust_kernel=RobustKernel.huber(1.0)))
    res, res_ref, _, _ = compare(solver, p, cfg)
    assert len(res.iterations) == len(res_ref.iterations)
    for a, b in zip(res.iterations, res_ref.iterations):
        assert a.step_accepted == b.step_accepted
        assert a.lambda_ == b.lambda_
        assert a.cost_after == pytest.approx(b.cost_after, rel=1e-4)


def test_solves_are_bitwise_repeatable(solver):
    p = synth.ring_problem(30, 2500, seed=31)
    cfg = BaConfig(max_iterations=8, robust_kernel=RobustKernel.huber(1.0))
    a, b = p.copy(), p.copy()
    assert solver.optimize(a, cfg)[0] == 0
    assert solver.optimize(b, cfg)[0] == 0
    assert np.array_equal(a.pose_q, b.pose_q)
    assert np.array_equal(a.pose_t, b.pose_t)
    assert np.array_equal(a.landmarks, b.landmarks)


def test_upload_solve_download_equals_optimize(solver):
    p = synth.ring_problem(16, 900, seed=41)
    cfg = BaConfig(max_iterations=6, robust_kernel=RobustKernel.huber(1.0))
    a = p.copy()
    assert solver.optimize(a, cfg)[0] == 0
    b = p.copy()
    assert solver.upload(b, cfg) == 0
    for _ in range(2):  # the uploaded initial state is reused
        st, res = solver.solve_uploaded(cfg)
        assert st == 0
    assert solver.download(b) == 0
    assert np.array_equal(a.pose_q, b.pose_q) and np.array_equal(a.landmarks, b.landmarks)


def test_errors_surface_as_ba_errors(solver):
    from visloc_ba import BaError, BundleAdjustment, BaObservation, Pose

    ba = BundleAdjustment(pinhole())
    ba.add_pose(1, Pose())
    ba.add_landmark(2, (0.0, 0.0, 5.0))
    ba.add_observation(BaObservation(1, 9, (320.0, 240.0)))
    acc = GpuBundleAdjuster(0)
    with pytest.raises(BaError) as e:
        acc.solve(ba, BaConfig())
    assert e.value.kind == "MissingLandmark" and e.value.id == 9


def test_unsupported_lens_is_declined():
    from visloc_ba import BaScope

    ba = drifted_bundle(Camera(CameraModel.OTHER, 640, 480, [300.0, 300.0, 320.0, 240.0]))
    acc = GpuBundleAdjuster(0)
    assert acc.optimize(ba, BaConfig(), BaScope.GLOBAL) is None
    assert acc.optimize(drifted_bundle(), BaConfig(), BaScope.LOCAL) is None  # local off


@pytest.mark.parametrize("ncams", [30, 70])  # 8-wide and 16-wide Schur tiles
def test_reduced_system_matches_the_oracle(solver, ncams):
    """The assembled damped reduced camera system S and its rhs against the
    oracle's FP64 Schur complement (normal_equations.rs:1621-1700)."""
    p = synth.ring_problem(ncams, 3000, seed=50 + ncams)
    cfg = BaConfig(robust_kernel=RobustKernel.huber(1.0))
    lam = 1e-3
    s, rhs = solver.reduced_system(p, cfg, lam)
    st, s_ref, rhs_ref, _, _ = oracle.reduced_system(p, lam, cfg, step=False)
    assert st == 0
    scale = np.abs(s_ref).max()
    assert np.abs(s - s_ref).max() <= 2e-5 * scale
    assert np.abs(rhs - rhs_ref).max() <= 2e-5 * np.abs(rhs_ref).max()


@pytest.mark.parametrize("ncams", [30, 70])
def test_linear_step_matches_the_exact_solve(solver, ncams):
    """One damped step (PCG on S + back-substitution) against the oracle's
    Cholesky solve of the same system."""
    p = synth.ring_problem(ncams, 3000, seed=60 + ncams)
    cfg = BaConfig(robust_kernel=RobustKernel.huber(1.0), max_pcg_iterations=500,
                   pcg_relative_tolerance=1e-7)
    lam = 1e-2
    dp, dl, iters, rr = solver.linear_step(p, cfg, lam)
    st, _, _, dp_ref, dl_ref = oracle.reduced_system(p, lam, cfg)
    assert st == 0
    assert rr <= 1e-7 and iters < 500
    assert np.abs(dp - dp_ref).max() <= 1e-3 * np.abs(dp_ref).max()
    assert np.abs(dl - dl_ref).max() <= 1e-3 * np.abs(dl_ref).max()


@pytest.mark.parametrize("flag", ["refine_intrinsics", "refine_distortion",
                                  "refine_tangential_distortion", "shared_focal"])
def test_accelerator_declines_intrinsics_refinement(flag):
    """BaConfig{refine_intrinsics: true} must not be solved with the
    intrinsics held: the plug-in returns None, as GpuBundleAdjuster::check
    makes it do (crates/ba-gpu/src/solver.rs:214-216), and `ba` is untouched;
    the same problem without the flag is solved."""
    ba = drifted_bundle()
    before = {k: p.world_to_camera for k, p in ba.poses.items()}
    acc = GpuBundleAdjuster(0, GpuBaSettings(100, 1e-6, True))
    assert acc.optimize(ba, BaConfig(**{flag: True})) is None
    assert {k: p.world_to_camera for k, p in ba.poses.items()} == before
    res = acc.optimize(ba, BaConfig())
    assert res is not None and res.final_cost < 1e-12
