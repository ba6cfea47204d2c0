"""External per-observation weights (BundleAdjustment::
optimize_with_observation_weights, bundle/optimize.rs:43-53): each weight
multiplies its observation's robust IRLS weight in the normal equations
(normal_equations.rs:458) and its robust cost (problem.rs:497-560); invalid
weights are rejected with the observation's index (optimize.rs:628-650).

The CPU tests pin the oracle's weighted solve by two exact identities of the
definition: unit weights change nothing, and a zero weight removes the
observation.  The GPU tests hold the CUDA path to the oracle."""

from __future__ import annotations

import numpy as np
import pytest

from _scenes import drifted_bundle
from oracle import oracle
from visloc_ba import BaConfig, BaError, PackedProblem, RobustKernel, synth
from visloc_ba import _abi
from visloc_ba.solver import GpuBaSettings, GpuBundleAdjuster, check

COST_RTOL = 1e-5
CENTER_TOL = 1e-5  # of the scene extent


def with_weights(p: PackedProblem, w) -> PackedProblem:
    q = p.copy()
    q.obs_weight = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
    return q


def without(p: PackedProblem, drop) -> PackedProblem:
    keep = ~drop
    return PackedProblem(p.pose_q.copy(), p.pose_t.copy(), p.landmarks.copy(), p.obs_pose[keep],
                         p.obs_landmark[keep], p.obs_xy[keep], p.cameras, p.pose_fixed,
                         p.landmark_fixed, None if p.obs_camera is None else p.obs_camera[keep])


def droppable(p: PackedProblem, n: int, seed: int) -> np.ndarray:
    """n observations, at most one per landmark and only of landmarks seen at
    least three times, so every landmark keeps two observations."""
    rng = np.random.default_rng(seed)
    counts = np.bincount(p.obs_landmark, minlength=p.num_landmarks)
    drop = np.zeros(p.num_observations, bool)
    used = set()
    for o in rng.permutation(p.num_observations):
        lm = int(p.obs_landmark[o])
        if counts[lm] >= 3 and lm not in used:
            drop[o] = True
            used.add(lm)
            if drop.sum() == n:
                break
    return drop


def cfg(**kw) -> BaConfig:
    base = dict(max_iterations=8, robust_kernel=RobustKernel.huber(1.0), max_pcg_iterations=300,
                pcg_relative_tolerance=1e-8)
    base.update(kw)
    return BaConfig(**base)


# ------------------------------------------------------------------ CPU side
def test_invalid_weights_are_reported_with_their_index():
    p = synth.ring_problem(8, 200, seed=3)
    w = np.ones(p.num_observations)
    w[17] = -0.5
    assert check(with_weights(p, w)) == (_abi.ERR_INVALID_OBSERVATION_WEIGHT, 17)
    w[17] = 1.0
    w[40] = np.nan
    assert check(with_weights(p, w)) == (_abi.ERR_INVALID_OBSERVATION_WEIGHT, 40)
    w[40] = np.inf
    assert check(with_weights(p, w)) == (_abi.ERR_INVALID_OBSERVATION_WEIGHT, 40)
    assert oracle.check(with_weights(p, w))[0] == _abi.ERR_INVALID_OBSERVATION_WEIGHT
    # Weights are checked before the problem itself, as the reference does.
    bad = PackedProblem(p.pose_q, p.pose_t, p.landmarks,
                        np.where(np.arange(p.num_observations) == 5, 999, p.obs_pose),
                        p.obs_landmark, p.obs_xy, p.cameras, p.pose_fixed, p.landmark_fixed)
    assert check(with_weights(bad, w))[0] == _abi.ERR_INVALID_OBSERVATION_WEIGHT
    w[40] = 0.0
    assert check(with_weights(p, w))[0] == _abi.OK
    assert check(with_weights(bad, w)) == (_abi.ERR_MISSING_POSE, 999)


def test_oracle_unit_weights_change_nothing():
    p = synth.ring_problem(16, 900, seed=41)
    c = cfg(robust_kernel=RobustKernel.cauchy(2.0))
    a, b = p.copy(), with_weights(p, np.ones(p.num_observations))
    st_a, ra = oracle.optimize(a, c)
    st_b, rb = oracle.optimize(b, c)
    assert st_a == st_b == 0
    assert ra.final_cost == rb.final_cost
    assert np.array_equal(a.pose_q, b.pose_q) and np.array_equal(a.landmarks, b.landmarks)


def test_oracle_zero_weight_removes_the_observation():
    p = synth.ring_problem(16, 900, seed=42)
    drop = droppable(p, 60, seed=1)
    w = np.where(drop, 0.0, 1.0)
    c = cfg()
    a, b = with_weights(p, w), without(p, drop)
    assert oracle.cost(a, c)[0] == pytest.approx(oracle.cost(b, c)[0], rel=1e-12)
    st_a, ra = oracle.optimize(a, c)
    st_b, rb = oracle.optimize(b, c)
    assert st_a == st_b == 0
    assert ra.final_cost == pytest.approx(rb.final_cost, rel=1e-10)
    assert np.abs(a.camera_centers() - b.camera_centers()).max() <= 1e-9 * synth.scene_extent(b)


def test_oracle_weights_scale_the_cost():
    p = synth.ring_problem(10, 400, seed=5)
    rng = np.random.default_rng(0)
    w = rng.uniform(0.0, 3.0, p.num_observations)
    for k in (RobustKernel.none(), RobustKernel.huber(1.0), RobustKernel.cauchy(2.0)):
        c = BaConfig(robust_kernel=k)
        total, _ = oracle.cost(with_weights(p, w), c)
        # Per-observation costs from single-observation weight vectors.
        parts = 0.0
        for o in range(0, p.num_observations, 97):
            e = np.zeros(p.num_observations)
            e[o] = 1.0
            parts += w[o] * oracle.cost(with_weights(p, e), c)[0]
        sub = np.zeros(p.num_observations)
        sub[::97] = w[::97]
        assert oracle.cost(with_weights(p, sub), c)[0] == pytest.approx(parts, rel=1e-12)
        assert total > 0.0


# ------------------------------------------------------------------ GPU side
@pytest.mark.gpu
@pytest.mark.parametrize("maker,kernel", [
    (lambda: synth.ring_problem(20, 1500, seed=21), RobustKernel.huber(1.0)),
    (lambda: synth.stereo_window(15, 900, seed=11), RobustKernel.cauchy(2.0)),
    (lambda: synth.pose_only(500, seed=6), RobustKernel.none()),
])
def test_weighted_solve_matches_the_oracle(solver, maker, kernel):
    p = maker()
    rng = np.random.default_rng(7)
    w = rng.uniform(0.2, 2.0, p.num_observations)
    w[rng.random(p.num_observations) < 0.05] = 0.0
    c = cfg(robust_kernel=kernel)
    gpu, ref = with_weights(p, w), with_weights(p, w)
    cost, bad = solver.cost(gpu, c)
    cost_ref, bad_ref = oracle.cost(ref, c)
    assert bad == bad_ref and cost == pytest.approx(cost_ref, rel=1e-12)
    st, res = solver.optimize(gpu, c)
    assert st == _abi.OK, solver.last_error()
    st_ref, res_ref = oracle.optimize(ref, c)
    assert st_ref == _abi.OK
    assert abs(res.final_cost - res_ref.final_cost) <= COST_RTOL * abs(res_ref.final_cost)
    extent = synth.scene_extent(ref)
    assert np.abs(gpu.camera_centers() - ref.camera_centers()).max() <= CENTER_TOL * extent


@pytest.mark.gpu
def test_unit_weights_are_bit_identical_on_the_device(solver):
    p = synth.ring_problem(20, 1500, seed=22)
    c = cfg()
    a, b = p.copy(), with_weights(p, np.ones(p.num_observations))
    st, ra = solver.optimize(a, c)
    assert st == _abi.OK
    st, rb = solver.optimize(b, c)
    assert st == _abi.OK
    assert ra.final_cost == rb.final_cost
    assert np.array_equal(a.pose_q, b.pose_q) and np.array_equal(a.landmarks, b.landmarks)


@pytest.mark.gpu
def test_weighted_and_plain_problems_in_one_batch(solver):
    """A batch that mixes weighted and unweighted problems: each result is the
    one the problem gets alone."""
    rng = np.random.default_rng(3)
    probs = [synth.stereo_window(12, 800, seed=1), synth.ring_problem(16, 900, seed=41),
             synth.stereo_window(8, 500, seed=9)]
    probs[1] = with_weights(probs[1], rng.uniform(0.5, 1.5, probs[1].num_observations))
    c = cfg()
    alone = []
    for p in probs:
        q = p.copy()
        st, r = solver.optimize(q, c)
        assert st == _abi.OK
        alone.append((q, r))
    batch = [p.copy() for p in probs]
    statuses, results = solver.batch_optimize(batch, c)
    assert statuses == [_abi.OK] * 3
    for (q, ra), b, rb in zip(alone, batch, results):
        assert rb.final_cost == ra.final_cost
        assert np.array_equal(q.pose_q, b.pose_q) and np.array_equal(q.landmarks, b.landmarks)


@pytest.mark.gpu
def test_accelerator_weight_errors():
    acc = GpuBundleAdjuster(0, GpuBaSettings(100, 1e-6, True))
    ba = drifted_bundle()
    n = len(ba.observations)
    with pytest.raises(BaError) as e:
        acc.optimize_with_observation_weights(ba, BaConfig(), np.ones(n + 1))
    assert e.value.kind == "ObservationWeightCount"
    w = np.ones(n)
    w[3] = -1.0
    with pytest.raises(BaError) as e:
        acc.optimize_with_observation_weights(ba, BaConfig(), w)
    assert e.value == BaError("InvalidObservationWeight", 3)
    res = acc.optimize_with_observation_weights(ba, BaConfig(), np.full(n, 2.0))
    assert res.final_cost < res.initial_cost
