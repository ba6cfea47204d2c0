"""Batched solves (visloc_ba_cuda_batch_*): many problems in one device
layout, every launch covering all of them.

Each problem keeps its own LM state and every sum is per problem in a fixed
order, so a problem's result is bit-for-bit the same solved alone or in any
batch; the CUDA-graph form of the LM loop runs the same kernels and gives the
same bits."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from visloc_ba import BaConfig, PackedProblem, RobustKernel, synth
from visloc_ba import _abi

pytestmark = pytest.mark.gpu


def mixed_problems():
    ring = synth.ring_problem(16, 900, seed=41)
    shared = synth.ring_problem(30, 2500, seed=42, width=2000, height=1500, focal=(1500, 1500),
                                k1=(0.0, 0.0), per_camera_intrinsics=False,
                                track=("geometric", 8.0, 2, 30))
    landmark_only = synth.ring_problem(10, 500, seed=8)
    landmark_only.pose_fixed[:] = 1
    return [
        synth.stereo_window(12, 800, seed=1),
        ring,
        synth.pose_only(600, seed=4),
        synth.stereo_window(33, 2000, seed=2),
        shared,
        landmark_only,
        synth.stereo_window(5, 300, seed=3),
    ]


def cfg(**kw):
    base = dict(max_iterations=10, robust_kernel=RobustKernel.huber(1.0),
                max_pcg_iterations=200, pcg_relative_tolerance=1e-6)
    base.update(kw)
    return BaConfig(**base)


def same_state(a: PackedProblem, b: PackedProblem) -> bool:
    return (np.array_equal(a.pose_q, b.pose_q) and np.array_equal(a.pose_t, b.pose_t)
            and np.array_equal(a.landmarks, b.landmarks))


def test_each_result_is_the_same_alone_and_in_the_batch(solver):
    probs = mixed_problems()
    c = cfg()
    alone = []
    for p in probs:
        q = p.copy()
        st, res = solver.optimize(q, c)
        assert st == _abi.OK, solver.last_error()
        alone.append((q, res))
    batch = [p.copy() for p in probs]
    statuses, results = solver.batch_optimize(batch, c)
    assert statuses == [_abi.OK] * len(probs)
    for (q, ra), b, rb in zip(alone, batch, results):
        assert rb.final_cost == ra.final_cost
        assert rb.initial_cost == ra.initial_cost
        assert [i.step_accepted for i in rb.iterations] == [i.step_accepted for i in ra.iterations]
        assert [i.pcg_iterations for i in rb.iterations] == [i.pcg_iterations for i in ra.iterations]
        assert same_state(q, b)


def test_batch_order_does_not_change_results(solver):
    probs = mixed_problems()
    c = cfg()
    fwd = [p.copy() for p in probs]
    rev = [p.copy() for p in reversed(probs)]
    _, r1 = solver.batch_optimize(fwd, c)
    _, r2 = solver.batch_optimize(rev, c)
    for a, b, ra, rb in zip(fwd, reversed(rev), r1, reversed(r2)):
        assert ra.final_cost == rb.final_cost
        assert same_state(a, b)


def test_per_problem_configs_and_matching_the_oracle(solver):
    probs = [synth.stereo_window(15, 900, seed=11), synth.ring_problem(20, 1500, seed=21),
             synth.pose_only(400, seed=5)]
    cfgs = [cfg(robust_kernel=RobustKernel.cauchy(2.0), pcg_relative_tolerance=1e-8,
                max_pcg_iterations=300),
            cfg(max_iterations=6, pcg_relative_tolerance=1e-8, max_pcg_iterations=300),
            cfg(robust_kernel=RobustKernel.none(), max_iterations=4)]
    batch = [p.copy() for p in probs]
    statuses, results = solver.batch_optimize(batch, cfgs)
    assert statuses == [_abi.OK] * 3
    for p, b, c, r in zip(probs, batch, cfgs, results):
        assert len(r.iterations) <= c.max_iterations
        ref = p.copy()
        st, rr = oracle.optimize(ref, c)
        assert st == 0
        assert abs(r.final_cost - rr.final_cost) <= 1e-5 * abs(rr.final_cost)
        extent = synth.scene_extent(ref)
        assert np.abs(b.camera_centers() - ref.camera_centers()).max() <= 1e-5 * extent


def test_invalid_problems_are_left_out(solver):
    good = synth.stereo_window(10, 500, seed=7)
    bad = synth.ring_problem(6, 50, seed=3)
    bad = PackedProblem(bad.pose_q, bad.pose_t, bad.landmarks, bad.obs_pose,
                        np.where(np.arange(bad.num_observations) == 4, 10_000, bad.obs_landmark),
                        bad.obs_xy, bad.cameras, bad.pose_fixed, bad.landmark_fixed,
                        bad.obs_camera)
    alone = good.copy()
    _, ra = solver.optimize(alone, cfg())
    batch = [bad.copy(), good.copy()]
    statuses, results = solver.batch_optimize(batch, cfg())
    assert statuses == [_abi.ERR_MISSING_LANDMARK, _abi.OK]
    assert results[0] is None
    assert results[1].final_cost == ra.final_cost
    assert same_state(alone, batch[1])


def test_graph_replay_matches_the_host_driven_loop(solver):
    probs = mixed_problems()
    plain = [p.copy() for p in probs]
    _, r_plain = solver.batch_optimize(plain, cfg())
    graph_cfg = cfg(graph=True)
    solver.batch_upload([p.copy() for p in probs], graph_cfg)
    for _ in range(2):  # capture, then replay
        r_graph = solver.batch_solve_uploaded()
        for a, b in zip(r_plain, r_graph):
            assert a.final_cost == b.final_cost
            assert [i.lambda_ for i in a.iterations] == [i.lambda_ for i in b.iterations]
    out = [p.copy() for p in probs]
    solver.batch_download(out)
    for a, b in zip(plain, out):
        assert same_state(a, b)


def test_single_problem_graph_mode(solver):
    p = synth.ring_problem(20, 1500, seed=21)
    a, b = p.copy(), p.copy()
    st, ra = solver.optimize(a, cfg())
    assert st == 0
    st, rb = solver.optimize(b, cfg(graph=True))
    assert st == 0, solver.last_error()
    assert ra.final_cost == rb.final_cost
    assert same_state(a, b)
    assert rb.kernel_launches >= ra.kernel_launches  # finished iterations still launch


def test_launch_shapes_do_not_change_results(solver):
    """The autotuner's choices (PCG blocks, L2-resident share of S) leave
    every bit of the result as it is."""
    probs = mixed_problems()
    c = cfg()
    outs = []
    for blocks, l2 in ((0, 0.5), (3, 0.0), (17, 0.9)):
        solver.batch_upload([p.copy() for p in probs], c)
        solver.set_launch_shape(blocks, l2)
        res = solver.batch_solve_uploaded()
        out = [p.copy() for p in probs]
        solver.batch_download(out)
        outs.append((res, out))
    (r0, o0) = outs[0]
    for r, o in outs[1:]:
        for a, b, pa, pb in zip(r0, r, o0, o):
            assert a.final_cost == b.final_cost
            assert same_state(pa, pb)
    solver.batch_upload([p.copy() for p in probs], c)
    shape = solver.autotune()
    assert shape["pcg_blocks"] >= 1 and shape["pcg_iteration_us"] > 0.0
    res = solver.batch_solve_uploaded()
    for a, b in zip(r0, res):
        assert a.final_cost == b.final_cost


def test_observation_order_does_not_change_the_solve(solver):
    """Observations listed by landmark skip the plan's counting sort (its
    stable result is then the identity); listed in another order they go
    through it.  Both give the same point-major plan, so the solves agree
    bit for bit."""
    sorted_ring = synth.ring_problem(120, 40000, seed=46, width=2000, height=1500,
                                     focal=(1500, 1500), k1=(0.0, 0.0),
                                     per_camera_intrinsics=False,
                                     track=("geometric", 8.0, 2, 40))
    ol = np.asarray(sorted_ring.obs_landmark)
    assert np.all(np.diff(ol.astype(np.int64)) >= 0)
    assert sorted_ring.num_observations >= 200_000
    starts = np.flatnonzero(np.r_[True, ol[1:] != ol[:-1]])
    ends = np.r_[starts[1:], len(ol)]
    perm = np.concatenate([np.arange(a, b) for a, b in zip(starts[::-1], ends[::-1])])
    p = sorted_ring
    shuffled = PackedProblem(p.pose_q, p.pose_t, p.landmarks, p.obs_pose[perm], p.obs_landmark[perm],
                             p.obs_xy[perm], p.cameras, p.pose_fixed, p.landmark_fixed,
                             None if p.obs_camera is None else p.obs_camera[perm])
    c = cfg(max_iterations=5)
    a, b = sorted_ring.copy(), shuffled.copy()
    st, ra = solver.optimize(a, c)
    assert st == _abi.OK, solver.last_error()
    st, rb = solver.optimize(b, c)
    assert st == _abi.OK, solver.last_error()
    assert ra.final_cost == rb.final_cost
    assert [i.pcg_iterations for i in ra.iterations] == [i.pcg_iterations for i in rb.iterations]
    assert same_state(a, b)


def test_device_built_terms_equal_the_host_build(solver):
    """A problem of at least 200,000 observations solved alone has its Schur
    terms built on the device; in a batch, the host builds them.  Both lay
    each block's terms out in ascending point order, so the two solves are
    bit-identical -- on a ring (dense reduced system) and a street loop
    (banded, closed)."""
    big_ring = synth.ring_problem(120, 40000, seed=43, width=2000, height=1500,
                                  focal=(1500, 1500), k1=(0.0, 0.0), per_camera_intrinsics=False,
                                  track=("geometric", 8.0, 2, 40))
    street = synth.street_loop(400, 60000, seed=44, fixed=(0, 1, 200))
    small = synth.ring_problem(8, 300, seed=45)
    c = cfg(max_iterations=6)
    for big in (big_ring, street):
        assert big.num_observations >= 200_000
        q = big.copy()
        st, alone = solver.optimize(q, c)
        assert st == _abi.OK, solver.last_error()
        batch = [big.copy(), small.copy()]
        statuses, results = solver.batch_optimize(batch, c)
        assert statuses == [_abi.OK, _abi.OK]
        assert results[0].final_cost == alone.final_cost
        assert [i.pcg_iterations for i in results[0].iterations] == \
            [i.pcg_iterations for i in alone.iterations]
        assert same_state(batch[0], q)
