"""The serving loop (visloc_ba_cuda_server_*): tickets planned on host
threads, admitted into batches by worker slots on their own streams.

The test the serving contract asks for: every result is the same solved
alone and in the mix (bit for bit here, since each problem keeps its own
fixed-order sums in any batch)."""

from __future__ import annotations

import threading

import numpy as np
import pytest

from visloc_ba import BaConfig, PackedProblem, RobustKernel, synth
from visloc_ba import _abi
from visloc_ba.solver import BaServer

pytestmark = pytest.mark.gpu


def mix(seed=0, n=24):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = rng.random()
        if kind < 0.6:
            out.append(synth.stereo_window(int(rng.integers(10, 41)), int(rng.integers(1000, 5001)),
                                           seed=100 + i))
        elif kind < 0.9:
            out.append(synth.pose_only(int(rng.integers(100, 2001)), seed=200 + i))
        else:
            out.append(synth.ring_problem(60, 6000, seed=300 + i, width=1920, height=1080,
                                          focal=(1500, 1500), k1=(0.0, 0.0),
                                          per_camera_intrinsics=False,
                                          track=("geometric", 6.7, 2, 40)))
    return out


CFG = BaConfig(max_iterations=10, robust_kernel=RobustKernel.huber(1.0),
               max_pcg_iterations=200, pcg_relative_tolerance=1e-6)


def test_results_are_the_same_alone_and_in_the_mix(solver):
    probs = mix()
    alone = []
    for p in probs:
        q = p.copy()
        st, r = solver.optimize(q, CFG)
        assert st == _abi.OK, solver.last_error()
        alone.append((q, r))
    served = [p.copy() for p in probs]
    with BaServer(0, slots=3, memory_bytes=4 << 30, max_batch=8) as srv:
        # Submitted from two threads at once, so batches mix them.
        tickets = [None] * len(served)

        def submit(idx):
            for i in idx:
                tickets[i] = srv.submit(served[i], CFG)

        th = [threading.Thread(target=submit, args=(range(k, len(served), 2),)) for k in (0, 1)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        batches = set()
        for i, tk in enumerate(tickets):
            st, r, info = srv.wait(tk)
            assert st == _abi.OK, srv.last_error()
            batches.add(info["batch_size"])
            q, ra = alone[i]
            assert r.final_cost == ra.final_cost
            assert [x.lambda_ for x in r.iterations] == [x.lambda_ for x in ra.iterations]
            assert np.array_equal(served[i].pose_q, q.pose_q)
            assert np.array_equal(served[i].landmarks, q.landmarks)
            assert info["latency_ms"] >= info["solve_ms"] >= 0.0
    assert max(batches) > 1  # requests were batched together


def test_invalid_and_oversized_requests_complete_with_their_status():
    good = synth.pose_only(300, seed=1)
    bad = synth.ring_problem(6, 50, seed=3)
    bad = PackedProblem(bad.pose_q, bad.pose_t, bad.landmarks,
                        np.where(np.arange(bad.num_observations) == 2, 99, bad.obs_pose),
                        bad.obs_landmark, bad.obs_xy, bad.cameras, bad.pose_fixed,
                        bad.landmark_fixed, bad.obs_camera)
    big = synth.ring_problem(40, 4000, seed=5)
    with BaServer(0, slots=2, memory_bytes=8 << 20) as srv:  # 4 MB per slot
        tg, tb, tbig = srv.submit(good, CFG), srv.submit(bad, CFG), srv.submit(big, CFG)
        assert srv.wait(tb)[0] == _abi.ERR_MISSING_POSE
        assert srv.wait(tbig)[0] == _abi.ERR_OUT_OF_MEMORY
        st, r, _ = srv.wait(tg)
        assert st == _abi.OK and r.final_cost < r.initial_cost


def test_close_finishes_the_submitted_tickets():
    probs = [synth.pose_only(500, seed=k) for k in range(6)]
    before = [p.pose_q.copy() for p in probs]
    srv = BaServer(0, slots=2, memory_bytes=1 << 30)
    for p in probs:
        srv.submit(p, CFG)
    srv.close()  # returns once every ticket has been solved and written back
    for p, q0 in zip(probs, before):
        assert not np.array_equal(p.pose_q, q0)


def test_wait_with_a_timeout():
    srv = BaServer(0, slots=1, memory_bytes=1 << 30)
    t = srv.submit(synth.stereo_window(30, 4000, seed=9), CFG)
    st, _, _ = srv.wait(t, timeout_ms=0.0)
    assert st in (_abi.ERR_BUSY, _abi.OK)
    if st == _abi.ERR_BUSY:
        st, r, info = srv.wait(t, timeout_ms=60_000.0)
        assert st == _abi.OK and info["batch_size"] == 1
    srv.close()
