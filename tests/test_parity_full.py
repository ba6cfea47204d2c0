"""The benchmarked workloads against the FP64 oracle, at full size and at the
benchmarked PCG settings (tolerance 1e-6, at most 200 iterations per LM
iteration), not the tight settings of the small parity cases.

The oracle's solves of these inputs take minutes of CPU, so they are
committed as fixtures (tests/golden/*_oracle.npz, made by
tests/golden/make_parity_fixtures.py); each fixture's input digest is
checked first, so a change of the seeded generator fails here instead of
being compared against a stale answer.  Tolerance: the north-star's final
cost within 1e-5 relative and camera centres within 1e-5 of the scene extent.
"""

from __future__ import annotations

import pytest

from oracle import parity
from visloc_ba import _abi, synth

TOL = parity.TOLERANCE


def test_ring4m_fixture_is_present_and_matches_the_generator():
    """The fixture exists and the seeded generator still makes its input."""
    fx = parity.load("ring4m")
    assert fx is not None
    p = synth.large_ring_problem(seed=2000)
    assert parity.input_digest(p) == str(fx["digest"])
    assert fx["centers"].shape == (p.num_poses, 3)


@pytest.mark.gpu
def test_ring4m_matches_the_oracle_at_the_benchmarked_settings(solver):
    """ring-4m (1,200 cameras, 500k points, 4.06M observations, Huber 1 px,
    30 LM iterations, PCG 1e-6 / 200): final cost and camera centres against
    the oracle's FP64 sparse solve of the same seeded input."""
    fx = parity.load("ring4m")
    p = synth.large_ring_problem(seed=2000)
    assert parity.input_digest(p) == str(fx["digest"])
    q = p.copy()
    st, res = solver.optimize(q, parity.ring4m_config())
    assert st == _abi.OK, solver.last_error()
    assert res.initial_cost == pytest.approx(float(fx["initial_cost"]), rel=1e-12)
    err = parity.ring4m_parity(p, res.final_cost, q.camera_centers())
    assert err is not None
    assert err["final_cost_rel"] <= TOL, err
    assert err["centre_err_of_extent"] <= TOL, err


def test_windows512_fixture_is_present_and_matches_the_generator():
    fx = parity.load("windows512_sample")
    assert fx is not None
    probs = synth.window_batch(512, seed=4000)
    for i, d in zip(fx["windows"], fx["digests"]):
        assert parity.input_digest(probs[i]) == str(d)


@pytest.mark.gpu
def test_windows512_sample_matches_the_oracle_at_the_benchmarked_settings(solver):
    """32 windows of the windows-512 batch (every 16th), solved as one batch
    with the bench's settings (10 LM iterations, PCG 1e-6 / 200, CUDA graph),
    each against the oracle's FP64 solve of that window alone."""
    fx = parity.load("windows512_sample")
    assert fx is not None
    probs = synth.window_batch(512, seed=4000)
    sample = [probs[i] for i in fx["windows"]]
    for p, d in zip(sample, fx["digests"]):
        assert parity.input_digest(p) == str(d)
    cfg = parity.windows_config()
    cfg.graph = True
    batch = [p.copy() for p in sample]
    statuses, results = solver.batch_optimize(batch, cfg)
    assert statuses == [_abi.OK] * len(batch)
    rows = fx["center_rows"]
    worst_cost, worst_centre = 0.0, 0.0
    for k, (q, r) in enumerate(zip(batch, results)):
        e = parity.compare_state(r.final_cost, q.camera_centers(), float(fx["final_cost"][k]),
                                 fx["centers"][rows[k]:rows[k + 1]], float(fx["extent"][k]))
        worst_cost = max(worst_cost, e["final_cost_rel"])
        worst_centre = max(worst_centre, e["centre_err_of_extent"])
    assert worst_cost <= TOL, worst_cost
    assert worst_centre <= TOL, worst_centre
