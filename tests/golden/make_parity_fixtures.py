"""Writes the full-size parity fixtures of tests/golden: the FP64 oracle's
solve of the benchmarked workloads, so that a GPU test and bench.py can state
the device solve's error against the reference solver's arithmetic on the
same seeded input without running the oracle for minutes on the GPU host.

Each fixture holds a digest of the generated input (so a change of the
generator is caught instead of compared against a stale answer), the initial
and final cost, the per-iteration trace (cost after each trial, accepted,
lambda) and the camera centres of the final state (f64).

    python tests/golden/make_parity_fixtures.py [ring-4m] [windows-512-sample] [street-20m]

ring-4m: 1,200 cameras, 500k points, 4.06M observations, Huber 1 px, 30 LM
iterations, the oracle's sparse Schur + block Cholesky solve (SPARSE) on all
host threads (about 5 minutes on 8 threads).  windows-512-sample: 32 windows
of the windows-512 batch (every 16th), 10 LM iterations each, dense solve.
street-20m: 5,600 cameras, ~19.7M observations, 15 LM iterations, the sparse
solve in band storage (about 3 minutes on 8 threads).
The expected values come from the oracle (this repository's FP64
restatement of the reference solver), not from the Rust reference, which
cannot run here.
"""

from __future__ import annotations

import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "visloc-rs_b200")]

import numpy as np  # noqa: E402

from oracle.parity import (WINDOW_SAMPLE, fixture_path, input_digest,  # noqa: E402
                           ring4m_config, street20m_config, windows_config)
from visloc_ba import synth  # noqa: E402


def trace_arrays(res):
    its = res.iterations
    return dict(cost_after=np.array([s.cost_after for s in its]),
                accepted=np.array([bool(s.step_accepted) for s in its]),
                lam=np.array([s.lambda_ for s in its]))


def make_ring4m():
    from oracle import oracle

    p = synth.large_ring_problem(seed=2000)
    digest = input_digest(p)
    q = p.copy()
    t0 = time.time()
    st, res = oracle.optimize(q, ring4m_config(), solver=oracle.SPARSE)
    assert st == 0, st
    print(f"ring-4m: oracle {time.time() - t0:.0f} s, cost {res.initial_cost:.10e} -> "
          f"{res.final_cost:.10e}, {len(res.iterations)} iterations")
    np.savez_compressed(fixture_path("ring4m"), digest=digest,
                        initial_cost=res.initial_cost, final_cost=res.final_cost,
                        extent=synth.scene_extent(q), centers=q.camera_centers(),
                        **trace_arrays(res))


def make_street20m():
    """street-20m: 5,600 cameras on a closed street loop, ~2.9M facade points,
    ~19.7M observations, Huber 1 px, 15 LM iterations; the oracle's Sparse
    solve in band storage (the loop's reduced system is a cyclic band), all
    host threads (about 10 s per LM iteration on 8 threads)."""
    from oracle import oracle

    p = synth.street_loop(seed=3000)
    digest = input_digest(p)
    q = p.copy()
    t0 = time.time()
    st, res = oracle.optimize(q, street20m_config(), solver=oracle.SPARSE_BANDED)
    assert st == 0, st
    print(f"street-20m: oracle {time.time() - t0:.0f} s, cost {res.initial_cost:.10e} -> "
          f"{res.final_cost:.10e}, {len(res.iterations)} iterations")
    np.savez_compressed(fixture_path("street20m"), digest=digest,
                        initial_cost=res.initial_cost, final_cost=res.final_cost,
                        extent=synth.scene_extent(q), centers=q.camera_centers(),
                        **trace_arrays(res))


def make_windows_sample():
    from oracle import oracle

    probs = synth.window_batch(512, seed=4000)
    out = {}
    finals, initials, centers, digests, extents = [], [], [], [], []
    for i in WINDOW_SAMPLE:
        p = probs[i]
        digests.append(input_digest(p))
        q = p.copy()
        st, res = oracle.optimize(q, windows_config())
        assert st == 0, (i, st)
        finals.append(res.final_cost)
        initials.append(res.initial_cost)
        centers.append(q.camera_centers())
        extents.append(synth.scene_extent(q))
    out["windows"] = np.array(WINDOW_SAMPLE)
    out["digests"] = np.array(digests)
    out["initial_cost"] = np.array(initials)
    out["final_cost"] = np.array(finals)
    out["extent"] = np.array(extents)
    out["centers"] = np.concatenate(centers)
    out["center_rows"] = np.cumsum([0] + [c.shape[0] for c in centers])
    np.savez_compressed(fixture_path("windows512_sample"), **out)
    print(f"windows-512 sample: {len(WINDOW_SAMPLE)} windows")


if __name__ == "__main__":
    which = sys.argv[1:] or ["ring-4m", "windows-512-sample", "street-20m"]
    if "windows-512-sample" in which:
        make_windows_sample()
    if "ring-4m" in which:
        make_ring4m()
    if "street-20m" in which:
        make_street20m()
