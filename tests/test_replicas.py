"""The multi-GPU form of the bench is replicas only: every rank solves its
own problem and the process group carries the barrier and the max/sum of the
timings.  This runs that host logic on two CPU ranks over gloo, each rank
solving a different problem with the FP64 oracle."""

from __future__ import annotations

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "visloc-rs_b200")]
    import time

    import bench
    from oracle import oracle
    from visloc_ba import BaConfig, RobustKernel, synth

    dist = bench.Dist(backend="gloo")
    p = synth.ring_problem(8, 200, seed=70 + rank)  # each replica its own problem
    cfg = BaConfig(max_iterations=3 + rank, robust_kernel=RobustKernel.huber(1.0))
    dist.barrier()
    t0 = time.perf_counter()
    st, res = oracle.optimize(p, cfg, threads=1)
    dt = time.perf_counter() - t0 + 0.05 * rank  # ranks of different speed
    dist.barrier()
    rate, t_max = bench.replica_rate(dist, len(res.iterations), dt)
    out.put((rank, st, len(res.iterations), dt, rate, t_max))
    dist.close()


def test_two_replicas_aggregate_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    rows = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, st0, it0, dt0, rate0, tmax0), (_, st1, it1, dt1, rate1, tmax1) = rows
    assert st0 == 0 and st1 == 0
    assert tmax0 == tmax1 == pytest.approx(max(dt0, dt1))
    assert rate0 == rate1 == pytest.approx((it0 + it1) / max(dt0, dt1))


def test_reduced_reference_arm_runs_on_the_cpu():
    """bench.py's reduced-camera workload, reference arm (the oracle's FP64
    iteration, no GPU), at a small size: one JSON line with the contract's
    keys, and the tile count of the device layout for its edges."""
    import json
    import subprocess

    out = subprocess.run(
        [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
         "reduced-5822", "--reduced-nodes", "160"],
        capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "reduced_pcg_iteration_ms"
    assert line["value"] > 0 and line["higher_is_better"] is False
    assert line["config"]["nodes"] == 160 and line["config"]["workload"] == "reduced-160"
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0


def test_reduced_tiles_counts_the_device_layout():
    sys.path[:0] = [ROOT]
    import numpy as np

    import bench

    edges = np.array([(0, 1), (0, 9), (3, 20), (8, 9), (16, 17)], np.uint32)
    # Tile rows of 8 nodes: 3 rows for 21 nodes; diagonal tiles (0,0), (1,1), (2,2) plus the
    # off-diagonal tiles (0,1) and (0,2).
    assert bench.reduced_tiles(edges, 21) == 5


def test_compact_keeps_the_named_keys():
    """The default line's other_workloads entries keep only the named keys of
    each workload's own line."""
    import bench

    line = {"value": 1.0, "unit": "u", "clocks": {}, "noise": [1, 2]}
    assert bench.compact(line, ["value", "unit", "clocks", "missing"]) == {
        "value": 1.0, "unit": "u", "clocks": {}}
    assert bench.compact(None, ["value"]) is None


def test_pcg_traffic_comes_only_from_the_workloads_own_capture():
    """The roofline's DRAM traffic is read from the committed ncu summary of
    the same workload; a workload without a capture of its own reports none."""
    sys.path[:0] = [ROOT]
    import bench

    ring = bench.traffic_per_pcg_iteration("ring-4m")
    assert ring is not None and 1e7 < ring < 1.1e8  # below B_pcg = 106.5 MB: S partly in L2
    for name in ("street-20m", "windows-512", "ring-50"):
        assert bench.traffic_per_pcg_iteration(name) is None
