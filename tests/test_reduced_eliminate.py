"""ReducedSolveAccelerator::eliminate (pipelines/slam/src/ba_accel.rs:74-144):
the off-diagonal blocks of the reduced camera system formed from camera-point
blocks and point inverses, the run blocks and coarse sums returned, and the
blocks kept on the device for the next solve with no off-diagonal blocks.

CPU: the oracle's pairwise FP64 restatement against the dense Schur
complement W V^-1 W^T of the same blocks, and its coarse sums against the
coarse level built from the full blocks (coarse_from_sums against
coarse_correction).  GPU: the device against the oracle on random
eliminations shaped like the reference's own tests (random_elimination,
crates/ba-gpu/src/reduced.rs:1271-1372: points of 2-12 nodes in a window of
16, every 37th point left out, a coupling on every 97th edge), the error of
each entry relative to its Cauchy-Schwarz bound, and the solve on resident
blocks against the solve on uploaded ones (:1453-1538)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from visloc_ba import _abi
from visloc_ba.solver import SolverError


def random_elimination(n, n_points, seed):
    """(edges, point_off, point_nodes, hcp, inverses, extra): each point
    observed by 2-12 distinct nodes within 16 of a random start, blocks
    30 U(-1, 1), V = I + sum hcp^T hcp, every 37th point (p % 37 == 5) left
    out, a random coupling on every 97th edge."""
    rng = np.random.default_rng(seed)
    point_off, point_nodes, hcp, inverses = [0], [], [], []
    for p in range(n_points):
        length = 2 + int(rng.random() * 11)
        start = min(int(rng.random() * n), n - 2)
        nodes = sorted({min(start + int(rng.random() * 16), n - 1) for _ in range(length)})
        if len(nodes) < 2:
            nodes = [start, start + 1]
        blocks = rng.uniform(-1.0, 1.0, (len(nodes), 6, 3)) * 30.0
        v = np.eye(3) + sum(b.T @ b for b in blocks)
        inverses.append(np.linalg.inv(v) if p % 37 != 5 else None)
        point_nodes += nodes
        hcp.append(blocks)
        point_off.append(len(point_nodes))
    edges = sorted({(point_nodes[k], point_nodes[j])
                    for p in range(n_points)
                    for k in range(point_off[p], point_off[p + 1])
                    for j in range(k + 1, point_off[p + 1])})
    edges = np.array(edges, np.uint32)
    extra = [(e, rng.uniform(-1.0, 1.0, (6, 6))) for e in range(0, len(edges), 97)]
    return (edges, np.array(point_off, np.uint64), np.array(point_nodes, np.uint32),
            np.concatenate(hcp), inverses, extra)


def bounds(n, point_off, point_nodes, hcp, inverses):
    """Per node, sqrt of the diagonal of sum hcp V^-1 hcp^T over its points
    (PointElimination::scale): |block(t, s)[r][c]| <= scale[t][r] scale[s][c]."""
    d = np.zeros((n, 6))
    for p in range(len(point_off) - 1):
        if inverses[p] is None:
            continue
        for o in range(int(point_off[p]), int(point_off[p + 1])):
            d[point_nodes[o]] += np.einsum("ri,ij,rj->r", hcp[o], inverses[p], hcp[o])
    return np.sqrt(np.maximum(d, 0.0))


# ------------------------------------------------------------------ CPU side
def test_oracle_blocks_are_the_dense_schur_complement():
    n = 40
    edges, point_off, point_nodes, hcp, inv, extra = random_elimination(n, 300, 3)
    blocks = oracle.eliminate_blocks(edges, point_off, point_nodes, hcp, inv, extra)
    W = np.zeros((6 * n, 3 * len(inv)))
    Vinv = np.zeros((3 * len(inv), 3 * len(inv)))
    for p in range(len(inv)):
        if inv[p] is None:
            continue
        Vinv[3 * p:3 * p + 3, 3 * p:3 * p + 3] = inv[p]
        for o in range(int(point_off[p]), int(point_off[p + 1])):
            s = int(point_nodes[o])
            W[6 * s:6 * s + 6, 3 * p:3 * p + 3] = hcp[o]
    S = -W @ Vinv @ W.T
    for (e, m) in extra:
        a, b = edges[e]
        S[6 * b:6 * b + 6, 6 * a:6 * a + 6] += m
    for e, (a, b) in enumerate(edges):
        np.testing.assert_allclose(blocks[e], S[6 * b:6 * b + 6, 6 * a:6 * a + 6],
                                   rtol=1e-12, atol=1e-9)


def test_oracle_coarse_sums_rebuild_the_coarse_level():
    n = 60
    edges, point_off, point_nodes, hcp, inv, extra = random_elimination(n, 500, 4)
    blocks = oracle.eliminate_blocks(edges, point_off, point_nodes, hcp, inv, extra)
    rowsum = np.zeros(n)
    for (a, b), m in zip(edges, blocks):
        rowsum[a] += np.abs(m).sum()
        rowsum[b] += np.abs(m).sum()
    diag = [np.eye(6) * (rowsum[i] + 1.0) for i in range(n)]
    group, nodes = 7, 55
    want = oracle.coarse_correction(diag, edges, blocks, nodes, group)
    got = oracle.coarse_from_sums(diag, oracle.coarse_block_sums(edges, blocks, group, nodes),
                                  nodes, group)
    assert want[0] == got[0] == group and want[1] == got[1] == nodes
    np.testing.assert_allclose(got[2], want[2], rtol=1e-10, atol=1e-14)


# ------------------------------------------------------------------ GPU side
def run_edges_of(edges, k):
    return np.array([e for e, (a, b) in enumerate(edges) if a // k == b // k], np.uint32)


@pytest.mark.gpu
def test_gpu_elimination_matches_the_f64_sums(solver):
    n = 150
    edges, point_off, point_nodes, hcp, inv, extra = random_elimination(n, 4000, 11)
    want = oracle.eliminate_blocks(edges, point_off, point_nodes, hcp, inv, extra)
    k, group = 8, 10
    runs = run_edges_of(edges, k)
    run_blocks, sums = solver.reduced_eliminate(1, 1, n, edges, point_off, point_nodes, hcp, inv,
                                                extra, runs, (group, n))
    scale = bounds(n, point_off, point_nodes, hcp, inv)
    b = scale[edges[runs, 1]][:, :, None] * scale[edges[runs, 0]][:, None, :] + 1.0
    worst = np.max(np.abs(run_blocks - want[runs]) / b)
    assert worst < 1e-6, worst
    m = -(-n // group)
    want_sums = oracle.coarse_block_sums(edges, want, group, n)
    assert sums.shape == (m * m, 6, 6)
    err = np.abs(sums - want_sums).max(axis=(1, 2))
    assert np.all(err <= 1e-5 * (1.0 + np.abs(want_sums).max(axis=(1, 2)))), err.max()
    # The same elimination again: the same blocks, bit for bit.
    again, sums2 = solver.reduced_eliminate(1, 1, n, edges, point_off, point_nodes, hcp, inv,
                                            extra, runs, (group, n))
    assert np.array_equal(again, run_blocks) and np.array_equal(sums2, sums)


@pytest.mark.gpu
def test_gpu_linearization_and_structure_changes(solver):
    n = 80
    edges, point_off, point_nodes, hcp, inv, extra = random_elimination(n, 1500, 12)
    allruns = np.arange(len(edges), dtype=np.uint32)
    solver.reduced_eliminate(5, 1, n, edges, point_off, point_nodes, hcp, inv, extra, allruns)
    # A new linearization under the same structure id: hcp is uploaded again.
    hcp2 = hcp * 0.5
    got, _ = solver.reduced_eliminate(5, 2, n, edges, point_off, point_nodes, hcp2, inv, extra,
                                      allruns)
    want = oracle.eliminate_blocks(edges, point_off, point_nodes, hcp2, inv, extra)
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    # Another structure.
    e2, o2, nd2, h2, i2, x2 = random_elimination(n, 900, 13)
    got, _ = solver.reduced_eliminate(6, 1, n, e2, o2, nd2, h2, i2, x2,
                                      np.arange(len(e2), dtype=np.uint32))
    want = oracle.eliminate_blocks(e2, o2, nd2, h2, i2, x2)
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


@pytest.mark.gpu
def test_gpu_resident_blocks_solve_like_uploaded_ones(solver):
    n = 120
    edges, point_off, point_nodes, hcp, inv, extra = random_elimination(n, 3000, 5)
    blocks = oracle.eliminate_blocks(edges, point_off, point_nodes, hcp, inv, extra)
    row = np.zeros(n)
    for (a, b), m in zip(edges, blocks):
        row[a] += np.abs(m).max()
        row[b] += np.abs(m).max()
    diag = np.array([np.eye(6) * (6.0 * row[i] + 1.0) for i in range(n)])
    rhs = np.array([[((i * 6 + r) % 7) - 3.0 for r in range(6)] for i in range(n)])
    up, it_up, _ = solver.reduced_solve(diag, edges, blocks, rhs, 1e-6, 500)
    # Without an elimination of these edges there are no resident blocks.
    with pytest.raises(SolverError) as e:
        solver.reduced_solve(diag, edges, None, rhs, 1e-6, 500)
    assert e.value.status == _abi.DECLINED
    solver.reduced_eliminate(7, 3, n, edges, point_off, point_nodes, hcp, inv, extra)
    res, it_res, _ = solver.reduced_solve(diag, edges, None, rhs, 1e-6, 500)
    size = np.linalg.norm(up, axis=1).max()
    assert abs(it_up - it_res) <= 1
    assert np.linalg.norm(up - res, axis=1).max() <= 1e-4 * size
    # The preconditioned entry on resident blocks, with runs and a coarse
    # level built from what the elimination returned.
    k, group = 16, 12
    runs = run_edges_of(edges, k)
    run_blocks, sums = solver.reduced_eliminate(7, 3, n, edges, point_off, point_nodes, hcp, inv,
                                                extra, runs, (group, n))
    clusters = oracle.cluster_inverses(diag, edges[runs], run_blocks, k)
    coarse = oracle.coarse_from_sums(diag, sums, n, group)
    x, it, _ = solver.reduced_solve(diag, edges, None, rhs, 1e-6, 500, clusters=clusters,
                                    coarse=coarse)
    x_ref, it_ref = oracle.reduced_pcg(diag, edges, blocks, rhs, 1e-6, 500,
                                       oracle.cluster_inverses(diag, edges, blocks, k),
                                       oracle.coarse_correction(diag, edges, blocks, n, group))
    assert abs(it - it_ref) <= max(2, it_ref // 10)
    assert np.abs(x - x_ref).max() <= 1e-4 * np.abs(x_ref).max()


@pytest.mark.gpu
def test_gpu_rejects_malformed_eliminations(solver):
    n = 30
    edges, point_off, point_nodes, hcp, inv, extra = random_elimination(n, 200, 14)
    cases = [
        dict(edges=edges[::-1]),                                # not sorted
        dict(edges=edges[1:]),                                  # a pair of nodes with no edge
        dict(extra=[(len(edges), np.eye(6))]),                  # coupling names no edge
        dict(run_edges=[len(edges)]),                           # run edge names no edge
        dict(coarse=(4, n + 1)),                                # more nodes than the system
        dict(structure_id=0),                                   # no structure id
    ]
    for kw in cases:
        args = dict(structure_id=9, linearization_id=1, num_nodes=n, edges=edges,
                    point_off=point_off, point_nodes=point_nodes, hcp=hcp, point_inverse=inv,
                    extra=extra, run_edges=(), coarse=None)
        args.update(kw)
        with pytest.raises(SolverError) as e:
            solver.reduced_eliminate(**args)
        assert e.value.status == _abi.ERR_INVALID_ARGUMENT, kw


def test_synthetic_reduced_workload_generators():
    """The bench's reduced-camera inputs (visloc_ba.synth): the covisibility
    system has sorted distinct edges and a diagonally dominant SPD matrix; the
    street elimination's edges are exactly the node pairs its points share,
    and its damped diagonal with the eliminated blocks is SPD."""
    from visloc_ba import synth

    diag, edges, off = synth.covisibility_system(200, 20, 8)
    keys = edges[:, 0].astype(np.int64) * 200 + edges[:, 1]
    assert np.all(np.diff(keys) > 0) and np.all(edges[:, 0] < edges[:, 1])
    S = np.zeros((1200, 1200))
    for i, d in enumerate(diag):
        S[6 * i:6 * i + 6, 6 * i:6 * i + 6] = d
    for (a, b), B in zip(edges, off.astype(np.float64)):
        S[6 * b:6 * b + 6, 6 * a:6 * a + 6] = B
        S[6 * a:6 * a + 6, 6 * b:6 * b + 6] = B.T
    assert np.all(np.diag(S) > np.abs(S).sum(axis=1) - np.diag(S))
    el = synth.street_elimination(150, 60, seed=3)
    po, pn = el["point_off"], el["point_nodes"]
    want = sorted({(int(pn[k]), int(pn[j])) for p in range(len(po) - 1)
                   for k in range(int(po[p]), int(po[p + 1]))
                   for j in range(k + 1, int(po[p + 1]))})
    assert [tuple(e) for e in el["edges"].tolist()] == want
    blocks = oracle.eliminate_blocks(el["edges"], po, pn, el["hcp"], list(el["point_inverse"]))
    S = np.zeros((900, 900))
    for i, d in enumerate(el["diag"]):
        S[6 * i:6 * i + 6, 6 * i:6 * i + 6] = d
    for (a, b), B in zip(el["edges"], blocks):
        S[6 * b:6 * b + 6, 6 * a:6 * a + 6] = B
        S[6 * a:6 * a + 6, 6 * b:6 * b + 6] = B.T
    assert np.linalg.eigvalsh(S).min() > 0.0
    # The full-size system the bench measures: the published edge count.
    assert abs(len(synth.covisibility_system()[1]) - 3.4e6) < 0.05e6
