"""Cluster and coarse-level preconditioners of the reduced solve
(ReducedCameraSystem::clusters / ::coarse, pipelines/slam/src/ba_accel.rs:
64-69; built by cluster_inverses and coarse_correction and applied by
pcg_core, pipelines/slam/src/colmap_incremental/rig_ba_solver.rs:1112-1140,
1235-1266 and 1406-1480).

CPU: the oracle's FP64 restatement on the two systems of the reference's own
tests (dense_covisibility_system and chain_system, rig_ba_solver.rs:
5158-5196 and 5244-5272), pinned to what those tests assert: both solves
reach the Cholesky solution, runs beat block-Jacobi, and the coarse level
takes the chain from 58 to 33 iterations (the counts the reference's test
records).  GPU: visloc_ba_cuda_reduced_solve_preconditioned against the
oracle on the same systems and on reduced systems of synthetic scenes."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from visloc_ba import BaConfig, RobustKernel, synth
from visloc_ba import _abi
from visloc_ba.solver import SolverError


def covisibility_system(n):
    """A city block revisited in four passes: every node couples to its
    +-150 capture-order neighbours (weight 1) and to 100 nodes of the other
    passes at the same place (weight 0.5, written last and so kept where
    both apply); block entries ((7 r + 3 c + lo + hi) mod 11) 1e-3 w,
    diagonal 10 I + (i mod 5) I.  Diagonally dominant SPD."""
    cols = [dict() for _ in range(n)]
    rr, cc = np.meshgrid(np.arange(6), np.arange(6), indexing="ij")

    def add(a, b, w):
        lo, hi = min(a, b), max(a, b)
        if lo != hi:
            cols[lo][hi] = ((rr * 7 + cc * 3 + lo + hi) % 11) * 1e-3 * w

    q = n // 4
    for i in range(n):
        for d in range(1, 151):
            if i + d < n:
                add(i, i + d, 1.0)
        for k in range(100):
            add(i, ((i // q + 1 + k % 3) % 4) * q + (i % q + k // 3) % q, 0.5)
    diag = [np.eye(6) * (10.0 + i % 5) for i in range(n)]
    edges = [(j, i) for j in range(n) for i in sorted(cols[j])]
    off = [cols[j][i] for j, i in edges]
    return diag, np.array(edges, np.uint32), np.array(off)


def chain_system(n):
    """A long open capture: each node coupled to its 8 successors by -w I,
    w = 1 + ((7 a + 3 b) mod 5) / 10, as a graph Laplacian plus diagonal
    damping 1e-4 (1 + (i + r) mod 3); its smooth modes have tiny eigenvalues."""
    diag = [np.diag([1e-4 * (1 + (i + r) % 3) for r in range(6)]) for i in range(n)]
    edges, off = [], []
    for a in range(n):
        for b in range(a + 1, min(a + 9, n)):
            w = 1.0 + ((a * 7 + b * 3) % 5) * 0.1
            diag[a] = diag[a] + w * np.eye(6)
            diag[b] = diag[b] + w * np.eye(6)
            edges.append((a, b))
            off.append(-w * np.eye(6))
    return diag, np.array(edges, np.uint32), np.array(off)


def dense(diag, edges, off):
    n = len(diag)
    S = np.zeros((6 * n, 6 * n))
    for i, d in enumerate(diag):
        S[6 * i:6 * i + 6, 6 * i:6 * i + 6] = d
    for (a, b), B in zip(edges, off):
        S[6 * b:6 * b + 6, 6 * a:6 * a + 6] = B
        S[6 * a:6 * a + 6, 6 * b:6 * b + 6] = np.asarray(B).T
    return S


def pattern_rhs(n):
    """The right-hand side of the reference's tests: (13 i mod 17) - 8."""
    return np.array([((i * 13) % 17) - 8.0 for i in range(6 * n)])


def scene_system(maker, lam):
    """A synthetic scene's damped reduced camera system in block layout."""
    st, S, rhs, _, _ = oracle.reduced_system(maker(), lam, BaConfig(robust_kernel=RobustKernel.huber(1.0)),
                                             step=False)
    assert st == 0
    n = S.shape[0] // 6
    B = S.reshape(n, 6, n, 6).transpose(0, 2, 1, 3)
    diag = [B[i, i] for i in range(n)]
    edges = [(a, b) for a in range(n) for b in range(a + 1, n) if np.any(B[b, a] != 0.0)]
    off = [B[b, a] for a, b in edges]
    return diag, np.array(edges, np.uint32).reshape(-1, 2), np.array(off).reshape(-1, 6, 6), rhs, S


# ------------------------------------------------------------------ CPU side
def test_oracle_runs_beat_block_jacobi():
    n = 120
    diag, edges, off = covisibility_system(n)
    b = pattern_rhs(n)
    exact = np.linalg.solve(dense(diag, edges, off), b)
    xj, itj = oracle.reduced_pcg(diag, edges, off, b, 1e-10, 500)
    runs = oracle.cluster_inverses(diag, edges, off, 16)
    assert [s for s, _ in runs] == list(range(0, n, 16)) and runs[-1][1].shape == (48, 48)
    xc, itc = oracle.reduced_pcg(diag, edges, off, b, 1e-10, 500, clusters=runs)
    scale = np.linalg.norm(exact)
    assert np.linalg.norm(xj.reshape(-1) - exact) < 1e-6 * scale
    assert np.linalg.norm(xc.reshape(-1) - exact) < 1e-6 * scale
    assert itc < itj


def test_oracle_coarse_level_pinned_to_the_reference_counts():
    n = 600
    diag, edges, off = chain_system(n)
    b = pattern_rhs(n)
    exact = np.linalg.solve(dense(diag, edges, off), b)
    runs = oracle.cluster_inverses(diag, edges, off, 32)
    coarse = oracle.coarse_correction(diag, edges, off, n, 32)
    assert coarse[0] == 32 and coarse[2].shape == (6 * 19, 6 * 19)
    one, it_one = oracle.reduced_pcg(diag, edges, off, b, 1e-8, 500, clusters=runs)
    two, it_two = oracle.reduced_pcg(diag, edges, off, b, 1e-8, 500, clusters=runs, coarse=coarse)
    scale = np.linalg.norm(exact)
    assert np.linalg.norm(one.reshape(-1) - exact) < 1e-4 * scale
    assert np.linalg.norm(two.reshape(-1) - exact) < 1e-4 * scale
    assert (it_one, it_two) == (58, 33)


def test_oracle_coarse_group_grows_past_256_aggregates():
    diag, edges, off = chain_system(600)
    g, nodes, inv = oracle.coarse_correction(diag, edges, off, 600, 2)
    assert g == 3 and nodes == 600 and inv.shape == (6 * 200, 6 * 200)
    assert oracle.coarse_correction(diag, edges, off, 20, 32) is None  # one aggregate


def test_oracle_breakdown_and_zero_rhs():
    diag = [np.eye(6), np.eye(6)]
    edges = np.array([(0, 1)], np.uint32)
    off = np.array([2.0 * np.eye(6)])  # S has eigenvalue -1
    b = np.concatenate([np.ones(6), -np.ones(6)])
    assert oracle.reduced_pcg(diag, edges, off, b, 1e-8, 50) is None
    x, it = oracle.reduced_pcg(diag, edges, off, np.zeros(12), 1e-8, 50)
    assert it == 0 and not x.any()


# ------------------------------------------------------------------ GPU side
def check_against_oracle(solver, diag, edges, off, b, tol, runs=None, coarse=None, exact=None):
    x, it, rr = solver.reduced_solve(diag, edges, off, b.reshape(-1, 6), tol, 500,
                                     clusters=runs if runs is not None else [], coarse=coarse)
    x_ref, it_ref = oracle.reduced_pcg(diag, edges, off, b, tol, 500, clusters=runs, coarse=coarse)
    assert rr <= tol
    assert abs(it - it_ref) <= max(2, it_ref // 10), (it, it_ref)
    if exact is None:
        exact = np.linalg.solve(dense(diag, edges, off), b)
    err = np.abs(x.reshape(-1) - exact).max() / np.abs(exact).max()
    err_ref = np.abs(x_ref.reshape(-1) - exact).max() / np.abs(exact).max()
    return x, it, err, err_ref


@pytest.mark.gpu
def test_gpu_runs_on_the_covisibility_system(solver):
    n = 120
    diag, edges, off = covisibility_system(n)
    b = pattern_rhs(n)
    runs = oracle.cluster_inverses(diag, edges, off, 16)
    _, itj, err, _ = check_against_oracle(solver, diag, edges, off, b, 1e-6)
    _, itc, errc, _ = check_against_oracle(solver, diag, edges, off, b, 1e-6, runs=runs)
    assert err < 1e-5 and errc < 1e-5
    assert itc <= itj


@pytest.mark.gpu
def test_gpu_coarse_level_on_the_chain(solver):
    n = 600
    diag, edges, off = chain_system(n)
    b = pattern_rhs(n)
    runs = oracle.cluster_inverses(diag, edges, off, 32)
    coarse = oracle.coarse_correction(diag, edges, off, n, 32)
    exact = np.linalg.solve(dense(diag, edges, off), b)
    _, it_one, e1, r1 = check_against_oracle(solver, diag, edges, off, b, 1e-6, runs, exact=exact)
    _, it_two, e2, r2 = check_against_oracle(solver, diag, edges, off, b, 1e-6, runs, coarse,
                                             exact=exact)
    assert 3 * it_two < 2 * it_one, (it_one, it_two)
    # The chain's condition number is about 3e5 (damping 1e-4 against
    # couplings near 10), so S and the vectors in FP32 (eps 6e-8) leave an
    # error floor near 1e-3 of the solution's scale whatever the iteration;
    # the FP64 iteration stops well inside it.
    assert max(e1, e2) <= 2e-3 and max(r1, r2) <= 1e-5, (e1, r1, e2, r2)


@pytest.mark.gpu
@pytest.mark.parametrize("maker,lam,k,group", [
    (lambda: synth.street_loop(200, 8000, seed=82), 1e-1, 32, 32),
    (lambda: synth.ring_problem(70, 4000, seed=81), 1e-2, 8, 4),
])
def test_gpu_scene_systems(solver, maker, lam, k, group):
    diag, edges, off, b, S = scene_system(maker, lam)
    n = len(diag)
    runs = oracle.cluster_inverses(diag, edges, off, k)
    coarse = oracle.coarse_correction(diag, edges, off, n, group)
    assert runs is not None and coarse is not None
    exact = np.linalg.solve(S, b)
    x, it, err, _ = check_against_oracle(solver, diag, edges, off, b, 1e-6, runs, coarse,
                                         exact=exact)
    assert err <= 1e-3
    # Deterministic: the same system gives the same step.
    x2, it2, _ = solver.reduced_solve(diag, edges, off, b.reshape(-1, 6), 1e-6, 500,
                                      clusters=runs, coarse=coarse)
    assert it2 == it and np.array_equal(x, x2)


@pytest.mark.gpu
def test_gpu_partial_runs_and_coarse_prefix(solver):
    """Runs that cover part of the system (block-Jacobi elsewhere) and a
    coarse level over a prefix with a ragged last aggregate."""
    diag, edges, off, b, S = scene_system(lambda: synth.street_loop(120, 5000, seed=86), 1e-1)
    n = len(diag)
    full = oracle.cluster_inverses(diag, edges, off, 10)
    runs = [full[1], full[3], full[4], full[-1]]
    coarse = oracle.coarse_correction(diag, edges, off, n - 7, 9)
    assert coarse is not None and (n - 7) % 9 != 0
    x, it, err, _ = check_against_oracle(solver, diag, edges, off, b, 1e-6, runs, coarse,
                                         exact=np.linalg.solve(S, b))
    assert err <= 1e-3


@pytest.mark.gpu
def test_gpu_iteration_cap_zero_rhs_and_breakdown(solver):
    diag, edges, off = chain_system(200)
    b = pattern_rhs(200).reshape(-1, 6)
    runs = oracle.cluster_inverses(diag, edges, off, 32)
    _, it, rr = solver.reduced_solve(diag, edges, off, b, 1e-12, 5, clusters=runs)
    assert it == 5 and rr > 1e-12
    x, it, rr = solver.reduced_solve(diag, edges, off, 0.0 * b, 1e-8, 50, clusters=runs)
    assert it == 0 and rr == 0.0 and not x.any()
    # Indefinite S: pcg_core returns None, the C entry declines.
    bad = [np.eye(6), np.eye(6)]
    with pytest.raises(SolverError) as e:
        solver.reduced_solve(bad, np.array([(0, 1)]), np.array([2.0 * np.eye(6)]),
                             np.concatenate([np.ones(6), -np.ones(6)]).reshape(2, 6), 1e-8, 50,
                             clusters=[])
    assert e.value.status == _abi.DECLINED


@pytest.mark.gpu
def test_gpu_rejects_malformed_preconditioners(solver):
    diag, edges, off = chain_system(40)
    b = pattern_rhs(40).reshape(-1, 6)
    runs = oracle.cluster_inverses(diag, edges, off, 10)
    coarse = oracle.coarse_correction(diag, edges, off, 40, 10)
    for kw in (dict(clusters=[runs[1], runs[0]]),              # not ascending
               dict(clusters=[(35, runs[0][1])]),               # leaves the system
               dict(clusters=[(0, np.zeros((0, 0)))]),          # empty run
               dict(coarse=(10, 46, np.eye(30)))):              # more nodes than the system
        with pytest.raises(SolverError) as e:
            solver.reduced_solve(diag, edges, off, b, 1e-6, 100, **kw)
        assert e.value.status == _abi.ERR_INVALID_ARGUMENT, kw
    for kw in (dict(coarse=(0, 40, coarse[2])), dict(coarse=(10, 40, np.eye(30))),
               dict(clusters=[(0, np.eye(10))])):
        with pytest.raises(ValueError):
            solver.reduced_solve(diag, edges, off, b, 1e-6, 100, **kw)


@pytest.mark.gpu
def test_gpu_unsorted_edges_decline(solver):
    """As the reference's solver (reduced.rs, solves_are_deterministic_and_
    unsorted_edges_decline): edges out of order are declined, for either
    preconditioner; malformed edges are an invalid argument."""
    diag, edges, off = chain_system(60)
    b = pattern_rhs(60).reshape(-1, 6)
    runs = oracle.cluster_inverses(diag, edges, off, 16)
    swapped = edges.copy()
    swapped[[0, -1]] = swapped[[-1, 0]]
    off_sw = off.copy()
    off_sw[[0, -1]] = off_sw[[-1, 0]]
    for kw in ({}, dict(clusters=runs)):
        with pytest.raises(SolverError) as e:
            solver.reduced_solve(diag, swapped, off_sw, b, 1e-6, 100, **kw)
        assert e.value.status == _abi.DECLINED, kw
    bad = edges.copy()
    bad[3] = (bad[3][1], bad[3][0])  # a > b
    with pytest.raises(SolverError) as e:
        solver.reduced_solve(diag, bad, off, b, 1e-6, 100)
    assert e.value.status == _abi.ERR_INVALID_ARGUMENT
    # The sorted system still solves afterwards.
    _, it, rr = solver.reduced_solve(diag, edges, off, b, 1e-6, 500, clusters=runs)
    assert rr <= 1e-6 and it > 0


def relative_constraint_system(n, seed):
    """J^T J of random relative constraints M (x_b - x_a) in scaled variables
    along a capture-ordered chain (four neighbours each, n / 4 long-range
    edges), node scales 10^(1 + U(-1, 1)), a weak prior 1e-3 s^2 I: SPD and
    Laplacian-like (the shape of the reference's random_system,
    crates/ba-gpu/src/reduced.rs:1050-1098).  Blocks are rounded to f32 as the
    system hands them over."""
    rng = np.random.default_rng(seed)
    edges = {(b - d, b) for b in range(1, n) for d in range(1, min(4, b) + 1)}
    for _ in range(n // 4):
        a, b = (int(v) for v in rng.integers(0, n, 2))
        if a + 4 < b:
            edges.add((a, b))
    edges = sorted(edges)
    scale = 10.0 ** (rng.uniform(-1.0, 1.0, n) + 1.0)
    diag = [np.eye(6) * 1e-3 * s * s for s in scale]
    off = []
    for a, b in edges:
        m = rng.uniform(-1.0, 1.0, (6, 6)) + 2.0 * np.eye(6)
        fa, fb = -m * scale[a], m * scale[b]
        diag[a] = diag[a] + fa.T @ fa
        diag[b] = diag[b] + fb.T @ fb
        off.append((fb.T @ fa).astype(np.float32).astype(np.float64))
    rhs = (rng.uniform(-1.0, 1.0, (n, 6)) * scale[:, None] * 1e3).reshape(-1)
    return diag, np.array(edges, np.uint32), np.array(off), rhs


@pytest.mark.gpu
@pytest.mark.parametrize("n,k,group", [(300, 32, 16), (150, 1, None), (77, 32, None),
                                       (61, 8, 7)])
def test_gpu_matches_the_fp64_iteration_on_relative_constraints(solver, n, k, group):
    """The reference's gpu_pcg_matches_the_cpu_iteration cases (reduced.rs:
    1197-1250): runs of k nodes (k = 1: block-Jacobi), an optional coarse
    level over every node, tolerance 1e-2; the device within 1 + 10% of the
    FP64 iteration count, its true residual within 1.2 tol and its step
    within 1e-3 of the FP64 one."""
    diag, edges, off, b = relative_constraint_system(n, 7 + n)
    S = dense(diag, edges, off)
    runs = oracle.cluster_inverses(diag, edges, off, k) if k > 1 else None
    coarse = None
    if group:
        m = -(-n // group)
        P = np.zeros((6 * n, 6 * m))
        for i in range(n):
            P[6 * i:6 * i + 6, 6 * (i // group):6 * (i // group) + 6] = np.eye(6)
        coarse = (group, n, np.linalg.inv(P.T @ S @ P))
    tol = 1e-2
    x_ref, it_ref = oracle.reduced_pcg(diag, edges, off, b, tol, 500, clusters=runs,
                                       coarse=coarse)
    assert it_ref > 3
    variants = [dict(clusters=runs or [], coarse=coarse)]
    if runs is None and coarse is None:
        variants.append({})  # block-Jacobi through the persistent kernel too
    for kw in variants:
        x, it, _ = solver.reduced_solve(diag, edges, off, b.reshape(-1, 6), tol, 500, **kw)
        x = x.reshape(-1)
        assert abs(it - it_ref) <= 1 + it_ref // 10, (kw.keys(), it, it_ref)
        assert np.linalg.norm(b - S @ x) <= 1.2 * tol * np.linalg.norm(b)
        xr = x_ref.reshape(-1)
        assert np.linalg.norm(x - xr) <= 1e-3 * np.linalg.norm(xr)


@pytest.mark.parametrize("k", [7, 8, 16, 32])
def test_caller_side_helpers_match_the_oracle(k):
    """visloc_ba.reduced (the caller's preparation of the preconditioners,
    vectorised) against the oracle's restatements of cluster_inverses,
    coarse_correction and coarse_from_sums, on the chain and covisibility
    systems (ragged last runs and aggregates included)."""
    from visloc_ba import reduced

    for diag, edges, off in (chain_system(100), covisibility_system(64)):
        want = oracle.cluster_inverses(diag, edges, off, k)
        got = reduced.cluster_inverses(diag, edges, off, k)
        assert [s for s, _ in got] == [s for s, _ in want]
        for (_, a), (_, b) in zip(got, want):
            np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12 * np.abs(b).max())
        n = len(diag)
        for nodes, group in ((n, k), (n - 5, k - 1)):
            want_c = oracle.coarse_correction(diag, edges, off, nodes, group)
            got_c = reduced.coarse_correction(diag, edges, off, nodes, group)
            assert got_c[:2] == want_c[:2]
            np.testing.assert_allclose(got_c[2], want_c[2], rtol=1e-8,
                                       atol=1e-10 * np.abs(want_c[2]).max())
            sums = oracle.coarse_block_sums(edges, off, want_c[0], nodes)
            from_sums = reduced.coarse_from_sums(diag, sums, nodes, want_c[0])
            np.testing.assert_allclose(from_sums[2], want_c[2], rtol=1e-8,
                                       atol=1e-10 * np.abs(want_c[2]).max())


@pytest.mark.parametrize("threads", [1, 4])
def test_threaded_oracle_iteration_matches_the_numpy_one(threads):
    """The oracle's threaded C++ pcg_core (the reduced workload's CPU
    baseline) against its numpy restatement, pinned above to the reference's
    recorded counts: the chain system with runs of 32 and the coarse level,
    block-Jacobi on the covisibility system, and the breakdown case."""
    diag, edges, off = chain_system(600)
    off32 = off.astype(np.float32).astype(np.float64)
    b = pattern_rhs(600)
    runs = oracle.cluster_inverses(diag, edges, off32, 32)
    coarse = oracle.coarse_correction(diag, edges, off32, 600, 32)
    for kw in (dict(clusters=runs), dict(clusters=runs, coarse=coarse)):
        x_np, it_np = oracle.reduced_pcg(diag, edges, off32, b, 1e-8, 500, **kw)
        x_c, it_c = oracle.reduced_pcg_threaded(diag, edges, off, b, 1e-8, 500, threads=threads,
                                                **kw)
        assert abs(it_c - it_np) <= 1, (it_c, it_np)
        assert np.abs(x_c - x_np).max() <= 1e-6 * np.abs(x_np).max()
    d2, e2, o2 = covisibility_system(64)
    b2 = pattern_rhs(64)
    x_np, it_np = oracle.reduced_pcg(d2, e2, o2.astype(np.float32).astype(np.float64), b2, 1e-10, 500)
    x_c, it_c = oracle.reduced_pcg_threaded(d2, e2, o2, b2, 1e-10, 500, threads=threads)
    assert it_c == it_np and np.abs(x_c - x_np).max() <= 1e-9 * np.abs(x_np).max()
    bad = [np.eye(6), np.eye(6)]
    assert oracle.reduced_pcg_threaded(bad, np.array([(0, 1)]), np.array([2.0 * np.eye(6)]),
                                       np.concatenate([np.ones(6), -np.ones(6)]), 1e-8, 50) is None
