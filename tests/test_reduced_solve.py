"""visloc_ba_cuda_reduced_solve: the ReducedSolveAccelerator::solve path
(pipelines/slam/src/ba_accel.rs:50-72, 128-135), block-Jacobi PCG on a
reduced camera system given in the reference's layout."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from visloc_ba import BaConfig, RobustKernel, synth

pytestmark = pytest.mark.gpu


def reference_layout(S, rhs):
    """Dense S (6n x 6n) to the reference's parts: diagonal blocks, sorted
    edges (a, b), a < b, with their (row b, column a) blocks."""
    n = S.shape[0] // 6
    B = S.reshape(n, 6, n, 6).transpose(0, 2, 1, 3)  # B[i, j] = block (i, j)
    diag = np.stack([B[i, i] for i in range(n)])
    edges, off = [], []
    for a in range(n):
        for b in range(a + 1, n):
            if np.any(B[b, a] != 0.0):
                edges.append((a, b))
                off.append(B[b, a])
    return diag, np.array(edges, np.uint32).reshape(-1, 2), np.array(off).reshape(-1, 6, 6), \
        rhs.reshape(n, 6)


def block_jacobi_pcg(S, b, tol, max_it):
    """The CPU iteration the accelerator replaces: PCG with the inverses of
    the 6x6 diagonal blocks, stopping once |r| <= tol |b| (FP64)."""
    n = S.shape[0] // 6
    Minv = [np.linalg.inv(S[6 * i:6 * i + 6, 6 * i:6 * i + 6]) for i in range(n)]

    def prec(r):
        return np.concatenate([Minv[i] @ r[6 * i:6 * i + 6] for i in range(n)])

    x = np.zeros_like(b)
    r = b.copy()
    z = prec(r)
    p = z.copy()
    rz = r @ z
    bn = np.linalg.norm(b)
    for k in range(max_it):
        if np.linalg.norm(r) <= tol * bn:
            return x, k
        q = S @ p
        alpha = rz / (p @ q)
        x += alpha * p
        r -= alpha * q
        z = prec(r)
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, max_it


@pytest.mark.parametrize("maker,lam", [
    (lambda: synth.ring_problem(70, 4000, seed=81), 1e-2),
    (lambda: synth.street_loop(200, 8000, seed=82), 1e-1),
    (lambda: synth.stereo_window(33, 2000, seed=83), 1e-3),
])
def test_reduced_solve_matches_the_fp64_iteration(solver, maker, lam):
    p = maker()
    cfg = BaConfig(robust_kernel=RobustKernel.huber(1.0))
    st, S, rhs, _, _ = oracle.reduced_system(p, lam, cfg, step=False)
    assert st == 0
    diag, edges, off, b = reference_layout(S, rhs)
    tol = 1e-6
    x, iters, rr = solver.reduced_solve(diag, edges, off, b, tol, 500)
    x_ref, it_ref = block_jacobi_pcg(S, rhs, tol, 500)
    exact = np.linalg.solve(S, rhs)
    assert rr <= tol
    assert abs(iters - it_ref) <= max(3, it_ref // 10), (iters, it_ref)
    assert np.abs(x.reshape(-1) - exact).max() <= 1e-3 * np.abs(exact).max()


def test_reduced_solve_stops_at_the_iteration_cap(solver):
    p = synth.street_loop(200, 8000, seed=84)
    st, S, rhs, _, _ = oracle.reduced_system(p, 1e-3, BaConfig(), step=False)
    diag, edges, off, b = reference_layout(S, rhs)
    x, iters, rr = solver.reduced_solve(diag, edges, off, b, 1e-12, 7)
    assert iters == 7 and rr > 1e-12


def test_layout_reuse_takes_each_calls_values(solver):
    """Solves of the same edges reuse the device layout: each call's blocks,
    right-hand side, tolerance and iteration cap must still be the ones
    used (twice the matrix gives half the step; a cap of 4, then a full
    solve, on the persistent kernel and on the preconditioned loop)."""
    p = synth.street_loop(120, 5000, seed=87)
    st, S, rhs, _, _ = oracle.reduced_system(p, 1e-1, BaConfig(), step=False)
    diag, edges, off, b = reference_layout(S, rhs)
    for kw in ({}, dict(clusters=[])):
        x1, it1, rr1 = solver.reduced_solve(diag, edges, off, b, 1e-6, 500, **kw)
        x2, it2, _ = solver.reduced_solve(2 * diag, edges, 2 * off, b, 1e-6, 500, **kw)
        assert rr1 <= 1e-6
        assert np.abs(2 * x2 - x1).max() <= 1e-4 * np.abs(x1).max()
        _, it3, rr3 = solver.reduced_solve(diag, edges, off, b, 1e-6, 4, **kw)
        assert it3 == 4 and rr3 > 1e-6
        _, it4, rr4 = solver.reduced_solve(diag, edges, off, b, 1e-6, 500, **kw)
        assert it4 == it1 and rr4 <= 1e-6
