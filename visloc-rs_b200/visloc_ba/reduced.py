"""Caller-side preparation of the reduced solve's preconditioners, in numpy:
what the COLMAP-port rig solver computes on its CPU before it offers a
ReducedCameraSystem (pipelines/slam/src/ba_accel.rs:50-72) to the
accelerator.

- cluster_inverses: inverses of the system restricted to runs of k
  consecutive nodes (cluster_inverses, pipelines/slam/src/colmap_incremental/
  rig_ba_solver.rs:1112-1140), one batched Cholesky per run length.
- coarse_correction / coarse_from_sums: the inverse of the aggregated matrix
  P^T S P of the additive coarse level (:1235-1266, :1276-1308), from the
  blocks or from the aggregate-pair sums that reduced_eliminate returns.

Blocks are numpy 6x6 matrices: diag[i] node i's damped diagonal block,
offdiag[e] the (row b, column a) block of edge edges[e] = (a, b), a < b."""

from __future__ import annotations

import numpy as np

COARSE_MAX_AGGREGATES = 256  # PCG_COARSE_MAX_AGGREGATES, rig_ba_solver.rs:1158


def _spd_inverse(a):
    """Inverses of a stack of SPD matrices by Cholesky; None if one is not
    positive definite."""
    try:
        L = np.linalg.cholesky(a)
    except np.linalg.LinAlgError:
        return None
    eye = np.broadcast_to(np.eye(a.shape[-1]), a.shape)
    Li = np.linalg.solve(L, eye)
    return np.swapaxes(Li, -1, -2) @ Li


def cluster_inverses(diag, edges, offdiag, k: int):
    """[(first node, inverse (6m, 6m))] over runs of k consecutive nodes (the
    last run shorter); None when a run is not positive definite."""
    diag = np.asarray(diag, np.float64)
    n = diag.shape[0]
    nfull, rest = divmod(n, k)
    runs = []
    edges = np.asarray(edges, np.int64).reshape(-1, 2)
    off = np.asarray(offdiag, np.float64).reshape(-1, 6, 6)
    inside = (edges[:, 0] // k) == (edges[:, 1] // k)
    ea, eb, blk = edges[inside, 0], edges[inside, 1], off[inside]
    for first, m, count in ((0, k, nfull), (nfull * k, rest, 1 if rest else 0)):
        if count == 0:
            continue
        mats = np.zeros((count, 6 * m, 6 * m))
        v = mats.reshape(count, m, 6, m, 6)
        local = np.arange(count * m)
        node = first + local
        v[local // m, local % m, :, local % m, :] = diag[node]
        sel = (ea >= first) & (ea < first + count * m)
        c, ia, ib = (ea[sel] - first) // m, (ea[sel] - first) % m, (eb[sel] - first) % m
        v[c, ib, :, ia, :] = blk[sel]
        v[c, ia, :, ib, :] = np.swapaxes(blk[sel], 1, 2)
        inv = _spd_inverse(mats)
        if inv is None:
            return None
        runs += [(first + i * m, inv[i]) for i in range(count)]
    return runs


def coarse_group_size(n_frames: int, group: int) -> int:
    """The aggregate size, raised so that there are at most 256 aggregates."""
    return max(group, -(-n_frames // COARSE_MAX_AGGREGATES))


def _coarse(a, group, n_frames):
    inv = _spd_inverse(a)
    return None if inv is None else (group, n_frames, inv)


def coarse_correction(diag, edges, offdiag, n_frames: int, group: int):
    """(group, n_frames, (P^T S P)^-1) over the leading n_frames nodes; None
    for fewer than two aggregates or a matrix that is not positive definite."""
    group = coarse_group_size(n_frames, group)
    m = -(-n_frames // group)
    if m < 2:
        return None
    diag = np.asarray(diag, np.float64)
    edges = np.asarray(edges, np.int64).reshape(-1, 2)
    off = np.asarray(offdiag, np.float64).reshape(-1, 6, 6)
    a = np.zeros((m, 6, m, 6))
    g = np.arange(n_frames) // group
    np.add.at(a, (g, slice(None), g, slice(None)), diag[:n_frames].transpose(0, 1, 2))
    sel = (edges[:, 0] < n_frames) & (edges[:, 1] < n_frames)
    ga, gb, blk = edges[sel, 0] // group, edges[sel, 1] // group, off[sel]
    sums = np.zeros((m, m, 6, 6))
    np.add.at(sums, (gb, ga), blk)
    a += sums.transpose(0, 2, 1, 3)
    a += sums.transpose(1, 3, 0, 2)
    return _coarse(a.reshape(6 * m, 6 * m), group, n_frames)


def coarse_from_sums(diag, sums, n_frames: int, group: int):
    """The same from aggregate-pair block sums sums[g m + h], g <= h (the
    edges from aggregate g to h), as reduced_eliminate returns them; group
    is already the adjusted aggregate size."""
    m = -(-n_frames // group)
    if m < 2 or len(sums) != m * m:
        return None
    diag = np.asarray(diag, np.float64)
    a = np.zeros((m, 6, m, 6))
    g = np.arange(n_frames) // group
    np.add.at(a, (g, slice(None), g, slice(None)), diag[:n_frames])
    s = np.asarray(sums, np.float64).reshape(m, m, 6, 6) * np.triu(np.ones((m, m)))[:, :, None, None]
    a += s.transpose(1, 2, 0, 3)   # sum (g, h) to the (h, g) block
    a += s.transpose(0, 3, 1, 2)   # its transpose to the (g, h) block
    return _coarse(a.reshape(6 * m, 6 * m), group, n_frames)
