"""ctypes wrapper of the FP64 CPU oracle (liboracle_ba.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker.  The product never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
_PKG = os.path.join(_ROOT, "visloc-rs_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from visloc_ba import _abi  # noqa: E402
from visloc_ba.problem import PackedProblem, BaConfig, result_from_abi  # noqa: E402

LIB_PATH = os.path.join(_HERE, "liboracle_ba.so")
P = C.POINTER

EXPORTS = {
    "vlba_oracle_check": (C.c_int, [P(_abi.Problem), P(_abi.Config), P(C.c_uint64)]),
    "vlba_oracle_cost": (
        C.c_int,
        [P(_abi.Problem), P(_abi.Config), C.c_int, P(C.c_double), P(C.c_uint64)],
    ),
    "vlba_oracle_squared_residuals": (C.c_int, [P(_abi.Problem), P(_abi.Config), P(C.c_double)]),
    "vlba_oracle_reduced_pcg": (
        C.c_int,
        [C.c_uint32, C.c_uint64, P(C.c_uint32), P(C.c_double), P(C.c_float), P(C.c_double),
         C.c_double, C.c_uint32, C.c_uint32, P(C.c_uint32), P(C.c_uint32), P(C.c_double),
         C.c_uint32, C.c_uint32, P(C.c_double), C.c_int, P(C.c_double), P(C.c_uint32)],
    ),
    "vlba_oracle_camera_project": (C.c_int, [P(_abi.Camera), P(C.c_double), P(C.c_double)]),
    "vlba_oracle_mono_project": (
        C.c_int,
        [P(_abi.Camera), P(C.c_double), P(C.c_double), P(C.c_double)],
    ),
    "vlba_oracle_pose_update": (None, [P(C.c_double), P(C.c_double), P(C.c_double)]),
    "vlba_oracle_normal_equations": (
        C.c_int,
        [P(_abi.Problem), P(_abi.Config), C.c_int, P(C.c_double), P(C.c_double),
         P(C.c_double), P(C.c_double)],
    ),
    "vlba_oracle_reduced_system": (
        C.c_int,
        [P(_abi.Problem), P(_abi.Config), C.c_double, C.c_int, P(C.c_double),
         P(C.c_double), P(C.c_double), P(C.c_double)],
    ),
    "vlba_oracle_optimize": (
        C.c_int,
        [P(_abi.Problem), P(_abi.Config), C.c_int, C.c_int, P(_abi.Result),
         P(_abi.Iteration), C.c_uint32],
    ),
    "vlba_oracle_optimize_matrix_free": (
        C.c_int,
        [P(_abi.Problem), P(_abi.Config), C.c_uint32, C.c_double, C.c_double, C.c_int, C.c_int,
         P(_abi.Result), P(_abi.Iteration), C.c_uint32, P(C.c_uint64), P(C.c_uint32)],
    ),
    "vlba_oracle_mf_system": (
        C.c_int,
        [C.c_uint32, P(C.c_double), P(C.c_double), C.c_uint32, P(C.c_double), P(C.c_double),
         P(C.c_uint32), P(C.c_uint32), P(C.c_double), C.c_double, C.c_int, P(C.c_double),
         P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double), C.c_int, P(C.c_double),
         C.c_uint32, C.c_double, C.c_double, P(C.c_double), P(C.c_uint32), P(C.c_double),
         P(C.c_double), P(C.c_double)],
    ),
}

_LIB = None


def build():
    """Compile the oracle with its Makefile (g++ -fopenmp)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        _LIB = _abi.bind(C.CDLL(LIB_PATH), EXPORTS)
    return _LIB


def _dp(a):
    return a.ctypes.data_as(P(C.c_double))


SPARSE = 1
DENSE = 0
# LinearSolver::Sparse factored in band storage (capture or fold order) when the
# reduced system is banded; otherwise as SPARSE.
SPARSE_BANDED = 2


def optimize(packed: PackedProblem, config: BaConfig, solver: int = DENSE, threads: int = 0):
    """Run the oracle LM in place on `packed`; returns (status, BaResult)."""
    prob = packed.abi()
    cfg = config.to_abi()
    res = _abi.Result()
    cap = max(1, int(config.max_iterations))
    iters = (_abi.Iteration * cap)()
    st = lib().vlba_oracle_optimize(C.byref(prob), C.byref(cfg), solver, threads,
                                    C.byref(res), iters, cap)
    return st, result_from_abi(res, iters, res.num_iterations)


# ImplicitSchurError of the matrix-free restatement (implicit_schur.rs).
MF_OK, MF_NON_FINITE, MF_NON_SPD_PRECONDITIONER, MF_MAX_ITERATIONS = 0, 1, 2, 3
MF_NON_POSITIVE_CURVATURE, MF_RESIDUAL_CHECK_FAILED, MF_EMPTY_SYSTEM = 4, 5, 6
MF_INVALID_TOLERANCE = 7


def optimize_matrix_free(packed: PackedProblem, config: BaConfig, max_pcg_iterations: int = 128,
                         pcg_relative_tolerance: float = 1e-12,
                         pcg_absolute_tolerance: float = 1e-12, cluster8: bool = False,
                         threads: int = 0):
    """BundleAdjustment::optimize_matrix_free (bundle/optimize.rs:105-139)
    in place on `packed`, the MatrixFreeBaOptions defaults as defaults:
    (status, BaResult, total PCG iterations, failed linear solves)."""
    prob = packed.abi()
    cfg = config.to_abi()
    res = _abi.Result()
    cap = max(1, int(config.max_iterations))
    iters = (_abi.Iteration * cap)()
    total = C.c_uint64()
    failed = C.c_uint32()
    st = lib().vlba_oracle_optimize_matrix_free(
        C.byref(prob), C.byref(cfg), int(max_pcg_iterations), float(pcg_relative_tolerance),
        float(pcg_absolute_tolerance), int(bool(cluster8)), threads, C.byref(res), iters, cap,
        C.byref(total), C.byref(failed))
    return st, result_from_abi(res, iters, res.num_iterations), total.value, failed.value


def mf_system(diag, b_p, h_ll, b_l, cross, lam, *, cluster8=False, x=None, probe=None,
              solve=False, rhs=None, max_iterations=128, relative_tolerance=1e-12,
              absolute_tolerance=1e-12):
    """The matrix-free operator on a normal-equation system given directly
    (NormalEquationsBa with pose blocks): diag (np,6,6), b_p (6 np), h_ll
    (nl,3,3), b_l (nl,3), cross: per landmark a list of (pose, 6x3 block).
    Returns a dict with the status and the requested outputs: rhs, apply
    (S x), precond (M^-1 probe), and with solve the PCG solution,
    iterations, residual, target and the landmark step delta_l."""
    diag = np.ascontiguousarray(diag, np.float64).reshape(-1, 36)
    npose = diag.shape[0]
    b_p = np.ascontiguousarray(b_p, np.float64).reshape(-1)
    h_ll = np.ascontiguousarray(h_ll, np.float64).reshape(-1, 9)
    nl = h_ll.shape[0]
    b_l = np.ascontiguousarray(b_l, np.float64).reshape(-1)
    counts = np.array([len(c) for c in cross], np.uint32)
    poses = np.array([p for c in cross for p, _ in c], np.uint32)
    blocks = np.ascontiguousarray(
        np.array([np.asarray(b, np.float64).reshape(6, 3) for c in cross for _, b in c]).reshape(-1))
    n = 6 * npose
    out = {"rhs": np.empty(n)}
    none = P(C.c_double)()
    args_x = none
    if x is not None:
        x = np.ascontiguousarray(x, np.float64)
        out["apply"] = np.empty(n)
        args_x = _dp(x)
    args_probe = none
    if probe is not None:
        probe = np.ascontiguousarray(probe, np.float64)
        out["precond"] = np.empty(n)
        args_probe = _dp(probe)
    sol = np.zeros(n)
    dl = np.zeros(3 * nl)
    it = C.c_uint32()
    resid = C.c_double()
    tgt = C.c_double()
    rhs_arr = None if rhs is None else np.ascontiguousarray(rhs, np.float64)
    st = lib().vlba_oracle_mf_system(
        npose, _dp(diag), _dp(b_p), nl, _dp(h_ll), _dp(b_l), counts.ctypes.data_as(P(C.c_uint32)),
        poses.ctypes.data_as(P(C.c_uint32)), _dp(blocks), float(lam), int(bool(cluster8)),
        args_x, _dp(out["apply"]) if x is not None else none, args_probe,
        _dp(out["precond"]) if probe is not None else none, _dp(out["rhs"]), int(bool(solve)),
        none if rhs_arr is None else _dp(rhs_arr), int(max_iterations), float(relative_tolerance),
        float(absolute_tolerance), _dp(sol), C.byref(it), C.byref(resid), C.byref(tgt), _dp(dl))
    out["status"] = st
    if solve:
        out.update(solution=sol, iterations=it.value, residual=resid.value, target=tgt.value,
                   delta_l=dl)
    return out


def cost(packed: PackedProblem, config: BaConfig | None = None, threads: int = 0):
    config = config or BaConfig()
    c = C.c_double()
    n = C.c_uint64()
    st = lib().vlba_oracle_cost(C.byref(packed.abi()), C.byref(config.to_abi()), threads,
                                C.byref(c), C.byref(n))
    if st != 0:
        raise RuntimeError(f"oracle cost failed: {_abi.STATUS_NAMES.get(st, st)}")
    return c.value, n.value


def squared_residuals(packed: PackedProblem, config: BaConfig | None = None):
    """Per-observation squared reprojection residual (NaN: not evaluable)."""
    import numpy as np

    config = config or BaConfig()
    out = np.empty(packed.num_observations)
    st = lib().vlba_oracle_squared_residuals(C.byref(packed.abi()), C.byref(config.to_abi()),
                                             _dp(out))
    if st != 0:
        raise RuntimeError(f"oracle residuals failed: {_abi.STATUS_NAMES.get(st, st)}")
    return out


# ------------------------------------------------------------------- GNC
# BundleAdjustment::optimize_gnc (bundle/lm.rs:28-142) over the oracle's
# weighted LM, with the surrogate math of the reference's crate gnc
# (pipelines/slam/src/gnc.rs:150-270) restated here in Python, apart from the
# library's C++ restatement it checks.
TLS_TERMINAL_MU = 200.0


class GncSurrogate:
    def __init__(self, kernel: int, c: float, factor: float, max_residual_sq: float):
        self.kernel, self.c2, self.factor = kernel, c * c, factor
        s_max = max(max_residual_sq, 0.0)
        if kernel == _abi.GNC_TRUNCATED_LEAST_SQUARES:
            denom = 2.0 * s_max - self.c2
            self.mu = TLS_TERMINAL_MU if denom <= 0.0 else min(max(self.c2 / denom, 2.2250738585072014e-308),
                                                                  TLS_TERMINAL_MU)
        else:
            self.mu = max(2.0 * s_max / self.c2, 1.0)

    def weight(self, s: float) -> float:
        s = max(s, 0.0)
        if self.kernel == _abi.GNC_TRUNCATED_LEAST_SQUARES:
            mu = self.mu
            lo, hi = mu / (mu + 1.0) * self.c2, (mu + 1.0) / mu * self.c2
            if s <= lo:
                return 1.0
            if s >= hi:
                return 0.0
            return (self.c2 * mu * (mu + 1.0) / s) ** 0.5 - mu
        m = self.mu * self.c2
        r = m / (s + m)
        return r * r

    def terminal(self) -> bool:
        if self.kernel == _abi.GNC_TRUNCATED_LEAST_SQUARES:
            return self.mu >= TLS_TERMINAL_MU
        return self.mu <= 1.0

    def anneal(self) -> bool:
        if self.kernel == _abi.GNC_TRUNCATED_LEAST_SQUARES:
            self.mu = min(self.mu * self.factor, TLS_TERMINAL_MU)
        else:
            self.mu = max(self.mu / self.factor, 1.0)
        return self.terminal()


def _median(v):
    v = sorted(v)
    n = len(v)
    return v[n // 2] if n % 2 else 0.5 * (v[n // 2 - 1] + v[n // 2])


def estimate_scale_mad(squared, k: float):
    import math

    rho = [math.sqrt(s) for s in squared if math.isfinite(s) and s >= 0.0]
    if len(rho) < 2:
        return None
    med = _median(rho)
    mad = _median([abs(r - med) for r in rho])
    return med + k * 1.4826 * mad


def optimize_gnc(packed: PackedProblem, config: BaConfig, gnc, threads: int = 0):
    """In place on `packed`: (BaGncResult fields as a dict, final weights)."""
    import copy
    import math

    import numpy as np

    none = BaConfig(robust_kernel=_abi_none_kernel())
    sq = squared_residuals(packed, none)
    finite = np.isfinite(sq)
    initial_cost = float(sq[finite].sum())
    s_max = float(sq[finite].max()) if finite.any() else 0.0
    c = gnc.c
    if gnc.auto_scale is not None:
        est = estimate_scale_mad(sq, gnc.auto_scale)
        if est is not None:
            c = max(est, gnc.c)
    inlier_scale = c
    state = GncSurrogate(gnc.kernel, c, gnc.anneal_factor, s_max)
    inner = copy.copy(config)
    inner.robust_kernel = _abi_none_kernel()
    inner.max_iterations = max(1, gnc.inner_iterations)
    w = np.ones(packed.num_observations)
    outer, converged = 0, False
    for _ in range(max(1, gnc.max_outer)):
        outer += 1
        terminal = state.terminal()
        sq = squared_residuals(packed, none)
        if gnc.auto_scale_readapt and gnc.auto_scale is not None:
            est = estimate_scale_mad(sq, gnc.auto_scale)
            if est is not None:
                cc = max(est, gnc.c)
                state.c2 = cc * cc
                inlier_scale = cc
        w = np.array([state.weight(s) if math.isfinite(s) else 1.0 for s in sq])
        packed.obs_weight = w
        st, _ = optimize(packed, inner, threads=threads)
        packed.obs_weight = None
        if st != 0:
            raise RuntimeError(f"oracle GNC inner solve failed: {_abi.STATUS_NAMES.get(st, st)}")
        if terminal:
            converged = True
            break
        state.anneal()
    sq = squared_residuals(packed, none)
    w = np.array([state.weight(s) if math.isfinite(s) else math.nan for s in sq])
    ok = np.isfinite(sq)
    final_cost = float((w[ok] * sq[ok]).sum())
    inlier_cost = float(sq[ok & (w >= 0.5)].sum())
    return {"initial_cost": initial_cost, "final_cost": final_cost, "inlier_cost": inlier_cost,
            "inlier_scale": inlier_scale, "observation_count": packed.num_observations,
            "outer_iterations": outer, "converged": converged}, w


def _abi_none_kernel():
    from visloc_ba.problem import RobustKernel

    return RobustKernel.none()


def check(packed: PackedProblem, config: BaConfig | None = None):
    config = config or BaConfig()
    idx = C.c_uint64()
    st = lib().vlba_oracle_check(C.byref(packed.abi()), C.byref(config.to_abi()), C.byref(idx))
    return st, idx.value


def camera_project(camera_abi, xc):
    xc = np.ascontiguousarray(xc, dtype=np.float64)
    out = np.zeros(2)
    ok = lib().vlba_oracle_camera_project(C.byref(camera_abi), _dp(xc), _dp(out))
    return (out if ok == 1 else None), ok


def mono_project(camera_abi, xc):
    xc = np.ascontiguousarray(xc, dtype=np.float64)
    pred = np.zeros(2)
    jac = np.zeros(6)
    ok = lib().vlba_oracle_mono_project(C.byref(camera_abi), _dp(xc), _dp(pred), _dp(jac))
    return (pred, jac.reshape(2, 3)) if ok == 1 else None


def pose_update(q, t, xi):
    q = np.array(q, dtype=np.float64)
    t = np.array(t, dtype=np.float64)
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    lib().vlba_oracle_pose_update(_dp(q), _dp(t), _dp(xi))
    return q, t


def normal_equations(packed: PackedProblem, config: BaConfig | None = None, threads: int = 0):
    config = config or BaConfig()
    npv = int(packed.num_poses - (0 if packed.pose_fixed is None else packed.pose_fixed.sum()))
    nlv = int(packed.num_landmarks
              - (0 if packed.landmark_fixed is None else packed.landmark_fixed.sum()))
    h_pp = np.zeros((npv, 6, 6))
    b_p = np.zeros((npv, 6))
    h_ll = np.zeros((nlv, 3, 3))
    b_l = np.zeros((nlv, 3))
    st = lib().vlba_oracle_normal_equations(C.byref(packed.abi()), C.byref(config.to_abi()),
                                            threads, _dp(h_pp), _dp(b_p), _dp(h_ll), _dp(b_l))
    if st != 0:
        raise RuntimeError(f"oracle normal equations failed: {st}")
    return h_pp, b_p, h_ll, b_l


def reduced_system(packed: PackedProblem, lam: float, config: BaConfig | None = None,
                   threads: int = 0, step: bool = True):
    """(S (6P x 6P), rhs (6P), dp (6P), dl (3L)) at damping `lam`."""
    config = config or BaConfig()
    npv = int(packed.num_poses - (0 if packed.pose_fixed is None else packed.pose_fixed.sum()))
    nlv = int(packed.num_landmarks
              - (0 if packed.landmark_fixed is None else packed.landmark_fixed.sum()))
    s = np.zeros((6 * npv, 6 * npv))
    rhs = np.zeros(6 * npv)
    dp = np.zeros(6 * npv)
    dl = np.zeros(3 * nlv)
    st = lib().vlba_oracle_reduced_system(
        C.byref(packed.abi()), C.byref(config.to_abi()), lam, threads, _dp(s), _dp(rhs),
        _dp(dp) if step else P(C.c_double)(), _dp(dl) if step else P(C.c_double)())
    return st, s, rhs, dp, dl


# ------------------------------------------- reduced solve preconditioners
# numpy restatement of the CPU iteration that ReducedSolveAccelerator::solve
# replaces, with its two preconditioners.  Blocks are numpy 6x6 matrices:
# diag[i] node i's damped diagonal block, offdiag[e] the (row b, column a)
# block of edge edges[e] = (a, b), a < b.

COARSE_MAX_AGGREGATES = 256  # PCG_COARSE_MAX_AGGREGATES, rig_ba_solver.rs:1158


def cluster_inverses(diag, edges, offdiag, k: int):
    """(first node, inverse) of S restricted to each run of k consecutive
    nodes, the last run shorter (cluster_inverses, pipelines/slam/src/
    colmap_incremental/rig_ba_solver.rs:1112-1140); None when a run is not
    positive definite."""
    n = len(diag)
    starts = list(range(0, n, k))
    mats = []
    for s in starts:
        m = min(k, n - s)
        a = np.zeros((6 * m, 6 * m))
        for i in range(m):
            a[6 * i:6 * i + 6, 6 * i:6 * i + 6] = diag[s + i]
        mats.append(a)
    for (ea, eb), blk in zip(np.asarray(edges).reshape(-1, 2), offdiag):
        ea, eb = int(ea), int(eb)
        if ea // k != eb // k:
            continue
        c, ia, ib = ea // k, ea % k, eb % k
        mats[c][6 * ib:6 * ib + 6, 6 * ia:6 * ia + 6] = blk
        mats[c][6 * ia:6 * ia + 6, 6 * ib:6 * ib + 6] = np.asarray(blk).T
    out = []
    for s, a in zip(starts, mats):
        try:
            L = np.linalg.cholesky(a)
        except np.linalg.LinAlgError:
            return None
        Li = np.linalg.inv(L)
        out.append((s, Li.T @ Li))
    return out


def coarse_correction(diag, edges, offdiag, n_frames: int, group: int):
    """(group, n_frames, (P^T S P)^-1) of the additive coarse level over the
    leading n_frames nodes, group raised so that there are at most 256
    aggregates (coarse_correction, rig_ba_solver.rs:1235-1266, and
    CoarseCorrection::inverse, :1218-1229); None for fewer than two
    aggregates or a coarse matrix that is not positive definite."""
    group = max(group, -(-n_frames // COARSE_MAX_AGGREGATES))
    m = -(-n_frames // group)
    if m < 2:
        return None
    a = np.zeros((6 * m, 6 * m))
    for i in range(n_frames):
        g = i // group * 6
        a[g:g + 6, g:g + 6] += diag[i]
    for (ea, eb), blk in zip(np.asarray(edges).reshape(-1, 2), offdiag):
        ea, eb = int(ea), int(eb)
        if ea >= n_frames or eb >= n_frames:
            continue
        ga, gb = ea // group * 6, eb // group * 6
        a[gb:gb + 6, ga:ga + 6] += blk
        a[ga:ga + 6, gb:gb + 6] += np.asarray(blk).T
    try:
        np.linalg.cholesky(a)
    except np.linalg.LinAlgError:
        return None
    return group, n_frames, np.linalg.inv(a)


def reduced_matvec(diag, edges, offdiag):
    """p -> S p over the block layout (edge_product, rig_ba_solver.rs:
    1314-1331: each edge adds B p_a to row b and B^T p_b to row a)."""
    diag = np.asarray(diag, np.float64)
    e = np.asarray(edges, np.int64).reshape(-1, 2)
    off = np.asarray(offdiag, np.float64).reshape(-1, 6, 6)

    def mv(p):
        p = p.reshape(-1, 6)
        q = np.einsum("nij,nj->ni", diag, p)
        if len(e):
            np.add.at(q, e[:, 1], np.einsum("eij,ej->ei", off, p[e[:, 0]]))
            np.add.at(q, e[:, 0], np.einsum("eji,ej->ei", off, p[e[:, 1]]))
        return q.reshape(-1)

    return mv


def reduced_pcg(diag, edges, offdiag, rhs, tol: float, max_iterations: int,
                clusters=None, coarse=None):
    """pcg_core (rig_ba_solver.rs:1406-1480) in FP64: z = M r by the run
    inverses (block-Jacobi without runs, and for nodes in no run) plus the
    coarse level z += P (P^T S P)^-1 P^T r (CoarseCorrection::add_to,
    :1198-1213); x = 0, r = b, p = z; stop once |r| <= tol |b| or after
    max_iterations.  Returns (x (n, 6), iterations), or None on a p.q that
    is not positive and finite."""
    n = len(diag)
    mv = reduced_matvec(diag, edges, offdiag)
    jac = [np.linalg.inv(np.asarray(d, np.float64)) for d in diag]
    runs = [(int(s), np.asarray(inv, np.float64)) for s, inv in (clusters or [])]

    def apply(r):
        rb = r.reshape(n, 6)
        z = np.stack([jac[i] @ rb[i] for i in range(n)]).reshape(-1)
        for s, inv in runs:
            m = inv.shape[0]
            z[6 * s:6 * s + m] = inv @ r[6 * s:6 * s + m]
        if coarse is not None:
            group, nodes, cinv = coarse
            m = cinv.shape[0] // 6
            rc = np.zeros(6 * m)
            for i in range(nodes):
                rc[i // group * 6:i // group * 6 + 6] += rb[i]
            yc = np.asarray(cinv) @ rc
            for i in range(nodes):
                z[6 * i:6 * i + 6] += yc[i // group * 6:i // group * 6 + 6]
        return z

    b = np.asarray(rhs, np.float64).reshape(-1)
    bn = np.sqrt(b @ b)
    x = np.zeros_like(b)
    if bn == 0.0:
        return x.reshape(n, 6), 0
    r = b.copy()
    z = apply(r)
    p = z.copy()
    rz = r @ z
    it = 0
    for _ in range(max_iterations):
        it += 1
        q = mv(p)
        pq = p @ q
        if not np.isfinite(pq) or pq <= 0.0:
            return None
        alpha = rz / pq
        x += alpha * p
        r -= alpha * q
        if np.sqrt(r @ r) <= tol * bn:
            break
        z = apply(r)
        rz_next = r @ z
        beta = rz_next / rz
        rz = rz_next
        p = z + beta * p
    return x.reshape(n, 6), it


def eliminate_blocks(num_edges_or_edges, point_off, point_nodes, hcp, point_inverse, extra=()):
    """The off-diagonal blocks of a point elimination in FP64 (the CPU's
    eliminate_by_output, pipelines/slam/src/colmap_incremental/
    rig_ba_solver.rs:2551-2648, as PointElimination documents it,
    pipelines/slam/src/ba_accel.rs:74-80): for each point and each pair of
    its nodes k < j, block(s, t) -= hcp[j] V^-1 hcp[k]^T, then the direct
    couplings are added.  Blocks are (row t, column s) numpy 6x6."""
    edges = np.asarray(num_edges_or_edges).reshape(-1, 2)
    index = {(int(a), int(b)): e for e, (a, b) in enumerate(edges)}
    blocks = np.zeros((len(edges), 6, 6))
    for p in range(len(point_off) - 1):
        v = point_inverse[p]
        if v is None:
            continue
        lo, hi = int(point_off[p]), int(point_off[p + 1])
        nodes = [int(x) for x in point_nodes[lo:hi]]
        h = np.asarray(hcp[lo:hi], np.float64)
        for k in range(len(nodes)):
            scaled = h[k] @ v
            for j in range(k + 1, len(nodes)):
                blocks[index[(nodes[k], nodes[j])]] -= h[j] @ scaled.T
    for e, m in extra:
        blocks[int(e)] += m
    return blocks


def coarse_block_sums(edges, blocks, group: int, nodes: int):
    """sums[g m + h] (g <= h): the sum of the blocks of edges (a, b) with a
    in aggregate g and b in aggregate h, both below `nodes`
    (EliminatedBlocks::coarse_sums, ba_accel.rs:119-125); zero for g > h."""
    m = -(-nodes // group)
    sums = np.zeros((m * m, 6, 6))
    for (a, b), blk in zip(np.asarray(edges).reshape(-1, 2), blocks):
        a, b = int(a), int(b)
        if a < nodes and b < nodes:
            sums[(a // group) * m + b // group] += blk
    return sums


def coarse_from_sums(diag, sums, n_frames: int, group: int):
    """(group, n_frames, inverse) of the coarse level from aggregate-pair
    block sums (coarse_from_sums, rig_ba_solver.rs:1276-1308): the diagonal
    blocks summed per aggregate, each sum added to the (h, g) block and its
    transpose to (g, h); None for fewer than two aggregates or a matrix that
    is not positive definite."""
    m = -(-n_frames // group)
    if m < 2 or len(sums) != m * m:
        return None
    a = np.zeros((6 * m, 6 * m))
    for i in range(n_frames):
        g = i // group * 6
        a[g:g + 6, g:g + 6] += diag[i]
    for g in range(m):
        for h in range(g, m):
            s = sums[g * m + h]
            a[6 * h:6 * h + 6, 6 * g:6 * g + 6] += s
            a[6 * g:6 * g + 6, 6 * h:6 * h + 6] += s.T
    try:
        np.linalg.cholesky(a)
    except np.linalg.LinAlgError:
        return None
    return group, n_frames, np.linalg.inv(a)


def reduced_pcg_threaded(diag, edges, offdiag, rhs, tol: float, max_iterations: int,
                         clusters=None, coarse=None, threads: int = 0):
    """pcg_core on the host's threads (the C++ restatement in ba_oracle.cpp):
    the same iteration as reduced_pcg with the off-diagonal blocks read as
    f32, as the plug-in receives them.  Returns (x (n, 6), iterations), or
    None where pcg_core returns None."""
    diag = np.ascontiguousarray(np.asarray(diag, np.float64).transpose(0, 2, 1))  # column-major
    off = np.ascontiguousarray(np.asarray(offdiag, np.float32).reshape(-1, 6, 6).transpose(0, 2, 1))
    e = np.ascontiguousarray(np.asarray(edges, np.uint32).reshape(-1, 2))
    b = np.ascontiguousarray(np.asarray(rhs, np.float64).reshape(-1))
    n = diag.shape[0]
    runs = clusters or []
    first = np.ascontiguousarray([r[0] for r in runs], np.uint32)
    size = np.ascontiguousarray([np.shape(r[1])[0] // 6 for r in runs], np.uint32)
    inv = np.ascontiguousarray(np.concatenate(
        [np.asarray(r[1], np.float64).T.reshape(-1) for r in runs]) if runs else np.zeros(1))
    group, nodes, cinv = coarse if coarse is not None else (0, 0, np.zeros((1, 1)))
    cinv = np.ascontiguousarray(np.asarray(cinv, np.float64).T)
    x = np.zeros(6 * n)
    it = C.c_uint32()
    st = lib().vlba_oracle_reduced_pcg(
        n, e.shape[0], e.ctypes.data_as(P(C.c_uint32)), _dp(diag), off.ctypes.data_as(P(C.c_float)),
        _dp(b), float(tol), int(max_iterations), len(runs), first.ctypes.data_as(P(C.c_uint32)),
        size.ctypes.data_as(P(C.c_uint32)), _dp(inv), int(group), int(nodes), _dp(cinv),
        int(threads), _dp(x), C.byref(it))
    if st != 0:
        return None
    return x.reshape(n, 6), it.value
