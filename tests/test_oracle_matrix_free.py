"""The oracle's matrix-free FP64 backend (the restatement of the reference's
ImplicitSchurOperator, its PCG and BundleAdjustment::optimize_matrix_free)
pinned by the reference's own tests of that code: the closed-form values of
the hand-check system, the operator against the explicit Schur complement,
the grouped rig block of the preconditioner, the PCG limits, determinism,
and the matrix-free LM against the sparse LM on the reference's fixture
(pipelines/slam/src/bundle/implicit_schur.rs:952-1619,
matrix_free_ba_api_tests.rs:20-158).  No GPU."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import oracle
from visloc_ba import BaConfig, BundleAdjustment, Camera, Pose, SE3, synth
from visloc_ba import _abi
from visloc_ba.problem import quat_to_matrix


# ----------------------------------------------------------- the fixtures
def synthetic_system():
    """synthetic_system (implicit_schur.rs:869-891): two poses, one landmark
    whose first two cross blocks share pose 0 (two sensors of one rig
    frame)."""
    diag = np.array([np.eye(6) * 20.0, np.eye(6) * 22.0])
    r, c = np.meshgrid(np.arange(6), np.arange(3), indexing="ij")
    cross0 = 0.02 * (r + 1.0) * (c + 1.0)
    cross1 = 0.015 * (r + 2.0) * (c + 1.0)
    cross2 = 0.01 * (r + 3.0) * (c + 2.0)
    b_p = 0.03 * np.arange(1, 13, dtype=float)
    h_ll = np.array([np.diag([7.0, 8.0, 9.0])])
    b_l = np.array([[0.2, -0.1, 0.3]])
    return diag, b_p, h_ll, b_l, [[(0, cross0), (0, cross1), (1, cross2)]]


def hand_check_system():
    """hand_check_system (implicit_schur.rs:893-912): B = 10 I, H_ll = 4 I,
    A = [I; 0], two sensors sharing pose 0 and one at pose 1."""
    a = np.zeros((6, 3))
    a[:3, :3] = np.eye(3)
    diag = np.array([np.eye(6) * 10.0, np.eye(6) * 10.0])
    b_p = np.arange(1, 13, dtype=float)
    h_ll = np.array([np.eye(3) * 4.0])
    b_l = np.array([[1.0, 2.0, 3.0]])
    return diag, b_p, h_ll, b_l, [[(0, a), (0, 2.0 * a), (1, -a)]]


def explicit_schur(system, lam):
    """The explicit reduced system of the same blocks (implicit_schur.rs:
    831-867): S = D + lam I - sum_l sum_(a,b) A_a H^-1 A_b^T over every pair
    of a landmark's cross blocks, repeated poses included."""
    diag, b_p, h_ll, b_l, cross = system
    n = 6 * len(diag)
    s = np.zeros((n, n))
    for p, d in enumerate(diag):
        s[6 * p:6 * p + 6, 6 * p:6 * p + 6] = d + lam * np.eye(6)
    for l, cr in enumerate(cross):
        hinv = np.linalg.inv(h_ll[l] + lam * np.eye(3))
        for pa, a in cr:
            for pb, b in cr:
                s[6 * pa:6 * pa + 6, 6 * pb:6 * pb + 6] -= a @ hinv @ b.T
    return s


def explicit_rhs(system, lam):
    diag, b_p, h_ll, b_l, cross = system
    rhs = -np.asarray(b_p, float).copy()
    for l, cr in enumerate(cross):
        hinv = np.linalg.inv(h_ll[l] + lam * np.eye(3))
        for p, a in cr:
            rhs[6 * p:6 * p + 6] += a @ hinv @ b_l[l]
    return rhs


def full_normal_step(system, lam):
    """full_normal_system (implicit_schur.rs:914-950) solved directly: the
    15 x 15 normal equations of two poses and the landmark."""
    diag, b_p, h_ll, b_l, cross = system
    n = 6 * len(diag)
    normal = np.zeros((n + 3, n + 3))
    for p, d in enumerate(diag):
        normal[6 * p:6 * p + 6, 6 * p:6 * p + 6] = d + lam * np.eye(6)
    normal[n:, n:] = h_ll[0] + lam * np.eye(3)
    for p, a in cross[0]:
        normal[6 * p:6 * p + 6, n:] += a
        normal[n:, 6 * p:6 * p + 6] += a.T
    rhs = -np.concatenate([b_p, b_l[0]])
    return np.linalg.solve(normal, rhs)


def run(system, lam, **kw):
    diag, b_p, h_ll, b_l, cross = system
    return oracle.mf_system(diag, b_p, h_ll, b_l, cross, lam, **kw)


# ------------------------------------------------------------- operator
@pytest.mark.parametrize("lam", [0.0, 0.5])
def test_hand_check_fixture_matches_schur_and_full_normal(lam):
    """hand_check_fixture_matches_schur_and_full_normal_for_both_damping_values
    (implicit_schur.rs:1117-1188): the reference's closed-form Schur
    entries and rhs, and the PCG step equal to the full normal solve."""
    sys_ = hand_check_system()
    s = explicit_schur(sys_, lam)
    e_pose0 = 7.75 if lam == 0.0 else 8.5
    e_pose1 = 9.75 if lam == 0.0 else 10.277777777777779
    e_cross = 0.75 if lam == 0.0 else 0.6666666666666666
    # The operator reproduces S column by column.
    cols = np.array([run(sys_, lam, x=np.eye(12)[k])["apply"] for k in range(12)]).T
    assert np.abs(cols - s).max() < 1e-12
    for c in range(3):
        assert abs(cols[c, c] - e_pose0) < 1e-12
        assert abs(cols[6 + c, 6 + c] - e_pose1) < 1e-12
        assert abs(cols[c, 6 + c] - e_cross) < 1e-12
        assert abs(cols[6 + c, c] - e_cross) < 1e-12
    for c in range(3, 6):
        assert abs(cols[c, c] - (10.0 + lam)) < 1e-12
        assert cols[c, 6 + c] == 0.0
    out = run(sys_, lam, solve=True)
    rhs0 = [-0.25, -0.5, -0.75] if lam == 0.0 else [-1 / 3, -2 / 3, -1.0]
    rhs1 = [-7.25, -8.5, -9.75] if lam == 0.0 else [-65 / 9, -76 / 9, -29 / 3]
    assert np.abs(out["rhs"][:3] - rhs0).max() < 1e-12
    assert np.abs(out["rhs"][6:9] - rhs1).max() < 1e-12
    full = full_normal_step(sys_, lam)
    assert out["status"] == oracle.MF_OK
    assert np.linalg.norm(out["solution"] - full[:12]) < 1e-9
    assert np.linalg.norm(out["delta_l"] - full[12:]) < 1e-9


def test_operator_matches_explicit_schur_rhs_preconditioner_and_step():
    """implicit_operator_matches_explicit_schur_rhs_preconditioner_and_step
    (implicit_schur.rs:952-1009), lambda = 0.25."""
    lam = 0.25
    sys_ = synthetic_system()
    s = explicit_schur(sys_, lam)
    x = 0.04 * np.arange(1, 13, dtype=float)
    probe = np.arange(1, 13, dtype=float)
    out = run(sys_, lam, x=x, probe=probe, solve=True)
    assert np.linalg.norm(s @ x - out["apply"]) < 1e-12
    rhs = explicit_rhs(sys_, lam)
    assert np.abs(out["rhs"] - rhs).max() <= 1e-15 * np.abs(rhs).max()
    direct = np.linalg.solve(s, rhs)
    assert out["status"] == oracle.MF_OK
    assert out["residual"] <= out["target"]
    assert np.linalg.norm(out["solution"] - direct) < 1e-9
    diag, b_p, h_ll, b_l, cross = sys_
    hinv = np.linalg.inv(h_ll[0] + lam * np.eye(3))
    dl = hinv @ (-b_l[0] - sum(a.T @ direct[6 * p:6 * p + 6] for p, a in cross[0]))
    assert np.linalg.norm(out["delta_l"] - dl) < 1e-9
    # The pose-0 preconditioner block holds the cross term between the two
    # pose-0 sensor blocks (their sum, not two independent terms).
    g = cross[0][0][1] + cross[0][1][1]
    expected = np.eye(6) * (20.0 + lam) - g @ hinv @ g.T
    want = np.linalg.inv(expected) @ probe[:6]
    assert np.linalg.norm(out["precond"][:6] - want) < 1e-12


def test_operator_without_damping():
    """implicit_operator_matches_explicit_schur_and_direct_step_without_damping
    (implicit_schur.rs:1190-1216)."""
    sys_ = synthetic_system()
    s = explicit_schur(sys_, 0.0)
    x = 0.02 * np.arange(2, 14, dtype=float)
    out = run(sys_, 0.0, x=x, solve=True)
    assert np.linalg.norm(out["apply"] - s @ x) < 1e-10
    direct = np.linalg.solve(s, explicit_rhs(sys_, 0.0))
    assert np.linalg.norm(out["solution"] - direct) < 1e-9


# ------------------------------------------------------------------ PCG
def test_pcg_reports_limits_curvature_and_zero_rhs():
    """pcg_reports_limits_curvature_and_zero_rhs_without_gauge_claim
    (implicit_schur.rs:1456-1568)."""
    sys_ = synthetic_system()
    zero = run(sys_, 0.25, solve=True, rhs=np.zeros(12), max_iterations=0)
    assert zero["status"] == oracle.MF_OK
    assert zero["iterations"] == 0 and zero["residual"] == 0.0
    limited = run(sys_, 0.25, solve=True, max_iterations=0)
    assert limited["status"] == oracle.MF_MAX_ITERATIONS
    # Indefinite: B = 5 I, H_ll = I, A = 2 e_0 e_0^T at both poses; the
    # direction e_0 + e_6 has negative curvature at lambda = 0.
    a = np.zeros((6, 3))
    a[0, 0] = 2.0
    diag = np.array([np.eye(6) * 5.0, np.eye(6) * 5.0])
    ind = (diag, np.zeros(12), np.array([np.eye(3)]), np.zeros((1, 3)), [[(0, a), (1, a)]])
    neg = np.zeros(12)
    neg[0] = neg[6] = 1.0
    out = run(ind, 0.0, solve=True, rhs=neg)
    assert out["status"] == oracle.MF_NON_POSITIVE_CURVATURE


def test_repeated_pcg_runs_are_deterministic():
    """repeated_pcg_runs_are_deterministic (implicit_schur.rs:1619-1629)."""
    sys_ = synthetic_system()
    a = run(sys_, 0.25, solve=True)
    b = run(sys_, 0.25, solve=True)
    assert a["iterations"] == b["iterations"]
    assert np.array_equal(a["solution"], b["solution"])


def test_cluster8_preconditioner_solves_the_same_system():
    """optimize_matrix_free_cluster8's preconditioner (implicit_schur.rs:
    302-376) changes only the iteration count: on the normal equations of a
    ring, the cluster8 and block-Jacobi solutions agree with the explicit
    solve of the same operator and cluster8 needs no more iterations."""
    rng = np.random.default_rng(3)
    npose, nl = 20, 60
    diag = np.array([np.eye(6) * 50.0 + 0.1 * rng.standard_normal((6, 6)) for _ in range(npose)])
    diag = 0.5 * (diag + diag.transpose(0, 2, 1))
    cross, h = [], []
    for _ in range(nl):
        poses = sorted(rng.choice(npose, 4, replace=False))
        cr = [(int(p), rng.standard_normal((6, 3))) for p in poses]
        hm = sum(a.T @ a for _, a in cr) + np.eye(3)
        cross.append(cr)
        h.append(hm)
    sys_ = (diag, rng.standard_normal(6 * npose), np.array(h), rng.standard_normal((nl, 3)), cross)
    s = explicit_schur(sys_, 1e-3)
    direct = np.linalg.solve(s, explicit_rhs(sys_, 1e-3))
    bj = run(sys_, 1e-3, solve=True, max_iterations=500)
    c8 = run(sys_, 1e-3, solve=True, max_iterations=500, cluster8=True)
    assert bj["status"] == oracle.MF_OK and c8["status"] == oracle.MF_OK
    for r in (bj, c8):
        assert np.linalg.norm(r["solution"] - direct) <= 1e-9 * np.linalg.norm(direct)
    assert c8["iterations"] <= bj["iterations"]


# ----------------------------------------------------------- the LM level
def quat_from_euler(roll, pitch, yaw):
    """nalgebra UnitQuaternion::from_euler_angles: Rz(yaw) Ry(pitch) Rx(roll)."""
    cr, sr = math.cos(roll / 2), math.sin(roll / 2)
    cp, sp = math.cos(pitch / 2), math.sin(pitch / 2)
    cy, sy = math.cos(yaw / 2), math.sin(yaw / 2)
    return (cr * cp * cy + sr * sp * sy, sr * cp * cy - cr * sp * sy,
            cr * sp * cy + sr * cp * sy, cr * cp * sy - sr * sp * cy)


def make_problem():
    """make_problem (matrix_free_ba_api_tests.rs:57-115): three poses (pose 0
    fixed at the identity), eight landmarks perturbed off the truth
    (landmark 0 fixed), every landmark seen from every pose."""
    cam = Camera.pinhole(640, 480, 420.0, 418.0, 320.0, 240.0)
    truth = [
        Pose(),
        Pose.from_world_to_camera(quat_from_euler(0.01, -0.02, 0.015), (-0.18, 0.015, 0.02)),
        Pose.from_world_to_camera(quat_from_euler(-0.015, 0.025, -0.01), (-0.34, -0.01, 0.04)),
    ]
    ba = BundleAdjustment(cam)
    ba.add_pose(0, truth[0])
    ba.add_pose(1, Pose.from_world_to_camera(quat_from_euler(0.012, -0.018, 0.016),
                                             (-0.205, 0.022, 0.026)))
    ba.add_pose(2, Pose.from_world_to_camera(quat_from_euler(-0.013, 0.023, -0.012),
                                             (-0.365, -0.004, 0.045)))
    ba.fix_pose(0)
    points = [(-0.8, -0.45, 3.8), (-0.35, 0.55, 4.2), (0.05, -0.25, 4.6), (0.45, 0.35, 5.0),
              (0.85, -0.5, 5.4), (-0.65, 0.25, 5.8), (0.25, 0.7, 6.2), (0.7, 0.15, 6.8)]
    from visloc_ba import BaObservation

    for lid, x in enumerate(points):
        ba.add_landmark(lid, (x[0] + 0.006, x[1] - 0.004, x[2] + 0.008))
        for kf, pose in enumerate(truth):
            xc = pose.transform_world_point(x)
            uv = (420.0 * xc[0] / xc[2] + 320.0, 418.0 * xc[1] / xc[2] + 240.0)
            ba.add_observation(BaObservation(kf, lid, uv))
    ba.fix_landmark(0)
    return ba


def pose_matrix(q, t):
    m = np.eye(4)
    m[:3, :3] = quat_to_matrix(q)
    m[:3, 3] = t
    return m


def test_matrix_free_lm_matches_the_sparse_lm():
    """matrix_free_mono_matches_sparse_cost_and_keeps_anchor_fixed
    (matrix_free_ba_api_tests.rs:127-176): 4 LM iterations, Sparse solver vs
    the matrix-free backend with MatrixFreeBaOptions::default()."""
    ba = make_problem()
    packed, _, _, _ = ba.pack()
    cfg = BaConfig(max_iterations=4)
    direct, mf = packed.copy(), packed.copy()
    st, rd = oracle.optimize(direct, cfg, solver=oracle.SPARSE)
    assert st == _abi.OK
    st, rm, total, failed = oracle.optimize_matrix_free(mf, cfg)
    assert st == _abi.OK
    assert rm.final_cost <= rm.initial_cost and rd.final_cost <= rd.initial_cost
    assert abs(rd.final_cost - rm.final_cost) < 1e-6
    assert failed == 0 and total > 0
    assert np.array_equal(mf.pose_q[0], packed.pose_q[0])
    assert np.array_equal(mf.pose_t[0], packed.pose_t[0])
    for i in (1, 2):
        assert not np.array_equal(mf.pose_q[i], packed.pose_q[i])
        dm = pose_matrix(direct.pose_q[i], direct.pose_t[i]) - pose_matrix(mf.pose_q[i], mf.pose_t[i])
        assert np.linalg.norm(dm) < 1e-5
    assert np.array_equal(mf.landmarks[0], packed.landmarks[0])
    assert np.linalg.norm(direct.landmarks[1:] - mf.landmarks[1:], axis=1).max() < 1e-5
    # Deterministic: the same state and result again.
    again = packed.copy()
    st, ra, total2, _ = oracle.optimize_matrix_free(again, cfg)
    assert ra.final_cost == rm.final_cost and total2 == total
    assert np.array_equal(again.pose_q, mf.pose_q) and np.array_equal(again.landmarks, mf.landmarks)


def test_matrix_free_lm_on_a_street_loop_tracks_the_sparse_lm():
    """On a forward-motion street loop (the C3 geometry at small size), the
    matrix-free LM with a tight PCG tolerance follows the sparse LM: the
    same final cost to 1e-9 relative, on all host threads and on one (the
    tolerance 1e-10: at 1e-12 the true residual of an FP64 solve can stop
    short of the target and the solve fails, as the reference's does)."""
    p = synth.street_loop(120, 6000, seed=23, fixed=(0, 1, 60), track=(10.0, 3, 30),
                          outlier_fraction=0.0)
    cfg = BaConfig(max_iterations=8)
    a, b, c = p.copy(), p.copy(), p.copy()
    st, rs = oracle.optimize(a, cfg, solver=oracle.SPARSE)
    assert st == _abi.OK
    st, rm, _, failed = oracle.optimize_matrix_free(b, cfg, max_pcg_iterations=3000,
                                                    pcg_relative_tolerance=1e-10,
                                                    cluster8=True)
    assert st == _abi.OK and failed == 0
    assert abs(rm.final_cost - rs.final_cost) <= 1e-9 * rs.final_cost
    st, r1, _, _ = oracle.optimize_matrix_free(c, cfg, max_pcg_iterations=3000,
                                               pcg_relative_tolerance=1e-10, cluster8=True,
                                               threads=1)
    assert r1.final_cost == rm.final_cost and np.array_equal(c.pose_q, b.pose_q)


# ------------------------------------------------------- banded direct solve
def test_banded_sparse_solve_matches_the_dense_factorisation():
    """The oracle's Sparse solve in band storage (capture or fold order) on a
    closed street loop gives the dense Cholesky's LM to rounding; a ring,
    whose reduced system is not banded, takes the dense path."""
    p = synth.street_loop(160, 6000, seed=29, fixed=(0, 1, 80), track=(10.0, 3, 30),
                          outlier_fraction=0.0)
    cfg = BaConfig(max_iterations=6)
    a, b = p.copy(), p.copy()
    st, rd = oracle.optimize(a, cfg, solver=oracle.SPARSE)
    assert st == _abi.OK
    st, rb = oracle.optimize(b, cfg, solver=oracle.SPARSE_BANDED)
    assert st == _abi.OK
    assert abs(rb.final_cost - rd.final_cost) <= 1e-12 * rd.final_cost
    assert [i.step_accepted for i in rb.iterations] == [i.step_accepted for i in rd.iterations]
    extent = synth.scene_extent(a)
    assert np.abs(a.camera_centers() - b.camera_centers()).max() <= 1e-12 * extent
    ring = synth.ring_problem(20, 800, seed=5)
    c, d = ring.copy(), ring.copy()
    _, r1 = oracle.optimize(c, BaConfig(max_iterations=3), solver=oracle.SPARSE)
    _, r2 = oracle.optimize(d, BaConfig(max_iterations=3), solver=oracle.SPARSE_BANDED)
    assert r1.final_cost == r2.final_cost
