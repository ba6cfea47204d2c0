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


def cost(packed: PackedProblem, config: BaConfig | None = None, threads: int = 0):
    config = config or BaConfig()
    c = C.c_double()
    n = C.c_uint64()
    st = lib().vlba_oracle_cost(C.byref(packed.abi()), C.byref(config.to_abi()), threads,
                                C.byref(c), C.byref(n))
    if st != 0:
        raise RuntimeError(f"oracle cost failed: {_abi.STATUS_NAMES.get(st, st)}")
    return c.value, n.value


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
