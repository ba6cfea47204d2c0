"""Binding of the CUDA solver's C ABI and the accelerator plug-in.

`GpuBundleAdjuster` mirrors the reference's plug-in
(crates/ba-gpu/src/solver.rs:80-85 and its `impl BaAccelerator`, :729-742):
`optimize(ba, config, scope)` returns None when it declines (the caller then
runs its CPU solver) and raises BaError for the reference's error variants.
"""

from __future__ import annotations

import copy
import ctypes as C
import os
import time
from dataclasses import dataclass

from . import _abi
from .problem import (
    BaConfig,
    BaError,
    BaGncResult,
    BaResult,
    BaScope,
    BundleAdjustment,
    GncConfig,
    PackedProblem,
    result_from_abi,
)

_ERROR_KIND = {
    _abi.ERR_NO_POSES: "NoPoses",
    _abi.ERR_NO_LANDMARKS: "NoLandmarks",
    _abi.ERR_NO_OBSERVATIONS: "NoObservations",
    _abi.ERR_ALL_POSES_FIXED: "AllPosesFixed",
    _abi.ERR_MISSING_POSE: "MissingPose",
    _abi.ERR_MISSING_LANDMARK: "MissingLandmark",
    _abi.ERR_UNSUPPORTED_CAMERA_MODEL: "UnsupportedCameraModel",
    _abi.ERR_SINGULAR_SYSTEM: "SingularSystem",
    _abi.ERR_MISSING_STEREO_BASELINE: "MissingStereoBaseline",
}


class SolverError(RuntimeError):
    """A non-BaError failure of the CUDA library (CUDA error, timeout...)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")


class CudaSolver:
    """One solver context (device memory, stream) of libvisloc_ba_cuda.so."""

    def __init__(self, device: int = 0, library: str | None = None):
        self.lib = _abi.load_solver_library(library)
        self.ctx = self.lib.visloc_ba_cuda_create(int(device))
        if not self.ctx:
            raise RuntimeError(
                "visloc_ba_cuda_create failed: no CUDA device of compute capability 10.x"
            )

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.visloc_ba_cuda_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def last_error(self) -> str:
        return self.lib.visloc_ba_cuda_last_error(self.ctx).decode()

    def _iters(self, config: BaConfig):
        cap = max(1, int(config.max_iterations))
        return (_abi.Iteration * cap)(), cap

    def optimize(self, packed: PackedProblem, config: BaConfig):
        """LM solve in place on `packed`.  Returns (status, BaResult|None)."""
        prob = packed.abi()
        cfg = config.to_abi()
        res = _abi.Result()
        iters, cap = self._iters(config)
        st = self.lib.visloc_ba_cuda_optimize(self.ctx, C.byref(prob), C.byref(cfg),
                                              C.byref(res), iters, cap)
        if st != _abi.OK:
            return st, res
        return st, result_from_abi(res, iters, res.num_iterations)

    def optimize_gnc(self, packed: PackedProblem, config: BaConfig, gnc: GncConfig | None = None):
        """BundleAdjustment::optimize_gnc (bundle/lm.rs:28-142) in place on
        `packed` (which must carry no weights of its own).  Returns (status,
        BaGncResult | None); the weights are in the problem's observation
        order, NaN where an observation cannot be evaluated."""
        import numpy as np

        gnc = gnc or GncConfig()
        res = _abi.GncResult()
        w = np.empty(packed.num_observations)
        st = self.lib.visloc_ba_cuda_optimize_gnc(
            self.ctx, C.byref(packed.abi()), C.byref(config.to_abi()), C.byref(gnc.to_abi()),
            C.byref(res), w.ctypes.data_as(C.POINTER(C.c_double)))
        if st != _abi.OK:
            return st, None
        return st, BaGncResult(res.initial_cost, res.final_cost, res.inlier_cost, res.inlier_scale,
                               int(res.observation_count), int(res.outer_iterations),
                               bool(res.converged), w, int(res.lm_iterations), res.device_ms)

    def upload(self, packed: PackedProblem, config: BaConfig) -> int:
        return self.lib.visloc_ba_cuda_upload(self.ctx, C.byref(packed.abi()),
                                              C.byref(config.to_abi()))

    def solve_uploaded(self, config: BaConfig | None = None):
        res = _abi.Result()
        cfg = config or BaConfig()
        iters, cap = self._iters(cfg)
        cfg_ptr = C.byref(config.to_abi()) if config is not None else None
        st = self.lib.visloc_ba_cuda_solve_uploaded(self.ctx, cfg_ptr, C.byref(res), iters, cap)
        if st != _abi.OK:
            return st, res
        return st, result_from_abi(res, iters, res.num_iterations)

    def download(self, packed: PackedProblem) -> int:
        return self.lib.visloc_ba_cuda_download(self.ctx, C.byref(packed.abi()))

    # ------------------------------------------------------ reduced solve
    def reduced_solve(self, diag, edges, offdiag, rhs, tol: float, max_iterations: int,
                      clusters=None, coarse=None):
        """ReducedSolveAccelerator::solve on a reduced camera system
        (ReducedCameraSystem, pipelines/slam/src/ba_accel.rs:50-72): diag
        (n,6,6) damped diagonal blocks, edges (e,2) sorted (a, b) with a < b,
        offdiag (e,6,6) the (row b, column a) blocks, rhs (n,6); clusters a
        list of (first node, inverse (6m,6m)) over runs of consecutive nodes,
        coarse (nodes per aggregate, leading nodes covered, inverse (6m,6m)).
        Without either: block-Jacobi through the persistent PCG kernel.
        Returns (x (n,6), iterations, relative residual); a breakdown raises
        SolverError with status DECLINED, as pcg_core returns None."""
        import numpy as np

        diag = np.ascontiguousarray(np.asarray(diag, np.float64).transpose(0, 2, 1))  # column-major
        # offdiag None: the blocks of the last reduced_eliminate of these edges.
        off = None if offdiag is None else np.ascontiguousarray(
            np.asarray(offdiag, np.float32).reshape(-1, 6, 6).transpose(0, 2, 1))
        edges = np.ascontiguousarray(np.asarray(edges, np.uint32).reshape(-1, 2))
        rhs = np.ascontiguousarray(np.asarray(rhs, np.float64).reshape(-1, 6))
        n = diag.shape[0]
        sysm = _abi.ReducedSystem()
        sysm.num_nodes = n
        sysm.num_edges = edges.shape[0]
        sysm.diag = diag.ctypes.data_as(C.POINTER(C.c_double))
        sysm.edges = edges.ctypes.data_as(C.POINTER(C.c_uint32))
        sysm.offdiag = (C.POINTER(C.c_float)() if off is None
                        else off.ctypes.data_as(C.POINTER(C.c_float)))
        sysm.rhs = rhs.ctypes.data_as(C.POINTER(C.c_double))
        sysm.tol = float(tol)
        sysm.max_iterations = int(max_iterations)
        x = np.zeros((n, 6))
        it = C.c_uint32()
        rr = C.c_double()
        xp = x.ctypes.data_as(C.POINTER(C.c_double))
        t0 = time.perf_counter()
        if clusters is None and coarse is None:
            st = self.lib.visloc_ba_cuda_reduced_solve(self.ctx, C.byref(sysm), xp,
                                                       C.byref(it), C.byref(rr))
        else:
            pre = _abi.ReducedPreconditioner()
            keep = []
            if clusters:
                for _, inv in clusters:
                    sh = np.shape(inv)
                    if len(sh) != 2 or sh[0] != sh[1] or sh[0] % 6:
                        raise ValueError(f"cluster inverse of shape {sh}")
                first = np.ascontiguousarray([c[0] for c in clusters], np.uint32)
                size = np.ascontiguousarray([np.asarray(c[1]).shape[0] // 6 for c in clusters],
                                            np.uint32)
                # nalgebra's DMatrix is column-major.
                inv = np.ascontiguousarray(np.concatenate(
                    [np.asarray(c[1], np.float64).T.reshape(-1) for c in clusters]))
                keep += [first, size, inv]
                pre.num_clusters = len(clusters)
                pre.cluster_first = first.ctypes.data_as(C.POINTER(C.c_uint32))
                pre.cluster_size = size.ctypes.data_as(C.POINTER(C.c_uint32))
                pre.cluster_inverse = inv.ctypes.data_as(C.POINTER(C.c_double))
            if coarse is not None:
                group, nodes, cinv = coarse
                m = -(-int(nodes) // int(group)) if int(group) > 0 else 0
                if np.shape(cinv) != (6 * m, 6 * m):
                    raise ValueError(f"coarse inverse of shape {np.shape(cinv)} for "
                                     f"{nodes} nodes in groups of {group}")
                cinv = np.ascontiguousarray(np.asarray(cinv, np.float64).T)
                keep.append(cinv)
                pre.coarse_group = int(group)
                pre.coarse_nodes = int(nodes)
                pre.coarse_inverse = cinv.ctypes.data_as(C.POINTER(C.c_double))
            t0 = time.perf_counter()
            st = self.lib.visloc_ba_cuda_reduced_solve_preconditioned(
                self.ctx, C.byref(sysm), C.byref(pre), xp, C.byref(it), C.byref(rr))
        # Wall time of the C call alone (the conversions above excluded).
        self.last_call_ms = (time.perf_counter() - t0) * 1e3
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        return x, it.value, rr.value

    def reduced_eliminate(self, structure_id: int, linearization_id: int, num_nodes: int,
                          edges, point_off, point_nodes, hcp, point_inverse, extra=(),
                          run_edges=(), coarse=None):
        """ReducedSolveAccelerator::eliminate (PointElimination,
        pipelines/slam/src/ba_accel.rs:74-130): edges (e,2) sorted (s, t),
        point_off (P+1), point_nodes, hcp (K,6,3) per (point, node),
        point_inverse a list of (3,3) damped point inverses or None (point
        left out), extra a list of (edge, (6,6) block), run_edges, coarse
        (nodes per aggregate, leading nodes covered) or None.  The blocks stay
        on the device for reduced_solve(..., offdiag=None).  Returns
        (run_blocks (len(run_edges),6,6), coarse_sums (m*m,6,6) or None);
        a non-finite block raises SolverError with status DECLINED."""
        import numpy as np

        edges = np.ascontiguousarray(np.asarray(edges, np.uint32).reshape(-1, 2))
        point_off = np.ascontiguousarray(np.asarray(point_off, np.uint64))
        point_nodes = np.ascontiguousarray(np.asarray(point_nodes, np.uint32))
        hcp = np.ascontiguousarray(np.asarray(hcp, np.float64).reshape(-1, 6, 3).transpose(0, 2, 1))
        npts = len(point_off) - 1
        if isinstance(point_inverse, np.ndarray):  # (P,3,3), every point used
            used = np.ones(npts, np.uint8)
            vinv = np.ascontiguousarray(np.asarray(point_inverse, np.float64).transpose(0, 2, 1))
        else:
            used = np.ascontiguousarray([v is not None for v in point_inverse], np.uint8)
            vinv = np.zeros((npts, 3, 3))
            for p, v in enumerate(point_inverse):
                if v is not None:
                    vinv[p] = np.asarray(v, np.float64).T  # column-major
            vinv = np.ascontiguousarray(vinv)
        ex_edge = np.ascontiguousarray([int(e) for e, _ in extra], np.uint32)
        ex_blk = np.ascontiguousarray(
            np.array([np.asarray(b, np.float64).T for _, b in extra]).reshape(-1, 36))
        run_edges = np.ascontiguousarray(np.asarray(run_edges, np.uint32).reshape(-1))
        el = _abi.PointElimination()
        el.structure_id = int(structure_id)
        el.linearization_id = int(linearization_id)
        el.num_nodes = int(num_nodes)
        el.num_points = npts
        el.num_edges = edges.shape[0]
        el.edges = edges.ctypes.data_as(C.POINTER(C.c_uint32))
        el.point_off = point_off.ctypes.data_as(C.POINTER(C.c_uint64))
        el.point_nodes = point_nodes.ctypes.data_as(C.POINTER(C.c_uint32))
        el.hcp = hcp.ctypes.data_as(C.POINTER(C.c_double))
        el.point_inverse = vinv.ctypes.data_as(C.POINTER(C.c_double))
        el.point_used = used.ctypes.data_as(C.POINTER(C.c_uint8))
        el.num_extra = len(ex_edge)
        el.extra_edge = ex_edge.ctypes.data_as(C.POINTER(C.c_uint32))
        el.extra_block = ex_blk.ctypes.data_as(C.POINTER(C.c_double))
        el.num_run_edges = len(run_edges)
        el.run_edges = run_edges.ctypes.data_as(C.POINTER(C.c_uint32))
        m = 0
        if coarse is not None:
            el.coarse_group, el.coarse_nodes = int(coarse[0]), int(coarse[1])
            m = -(-int(coarse[1]) // int(coarse[0])) if int(coarse[0]) > 0 else 0
        run_out = np.zeros((len(run_edges), 36))
        sums = np.zeros((m * m, 36)) if m else None
        t0 = time.perf_counter()
        st = self.lib.visloc_ba_cuda_reduced_eliminate(
            self.ctx, C.byref(el), run_out.ctypes.data_as(C.POINTER(C.c_double)),
            sums.ctypes.data_as(C.POINTER(C.c_double)) if sums is not None
            else C.POINTER(C.c_double)())
        self.last_call_ms = (time.perf_counter() - t0) * 1e3
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        unpack = lambda a: a.reshape(-1, 6, 6).transpose(0, 2, 1).copy()  # noqa: E731
        return unpack(run_out), (unpack(sums) if sums is not None else None)

    def reduced_timing(self) -> dict:
        """Device times (ms) of the last reduced solve and elimination:
        fill_ms, pcg_ms, eliminate_ms."""
        t = _abi.ReducedTiming()
        st = self.lib.visloc_ba_cuda_reduced_timing(self.ctx, C.byref(t))
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        return {"fill_ms": t.fill_ms, "pcg_ms": t.pcg_ms, "eliminate_ms": t.eliminate_ms}

    def wait_probe(self, limit_ms: float):
        """(status, waited ms) of the bounded-wait self-test."""
        waited = C.c_double()
        st = self.lib.visloc_ba_cuda_wait_probe(self.ctx, float(limit_ms), C.byref(waited))
        return st, waited.value

    # ---------------------------------------------------------- autotuner
    def autotune(self) -> dict:
        """Time candidate launch shapes on the uploaded system; apply and
        return the fastest."""
        sh = _abi.LaunchShape()
        st = self.lib.visloc_ba_cuda_autotune(self.ctx, C.byref(sh))
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        return {"pcg_blocks": sh.pcg_blocks, "l2_resident_fraction": sh.l2_resident_fraction,
                "pcg_iteration_us": sh.pcg_iteration_us}

    def set_launch_shape(self, pcg_blocks: int, l2_resident_fraction: float) -> None:
        sh = _abi.LaunchShape(int(pcg_blocks), 0, float(l2_resident_fraction), 0.0)
        st = self.lib.visloc_ba_cuda_set_launch_shape(self.ctx, C.byref(sh))
        if st != _abi.OK:
            raise SolverError(st, self.last_error())

    # ------------------------------------------------------------ batches
    def _batch_arrays(self, problems, configs):
        n = len(problems)
        if isinstance(configs, BaConfig):
            configs = [configs] * n
        probs = [p.abi() for p in problems]
        cfgs = [c.to_abi() for c in configs]
        pp = (C.POINTER(_abi.Problem) * n)(*[C.pointer(x) for x in probs])
        cp = (C.POINTER(_abi.Config) * n)(*[C.pointer(x) for x in cfgs])
        cap = max(1, max(int(c.max_iterations) for c in configs)) if n else 1
        self._batch_keep = (probs, cfgs, pp, cp)
        self._batch_n, self._batch_cap = n, cap
        return n, pp, cp, cap

    def _batch_results(self, res, iters, statuses, n, cap):
        out = []
        for i in range(n):
            if statuses is not None and statuses[i] != _abi.OK:
                out.append(None)
                continue
            row = (_abi.Iteration * cap).from_buffer(iters, i * cap * C.sizeof(_abi.Iteration))
            out.append(result_from_abi(res[i], row, res[i].num_iterations))
        return out

    def batch_upload(self, problems, configs):
        """Upload a batch (configs: one BaConfig or one per problem).  Returns
        the per-problem validation statuses; raises SolverError if none is
        left."""
        n, pp, cp, _ = self._batch_arrays(problems, configs)
        statuses = (C.c_int * n)()
        st = self.lib.visloc_ba_cuda_batch_upload(self.ctx, n, pp, cp, statuses)
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        self._batch_statuses = list(statuses)
        return list(statuses)

    def batch_solve_uploaded(self):
        """Solve the uploaded batch from its initial state: list of BaResult
        (None for problems left out)."""
        n, cap = self._batch_n, self._batch_cap
        res = (_abi.Result * n)()
        iters = (_abi.Iteration * (n * cap))()
        st = self.lib.visloc_ba_cuda_batch_solve_uploaded(self.ctx, res, iters, cap)
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        return self._batch_results(res, iters, self._batch_statuses, n, cap)

    def batch_download(self, problems) -> None:
        n = len(problems)
        probs = [p.abi() for p in problems]
        pp = (C.POINTER(_abi.Problem) * n)(*[C.pointer(x) for x in probs])
        st = self.lib.visloc_ba_cuda_batch_download(self.ctx, n, pp)
        if st != _abi.OK:
            raise SolverError(st, self.last_error())

    def batch_optimize(self, problems, configs):
        """Solve a batch in place: (statuses, [BaResult | None])."""
        n, pp, cp, cap = self._batch_arrays(problems, configs)
        statuses = (C.c_int * n)()
        res = (_abi.Result * n)()
        iters = (_abi.Iteration * (n * cap))()
        st = self.lib.visloc_ba_cuda_batch_optimize(self.ctx, n, pp, cp, statuses, res, iters, cap)
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        return list(statuses), self._batch_results(res, iters, list(statuses), n, cap)

    def linear_step(self, packed: PackedProblem, config: BaConfig, lam: float):
        """One damped step at the current state: (dp (6 per variable pose),
        dl (3 per variable landmark), PCG iterations, PCG relative residual)."""
        import numpy as np

        npv = int(packed.num_poses - (0 if packed.pose_fixed is None else packed.pose_fixed.sum()))
        nlv = int(packed.num_landmarks
                  - (0 if packed.landmark_fixed is None else packed.landmark_fixed.sum()))
        dp = np.zeros(6 * npv)
        dl = np.zeros(3 * nlv)
        it = C.c_uint32()
        rr = C.c_double()
        st = self.lib.visloc_ba_cuda_linear_step(
            self.ctx, C.byref(packed.abi()), C.byref(config.to_abi()), float(lam),
            dp.ctypes.data_as(C.POINTER(C.c_double)), dl.ctypes.data_as(C.POINTER(C.c_double)),
            C.byref(it), C.byref(rr))
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        return dp, dl, it.value, rr.value

    def reduced_system(self, packed: PackedProblem, config: BaConfig, lam: float):
        """The assembled damped reduced system (S dense, rhs) at the state."""
        import numpy as np

        npv = int(packed.num_poses - (0 if packed.pose_fixed is None else packed.pose_fixed.sum()))
        s = np.zeros((6 * npv, 6 * npv))
        rhs = np.zeros(6 * npv)
        st = self.lib.visloc_ba_cuda_reduced_system(
            self.ctx, C.byref(packed.abi()), C.byref(config.to_abi()), float(lam),
            s.ctypes.data_as(C.POINTER(C.c_double)), rhs.ctypes.data_as(C.POINTER(C.c_double)))
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        return s, rhs

    def cost(self, packed: PackedProblem, config: BaConfig | None = None):
        config = config or BaConfig()
        c = C.c_double()
        n = C.c_uint64()
        st = self.lib.visloc_ba_cuda_cost(self.ctx, C.byref(packed.abi()),
                                          C.byref(config.to_abi()), C.byref(c), C.byref(n))
        if st != _abi.OK:
            raise SolverError(st, self.last_error())
        return c.value, n.value


def check(packed: PackedProblem, config: BaConfig | None = None):
    """Validation only (no device needed): (status, error_index)."""
    lib = _abi.load_solver_library()
    idx = C.c_uint64()
    st = lib.visloc_ba_cuda_check(C.byref(packed.abi()), C.byref((config or BaConfig()).to_abi()),
                                  C.byref(idx))
    return st, idx.value


def plan(packed: PackedProblem, config: BaConfig | None = None, pcg_iterations: float = 40.0):
    """Host-only device layout of a problem (no device needed): (status, PlanInfo)."""
    lib = _abi.load_solver_library()
    info = _abi.PlanInfo()
    st = lib.visloc_ba_cuda_plan(C.byref(packed.abi()), C.byref((config or BaConfig()).to_abi()),
                                 float(pcg_iterations), C.byref(info))
    return st, info


def _env_num(name, cast, default):
    try:
        return cast(os.environ[name])
    except (KeyError, ValueError):
        return default


@dataclass
class GpuBaSettings:
    """PCG controls of each LM linear solve (solver.rs:25-50)."""

    max_pcg_iterations: int = 100
    pcg_relative_tolerance: float = 1e-4
    local_windows: bool = False

    @staticmethod
    def from_env() -> "GpuBaSettings":
        return GpuBaSettings(
            _env_num("VISLOC_BA_GPU_PCG_ITERS", int, 100),
            _env_num("VISLOC_BA_GPU_PCG_TOL", float, 1e-4),
            "VISLOC_BA_GPU_LOCAL" in os.environ,
        )


class GpuBundleAdjuster:
    """The BaAccelerator of this solver (drop-in for crates/ba-gpu)."""

    def __init__(self, device: int = 0, settings: GpuBaSettings | None = None):
        self.solver = CudaSolver(device)
        self.settings = settings or GpuBaSettings.from_env()

    def _config(self, config: BaConfig) -> BaConfig:
        cfg = copy.copy(config)
        cfg.max_pcg_iterations = self.settings.max_pcg_iterations
        cfg.pcg_relative_tolerance = self.settings.pcg_relative_tolerance
        return cfg

    def solve(self, ba: BundleAdjustment, config: BaConfig, observation_weights=None) -> BaResult:
        """BundleAdjustment::optimize semantics: mutate `ba`, return BaResult,
        raise BaError.  Raises SolverError when the library declines.  With
        `observation_weights` (one per observation, in the problem's
        observation order), the semantics of
        optimize_with_observation_weights (optimize.rs:43-53, 628-650)."""
        packed, pose_ids, lm_ids, missing = ba.pack()
        if observation_weights is not None:
            import numpy as np

            w = np.ascontiguousarray(observation_weights, dtype=np.float64).reshape(-1)
            expected = len(ba.observations) + len(ba.rig_observations)
            if w.shape[0] != expected:
                raise BaError("ObservationWeightCount",
                              message=f"expected {expected}, got {w.shape[0]}")
            packed.obs_weight = w
        cfg = self._config(config)
        st, res = self.solver.optimize(packed, cfg)
        if st == _abi.ERR_INVALID_OBSERVATION_WEIGHT:
            raise BaError("InvalidObservationWeight", int(res.error_index))
        if st in (_abi.ERR_MISSING_POSE, _abi.ERR_MISSING_LANDMARK) and missing is not None:
            raise missing
        if st in _ERROR_KIND:
            raise BaError(_ERROR_KIND[st])
        if st != _abi.OK:
            raise SolverError(st, self.solver.last_error())
        ba.unpack(packed, pose_ids, lm_ids)
        return res

    def optimize_with_observation_weights(self, ba: BundleAdjustment, config: BaConfig,
                                          observation_weights) -> BaResult:
        """BundleAdjustment::optimize_with_observation_weights (optimize.rs:43-53)
        on the device: each weight multiplies its observation's robust IRLS
        weight and robust cost."""
        return self.solve(ba, config, observation_weights)

    def optimize_gnc(self, ba: BundleAdjustment, config: BaConfig,
                     gnc: GncConfig | None = None) -> BaGncResult:
        """BundleAdjustment::optimize_gnc (bundle/lm.rs:28-142) on the device:
        mutates `ba`; the weights follow the problem's observation order."""
        packed, pose_ids, lm_ids, missing = ba.pack()
        st, res = self.solver.optimize_gnc(packed, self._config(config), gnc)
        if st in (_abi.ERR_MISSING_POSE, _abi.ERR_MISSING_LANDMARK) and missing is not None:
            raise missing
        if st in _ERROR_KIND:
            raise BaError(_ERROR_KIND[st])
        if st != _abi.OK:
            raise SolverError(st, self.solver.last_error())
        ba.unpack(packed, pose_ids, lm_ids)
        return res

    def optimize(self, ba: BundleAdjustment, config: BaConfig, scope: BaScope = BaScope.GLOBAL):
        """BaAccelerator::optimize: None = declined (run the CPU solver).
        Declined: local windows unless enabled (solver.rs:29-33); priors, the
        inertial state and rotation-fixed poses, which the device solver does
        not model (solver.rs:230-246); and, in the library, joint intrinsics
        refinement (solver.rs:214-216)."""
        if scope == BaScope.LOCAL and not self.settings.local_windows:
            return None
        if ba.unsupported_terms() is not None:
            return None
        try:
            return self.solve(ba, config)
        except SolverError as e:
            if e.status == _abi.DECLINED:
                return None
            raise


class BaServer:
    """The request loop of libvisloc_ba_cuda.so (visloc_ba_cuda_server_*):
    submit problems from any thread, wait for their results.  A submitted
    problem's arrays are written in place when its ticket completes; the
    server keeps the problem (and its config) alive until then."""

    def __init__(self, device: int = 0, slots: int = 3, memory_bytes: int = 0,
                 max_batch: int = 64, library: str | None = None):
        self.lib = _abi.load_solver_library(library)
        self.srv = self.lib.visloc_ba_cuda_server_create(int(device), int(slots),
                                                          int(memory_bytes), int(max_batch))
        if not self.srv:
            raise RuntimeError("visloc_ba_cuda_server_create failed")
        self._live = {}

    def submit(self, packed: PackedProblem, config: BaConfig) -> int:
        prob = packed.abi()
        cfg = config.to_abi()
        ticket = C.c_uint64()
        st = self.lib.visloc_ba_cuda_server_submit(self.srv, C.byref(prob), C.byref(cfg),
                                                   C.byref(ticket))
        if st != _abi.OK:
            raise SolverError(st, "submit")
        self._live[ticket.value] = (packed, prob, cfg, max(1, int(config.max_iterations)))
        return ticket.value

    def wait(self, ticket: int, timeout_ms: float = -1.0):
        """(status, BaResult | None, info dict); status BUSY if not done."""
        packed, prob, cfg, cap = self._live[ticket]
        res = _abi.Result()
        iters = (_abi.Iteration * cap)()
        info = _abi.TicketInfo()
        st = self.lib.visloc_ba_cuda_server_wait(self.srv, ticket, float(timeout_ms),
                                                 C.byref(res), iters, cap, C.byref(info))
        if st == _abi.ERR_BUSY:
            return st, None, None
        del self._live[ticket]
        meta = {"latency_ms": info.latency_ms, "queue_ms": info.queue_ms,
                "solve_ms": info.solve_ms, "batch_size": info.batch_size, "slot": info.slot}
        if st != _abi.OK:
            return st, None, meta
        return st, result_from_abi(res, iters, res.num_iterations), meta

    def last_error(self) -> str:
        return self.lib.visloc_ba_cuda_server_last_error(self.srv).decode()

    def close(self):
        if getattr(self, "srv", None):
            self.lib.visloc_ba_cuda_server_destroy(self.srv)
            self.srv = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
