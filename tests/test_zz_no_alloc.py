"""visloc_ba_cuda_cost_noalloc: the robust cost without any device allocation.

The entry point serves callers that cannot allocate device memory when they
need a cost -- a tracking thread with a frame deadline, where cudaMalloc and
cudaFree may synchronise the device and stall it, or a process whose device
memory belongs to another allocator.  Their problem arrays are already on the
device; the library evaluates the cost there with a fixed scratch array of its
own.  These tests hold it to visloc_ba_cuda_cost (which builds its own device
copy of the problem) within that entry point's tolerance against the oracle,
on calls made back to back so that each call meets the scratch contents the
previous one left.

The file name puts it last in collection order: a run that stops at the first
failure has run every other test before this one.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from _scenes import general_stereo_window_packed, mixed_stereo_window_packed, stereo_window_packed
from visloc_ba import BaConfig, Camera, CameraModel, PackedProblem, RobustKernel, synth
from visloc_ba import _abi

COST_RTOL = 1e-12  # the cost tolerance of the GPU-vs-oracle cost test
MAX_OBS = 16777216  # VLBA_NOALLOC_MAX_OBSERVATIONS


class DeviceProblem:
    """A PackedProblem's arrays copied into device memory (by torch, on the
    test's side: the entry point under test allocates nothing itself).  Every
    array field of the problem is copied; one left on the host would hand the
    kernel a host pointer, so an array field this helper does not know fails
    here instead."""

    ARRAYS = {
        "pose_q": C.c_double, "pose_t": C.c_double, "landmarks": C.c_double,
        "obs_pose": C.c_uint32, "obs_landmark": C.c_uint32, "obs_xy": C.c_double,
        "obs_camera": C.c_uint32, "obs_weight": C.c_double, "obs_kind": C.c_uint8,
        "obs_stereo": C.c_double, "obs_right_camera": C.c_uint32,
    }
    # Read on the host (cameras) or ignored by the entry point (fixed flags).
    HOST = {"cameras", "pose_fixed", "landmark_fixed"}

    def __init__(self, packed: PackedProblem):
        import torch

        self.packed = packed
        self.keep = []
        p = packed.abi()  # host cameras; array fields replaced below
        pointer_fields = {name for name, t in _abi.Problem._fields_
                          if issubclass(t, C._Pointer)}
        assert pointer_fields == set(self.ARRAYS) | self.HOST, pointer_fields
        for name, ctype in self.ARRAYS.items():
            a = getattr(packed, name)
            if a is None:
                assert not getattr(p, name), name
                continue
            t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
            self.keep.append(t)
            setattr(p, name, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ctype)))
        self.abi = p
        self.cost = torch.empty(1, dtype=torch.float64, device="cuda")
        self.counts = torch.empty(2, dtype=torch.int64, device="cuda")


def noalloc_cost(lib, dp: DeviceProblem, cfg: BaConfig):
    import torch

    dp.cost.fill_(float("nan"))
    dp.counts.fill_(-1)
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.visloc_ba_cuda_cost_noalloc(
        C.byref(dp.abi), C.byref(cfg.to_abi()), C.c_void_p(stream),
        C.c_void_p(dp.cost.data_ptr()), C.c_void_p(dp.counts.data_ptr()), err, len(err))
    assert st == _abi.OK, err.value.decode()
    torch.cuda.current_stream().synchronize()
    counts = dp.counts.cpu().numpy()
    return float(dp.cost.cpu().item()), int(counts[0]), int(counts[1])


def problems():
    shared = synth.ring_problem(40, 4000, seed=2, width=2000, height=1500, focal=(1500, 1500),
                                k1=(0.0, 0.0), per_camera_intrinsics=False,
                                track=("geometric", 8.0, 2, 40))
    return [
        ("ring-12-per-camera-radial", synth.ring_problem(12, 1500, seed=71)),
        ("ring-40-shared-pinhole", shared),
        ("stereo-rig-window", synth.stereo_window(20, 1500, seed=6)),
        ("rectified-stereo-window", stereo_window_packed(seed=7, cams=16, points=1200)),
        ("general-stereo-window", general_stereo_window_packed(seed=8, cams=16, points=1200)),
        ("mono-and-rectified-window", mixed_stereo_window_packed(seed=9, cams=16, points=1200)[0]),
        ("pose-only", synth.pose_only(800, seed=4)),
    ]


KERNELS = [RobustKernel.none(), RobustKernel.huber(1.0), RobustKernel.cauchy(2.0)]


@pytest.mark.gpu
def test_matches_the_allocating_cost_on_calls_in_a_row(solver):
    lib = solver.lib
    cases = [(name, DeviceProblem(p)) for name, p in problems()]
    # Back to back: each problem twice, then the next one (a smaller problem
    # after a larger one meets the larger one's partials in the scratch).
    for kernel in KERNELS:
        cfg = BaConfig(robust_kernel=kernel)
        for name, dp in cases:
            want, want_bad = solver.cost(dp.packed, cfg)
            for _ in range(2):
                got, bad, invalid = noalloc_cost(lib, dp, cfg)
                assert invalid == 0, name
                assert bad == want_bad, name
                assert got == pytest.approx(want, rel=COST_RTOL), (name, got, want)


@pytest.mark.gpu
def test_out_of_range_indices_are_counted_and_skipped(solver):
    """Where visloc_ba_cuda_cost rejects the whole problem, this entry point
    counts the offending observation as invalid and skips it: a pose,
    landmark or camera index out of range, a NaN or infinite weight."""
    lib = solver.lib
    p = synth.ring_problem(12, 800, seed=72)
    cfg = BaConfig(robust_kernel=RobustKernel.huber(1.0))
    rng = np.random.default_rng(5)
    w = rng.uniform(0.5, 1.5, p.num_observations)
    broken = PackedProblem(p.pose_q, p.pose_t, p.landmarks, p.obs_pose.copy(),
                           p.obs_landmark.copy(), p.obs_xy, p.cameras, p.pose_fixed,
                           p.landmark_fixed, p.obs_camera.copy(), w.copy())
    broken.obs_pose[5] = p.num_poses
    broken.obs_landmark[17] = p.num_landmarks + 3
    broken.obs_camera[31] = len(p.cameras)
    broken.obs_weight[23] = np.nan
    broken.obs_weight[40] = np.inf
    bad_rows = [5, 17, 23, 31, 40]
    keep = np.ones(p.num_observations, bool)
    keep[bad_rows] = False
    trimmed = PackedProblem(p.pose_q, p.pose_t, p.landmarks, p.obs_pose[keep],
                            p.obs_landmark[keep], p.obs_xy[keep], p.cameras, p.pose_fixed,
                            p.landmark_fixed, p.obs_camera[keep], w[keep])
    want, want_bad = solver.cost(trimmed, cfg)
    dp = DeviceProblem(broken)
    for _ in range(2):
        got, bad, invalid = noalloc_cost(lib, dp, cfg)
        assert invalid == len(bad_rows) and bad == want_bad
        assert got == pytest.approx(want, rel=COST_RTOL)


@pytest.mark.gpu
def test_unusable_stereo_observations_are_counted_and_skipped(solver):
    """Rectified stereo observations without a usable baseline (0, negative,
    NaN), or with a cameras[0] outside the pinhole models, are counted as
    invalid and skipped; the monocular observations of the same problem are
    still summed, to the cost visloc_ba_cuda_cost gives for them alone."""
    lib = solver.lib
    cfg = BaConfig(robust_kernel=RobustKernel.cauchy(2.0))
    mixed, mono = mixed_stereo_window_packed(seed=10, cams=16, points=1200)
    n_stereo = int((mixed.obs_kind == _abi.OBS_STEREO).sum())
    assert 0 < n_stereo < mixed.num_observations
    want, want_bad = solver.cost(mono, cfg)
    for baseline in (0.0, -0.11, float("nan")):
        q = mixed.copy()
        q.stereo_baseline = baseline
        dp = DeviceProblem(q)
        for _ in range(2):
            got, bad, invalid = noalloc_cost(lib, dp, cfg)
            assert invalid == n_stereo and bad == want_bad
            assert got == pytest.approx(want, rel=COST_RTOL)
    left = mixed.cameras[0][0]
    radial = Camera(CameraModel.SIMPLE_RADIAL, left.width, left.height,
                    [left.params[0], left.params[2], left.params[3], 0.02])
    mixed_r, mono_r = mixed_stereo_window_packed(seed=10, cams=16, points=1200, camera=radial)
    want, want_bad = solver.cost(mono_r, cfg)
    dp = DeviceProblem(mixed_r)
    for _ in range(2):
        got, bad, invalid = noalloc_cost(lib, dp, cfg)
        assert invalid == n_stereo and bad == want_bad
        assert got == pytest.approx(want, rel=COST_RTOL)


@pytest.mark.gpu
def test_external_weights_match_the_allocating_cost(solver):
    """Per-observation weights (device array): the same weighted cost as
    visloc_ba_cuda_cost; a negative weight is counted and its observation
    skipped."""
    lib = solver.lib
    p = synth.stereo_window(20, 1500, seed=6)
    rng = np.random.default_rng(11)
    p.obs_weight = rng.uniform(0.0, 2.0, p.num_observations)
    cfg = BaConfig(robust_kernel=RobustKernel.huber(1.0))
    want, want_bad = solver.cost(p, cfg)
    dp = DeviceProblem(p)
    for _ in range(2):
        got, bad, invalid = noalloc_cost(lib, dp, cfg)
        assert invalid == 0 and bad == want_bad
        assert got == pytest.approx(want, rel=COST_RTOL)
    w = p.obs_weight.copy()
    w[9] = -1.0
    skipped = p.copy()
    skipped.obs_weight = np.where(np.arange(p.num_observations) == 9, 0.0, w)
    want, _ = solver.cost(skipped, cfg)
    broken = p.copy()
    broken.obs_weight = w
    got, bad, invalid = noalloc_cost(lib, DeviceProblem(broken), cfg)
    assert invalid == 1 and got == pytest.approx(want, rel=COST_RTOL)


def test_rejects_more_observations_than_the_scratch_holds():
    """Rejected on the host before any device work (no GPU needed)."""
    lib = _abi.load_solver_library()
    p = synth.ring_problem(6, 50, seed=3).abi()
    p.num_observations = MAX_OBS + 1
    cost = C.c_double()
    counts = (C.c_uint64 * 2)()
    err = C.create_string_buffer(256)
    st = lib.visloc_ba_cuda_cost_noalloc(C.byref(p), C.byref(BaConfig().to_abi()), None,
                                         C.cast(C.byref(cost), C.c_void_p),
                                         C.cast(counts, C.c_void_p), err, len(err))
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert b"at most 16777216" in err.value
