"""The reference's problem dump format (ba_problem_io.rs) and the replay of a
dumped problem, against the committed fixtures of tests/golden (written by
tests/golden/make_golden.py: problems in the dump format and the FP64
oracle's solve of each)."""

from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle
from visloc_ba import BaConfig, RobustKernel
from visloc_ba.problem_io import (
    read_ba_problem,
    read_packed_problem,
    write_ba_problem,
    write_packed_problem,
)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = ["ring12", "street160"]


def expected(name):
    with open(os.path.join(GOLDEN, f"{name}_expected.json")) as f:
        return json.load(f)


def config_of(spec) -> BaConfig:
    kind, value = spec["robust_kernel"]
    rk = {"none": RobustKernel.none(), "huber": RobustKernel.huber(value),
          "cauchy": RobustKernel.cauchy(value)}[kind]
    return BaConfig(max_iterations=spec["max_iterations"], robust_kernel=rk)


def same_dump(a: str, b: str) -> bool:
    """Equal dumps, but for the quaternions, which the reader normalises (as
    UnitQuaternion::from_quaternion does): those within 2 ulp."""
    la, lb = a.split("\n"), b.split("\n")
    if len(la) != len(lb):
        return False
    npose = int(la[1].split()[1])
    for i, (x, y) in enumerate(zip(la, lb)):
        if 2 <= i < 2 + npose:
            fx, fy = x.split(), y.split()
            if fx[0] != fy[0] or fx[5:] != fy[5:]:
                return False
            qx = np.array(fx[1:5], float)
            qy = np.array(fy[1:5], float)
            if np.any(np.abs(qx - qy) > 2 * np.spacing(np.maximum(np.abs(qx), 1e-300))):
                return False
        elif x != y:
            return False
    return True


@pytest.mark.parametrize("name", CASES)
def test_dump_round_trips(name, tmp_path):
    path = os.path.join(GOLDEN, f"{name}_problem.txt")
    packed, pids, lids, w = read_packed_problem(path)
    out = tmp_path / "again.txt"
    write_packed_problem(packed, pids, lids, w, out)
    assert same_dump(open(path).read(), open(out).read())
    ba, w2 = read_ba_problem(path)
    out2 = tmp_path / "again_ba.txt"
    write_ba_problem(ba, w2, out2)
    assert open(out).read() == open(out2).read()  # both readers agree bit for bit


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_the_fixture(name):
    """The oracle's solve of the dumped problem, bit for bit as committed."""
    e = expected(name)
    packed, _, _, _ = read_packed_problem(os.path.join(GOLDEN, f"{name}_problem.txt"))
    st, res = oracle.optimize(packed, config_of(e["config"]))
    assert st == 0
    assert res.initial_cost == e["initial_cost"]
    assert res.final_cost == e["final_cost"]
    assert [bool(i.step_accepted) for i in res.iterations] == e["step_accepted"]
    assert [i.lambda_ for i in res.iterations] == e["lambda"]
    assert np.array_equal(packed.camera_centers(), np.array(e["camera_centers"]))


def test_reader_resolves_ids_and_normalises_quaternions(tmp_path):
    text = ("camera 640 480 500 500 320 240\nposes 2\n"
            "5 2 0 0 0 0 0 0 1\n9 1 0 0 0 -1 0 0 0\n"
            "landmarks 2\n4 0 0 5\n8 1 0 5\n"
            "observations 3 1\n5 4 320 240 1.5\n9 8 420 240 1\n9 6 1 1 1\n")
    path = tmp_path / "p.txt"
    path.write_text(text)
    packed, pids, lids, w = read_packed_problem(path)
    assert pids == [5, 9] and lids == [4, 8]
    assert packed.pose_q[0].tolist() == [1.0, 0.0, 0.0, 0.0]  # (2,0,0,0) normalised
    assert packed.obs_pose.tolist() == [0, 1, 1]
    assert packed.obs_landmark.tolist() == [0, 1, 0xFFFFFFFF]  # id 6 does not resolve
    assert w.tolist() == [1.5, 1.0, 1.0]
    assert packed.pose_fixed.tolist() == [1, 0]
    ba, wb = read_ba_problem(path)
    assert sorted(ba.poses) == [5, 9] and 5 in ba.fixed_poses and wb == [1.5, 1.0, 1.0]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_replay_of_the_fixture_matches_the_oracle(name):
    """replay.py (the ba_gpu_replay counterpart) on the committed dump."""
    e = expected(name)
    cfg = e["config"]
    kind, value = cfg["robust_kernel"]
    robust = "none" if kind == "none" else f"{kind}:{value}"
    cmd = [sys.executable, os.path.join(ROOT, "visloc-rs_b200", "visloc_ba", "replay.py"),
           os.path.join(GOLDEN, f"{name}_problem.txt"), "--iterations",
           str(cfg["max_iterations"]), "--robust", robust, "--pcg-tol", "1e-8",
           "--pcg-max", "300"]
    out = json.loads(subprocess.run(cmd, check=True, capture_output=True, text=True).stdout)
    run = out["gpu"][0]
    assert run["initial_cost"] == pytest.approx(e["initial_cost"], rel=1e-12)
    assert abs(run["final_cost"] - e["final_cost"]) <= 1e-5 * e["final_cost"]
    assert out["rms_px_after"] < out["rms_px_before"]
