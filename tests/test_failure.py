"""Failure handling without a GPU fault: a device wait that can never be
satisfied runs out of its bounded time, the kernel returns an error status
that the host reports (VLBA_ERR_TIMEOUT), and the context keeps working.
Host-side failures (invalid requests in a batch or a served stream) are
covered in test_batch.py and test_server.py."""

from __future__ import annotations

import pytest

from visloc_ba import BaConfig, RobustKernel, synth
from visloc_ba import _abi


@pytest.mark.gpu
def test_a_wait_on_a_flag_nothing_sets_times_out_and_the_context_survives(solver):
    st, waited = solver.wait_probe(250.0)
    assert st == _abi.ERR_TIMEOUT
    assert 200.0 <= waited <= 2000.0
    p = synth.ring_problem(10, 300, seed=5)
    st, res = solver.optimize(p.copy(), BaConfig(max_iterations=5,
                                                 robust_kernel=RobustKernel.huber(1.0)))
    assert st == _abi.OK and res.final_cost < res.initial_cost


def test_probe_limits_are_checked():
    lib = _abi.load_solver_library()
    import ctypes as C

    assert lib.visloc_ba_cuda_wait_probe(None, 10.0, C.byref(C.c_double())) == \
        _abi.ERR_INVALID_ARGUMENT
