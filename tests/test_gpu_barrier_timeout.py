"""Failure detection of the persistent kernels' device barriers.

Every wait of a persistent launch polls a bounded number of times; when the
budget runs out it sets status bit 1024 (``PD_STATUS_BARRIER_TIMEOUT``), raises
the team's abort flag, and the kernel returns instead of hanging. These tests
make the waits run out without any fault: a barrier that expects more
arrivals than blocks were launched (nothing ever completes it), and a real
step whose poll budget is lowered to one poll. No GPU is hung or faulted: every
wait ends within its budget.
"""

import ctypes

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import SolverDiffPhD, _lib
from tests.helpers import DENSITY, deformed_arrays, tet_grid_model

pytestmark = pytest.mark.gpu


def _probe(blocks, missing, mode, polls):
    status, returned = ctypes.c_int32(), ctypes.c_int32()
    _lib.check(_lib.library().pd_barrier_probe(torch.cuda.current_device(), blocks, missing, mode, polls,
                                               ctypes.byref(status), ctypes.byref(returned)))
    return status.value, returned.value


@pytest.mark.parametrize("mode", [0, 1], ids=["grid_sync", "serial_section"])
@pytest.mark.parametrize("blocks", [2, 64])
def test_barrier_missing_an_arrival_times_out_and_every_block_returns(mode, blocks):
    status, returned = _probe(blocks, 1, mode, 2000)
    assert status & _lib.STATUS_BARRIER_TIMEOUT
    assert returned == blocks


def test_barrier_probe_rejects_an_unbounded_request():
    lib = _lib.library()
    status, returned = ctypes.c_int32(), ctypes.c_int32()
    assert lib.pd_barrier_probe(0, 4, 0, 0, 100, ctypes.byref(status), ctypes.byref(returned)) == _lib.PD_ERR_INVALID
    assert lib.pd_barrier_probe(0, 4, 1, 0, 0, ctypes.byref(status), ctypes.byref(returned)) == _lib.PD_ERR_INVALID


def test_step_with_an_exhausted_poll_budget_reports_the_timeout_and_recovers():
    model = tet_grid_model()
    solver = SolverDiffPhD(model, density=DENSITY, blocks=16, rel_tol=1e-10, abs_tol=1e-12)
    free = model.particle_inv_mass.cpu().numpy() > 0
    q, qd = deformed_arrays(model.particle_q.cpu().numpy(), free)
    state_in, state_out = model.state(), model.state()
    state_in.particle_q.copy_(torch.tensor(q))
    state_in.particle_qd.copy_(torch.tensor(qd))
    solver.step(state_in, state_out, None, None, 0.004)  # build and a normal step
    torch.cuda.synchronize()
    assert solver.read_status() == 0
    expected = state_out.particle_q.clone()
    lib = _lib.library()
    _lib.check(lib.pd_set_spin_limit(solver._handle, 1))
    timed_out = 0
    for _ in range(4):  # one poll: some block arrives early and gives up
        solver.step(state_in, state_out, None, None, 0.004)
        torch.cuda.synchronize()
        timed_out |= solver.read_status()
    assert timed_out & _lib.STATUS_BARRIER_TIMEOUT
    _lib.check(lib.pd_set_spin_limit(solver._handle, 0))
    solver.step(state_in, state_out, None, None, 0.004)
    torch.cuda.synchronize()
    assert solver.read_status() == 0
    np.testing.assert_array_equal(state_out.particle_q.cpu().numpy(), expected.cpu().numpy())


def test_check_status_raises_on_the_timeout_bit():
    model = tet_grid_model()
    solver = SolverDiffPhD(model, density=DENSITY, blocks=16)
    state_in, state_out = model.state(), model.state()
    solver.step(state_in, state_out, None, None, 0.004)
    torch.cuda.synchronize()
    solver.read_status()
    _lib.check(_lib.library().pd_set_spin_limit(solver._handle, 1))
    raised = False
    for _ in range(4):
        solver.step(state_in, state_out, None, None, 0.004)
        try:
            solver.check_status()
        except RuntimeError as error:
            assert "barrier" in str(error)
            raised = True
            break
    _lib.check(_lib.library().pd_set_spin_limit(solver._handle, 0))
    assert raised
