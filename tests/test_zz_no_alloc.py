"""The allocation-free inverse application against the regular one.

``pd_apply_inverse_static`` serves callers that cannot allocate device memory
at solve time (inside a stream capture, under a host-owned allocator, in a
real-time loop): its intermediate vector lives in a fixed device array of the
library. It must agree with ``pd_apply_inverse``, which uses solver-owned
scratch, on consecutive calls (the shared array keeps the previous call's
contents). This file sorts last so that a failure here comes after every
other test has run.
"""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import SolverDiffPhD, _lib
from tests.helpers import DENSITY, tet_grid_model

pytestmark = pytest.mark.gpu


def _apply(solver, name, rhs):
    out = torch.empty_like(rhs)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(getattr(_lib.library(), name)(solver._handle, _lib.ptr(rhs), _lib.ptr(out), stream))
    torch.cuda.synchronize()
    return out


def test_static_scratch_apply_matches_solver_scratch_apply_on_consecutive_calls():
    model = tet_grid_model(contrast=10.0)
    solver = SolverDiffPhD(model, density=DENSITY)
    solver.step(model.state(), model.state(), None, None, 0.004)  # builds and uploads the factor
    rng = np.random.default_rng(11)
    for call in range(2):
        rhs = torch.tensor(rng.standard_normal((model.particle_count, 3)), dtype=torch.float64, device="cuda")
        expected = _apply(solver, "pd_apply_inverse", rhs)
        actual = _apply(solver, "pd_apply_inverse_static", rhs)
        np.testing.assert_allclose(actual.cpu().numpy(), expected.cpu().numpy(), rtol=1e-14, atol=1e-16,
                                   err_msg=f"call {call}")


def test_static_scratch_apply_refuses_more_particles_than_its_array_holds_and_keeps_the_device():
    from newton_solver_diff_phd_b200 import ModelBuilder

    # 41 x 41 x 40 vertices = 67,240 particles: one more layer than the
    # 65,536-particle array holds. The factor is never built: the size check
    # comes first.
    builder = ModelBuilder(gravity=(0.0, 0.0, 0.0))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=40, dim_y=40, dim_z=39,
                          cell_x=0.01, cell_y=0.01, cell_z=0.01, density=DENSITY, k_mu=1.0e4, k_lambda=1.0e4,
                          k_damp=0.0, fix_left=True)
    model = builder.finalize("cuda")
    assert model.particle_count > 65536
    solver = SolverDiffPhD(model, density=DENSITY)
    rhs = torch.zeros((model.particle_count, 3), dtype=torch.float64, device="cuda")
    out = torch.empty_like(rhs)
    device = torch.cuda.current_device()
    lib = _lib.library()
    code = lib.pd_apply_inverse_static(solver._handle, _lib.ptr(rhs), _lib.ptr(out),
                                       torch.cuda.current_stream().cuda_stream)
    assert code == _lib.PD_ERR_INVALID
    assert b"65536" in lib.pd_last_error()
    assert torch.cuda.current_device() == device
