"""Steps captured in a caller's CUDA graph (tests/test_diff_phd_solver.py:337-371 and
tests/test_diff_phd_contact.py:142 of the reference): replays equal direct steps bitwise,
and replays observe device parameters edited between them."""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import SolverDiffPhD
from tests.helpers import DENSITY, deformed_arrays, golden, tet_grid_model

pytestmark = pytest.mark.gpu

OPTIONS = {"max_iterations": 500, "abs_tol": 1.0e-11, "rel_tol": 1.0e-10}


def _state(model, q, v):
    state = model.state()
    state.particle_q.copy_(torch.as_tensor(q, dtype=torch.float32))
    state.particle_qd.copy_(torch.as_tensor(v, dtype=torch.float32))
    return state


def test_captured_step_replays_equal_direct_steps_bitwise():
    model = tet_grid_model()
    free = model.particle_inv_mass.cpu().numpy() > 0
    q, v = deformed_arrays(model.particle_q.cpu().numpy(), free)
    direct = SolverDiffPhD(model, density=DENSITY, **OPTIONS)
    captured = SolverDiffPhD(model, density=DENSITY, **OPTIONS)
    state_in, direct_out, captured_out = _state(model, q, v), model.state(), model.state()
    captured.step(state_in, captured_out, None, None, 0.004)  # builds the factor outside the capture
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        captured.step(state_in, captured_out, None, None, 0.004)
    for _ in range(2):
        captured_out.particle_q.zero_()
        graph.replay()
        direct.step(state_in, direct_out, None, None, 0.004)
        torch.cuda.synchronize()
        assert torch.equal(captured_out.particle_q, direct_out.particle_q)
        assert torch.equal(captured_out.particle_qd, direct_out.particle_qd)
    captured.check_status()
    direct.check_status()


def test_graph_replay_observes_edited_sphere_parameters():
    g = golden("frictional_contact.npz")
    model = tet_grid_model(fix_left=False)
    center = g["sphere__parameters"]
    options = {"max_iterations": 2000, "abs_tol": 1.0e-9, "rel_tol": 1.0e-6}
    direct = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("spherical", center), friction=0.4, **options)
    captured = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("spherical", center), friction=0.4,
                             **options)
    state_in = _state(model, g["sphere__s1__q"], g["sphere__s1__v"])
    direct_out, captured_out = model.state(), model.state()
    captured.step(state_in, captured_out, None, None, 0.004)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        captured.step(state_in, captured_out, None, None, 0.004)
    for offset in (0.0, 0.01, 0.02):
        parameters = torch.tensor([[center[0] + offset, center[1], center[2] + offset, center[3]]],
                                  dtype=torch.float64, device="cuda")
        direct.boundary_parameters.copy_(parameters)
        captured.boundary_parameters.copy_(parameters)
        # Same multiplier warm start for both solvers.
        captured.contact_multipliers.copy_(direct.contact_multipliers)
        graph.replay()
        direct.step(state_in, direct_out, None, None, 0.004)
        torch.cuda.synchronize()
        assert torch.equal(captured_out.particle_q, direct_out.particle_q), offset
        np.testing.assert_array_equal(captured.contact_multipliers.cpu().numpy(),
                                      direct.contact_multipliers.cpu().numpy())
    captured.check_status()
    direct.check_status()
