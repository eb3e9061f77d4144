"""The mesh_contact state force (tests/test_diff_phd_mesh_contact.py of the reference)."""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import ModelBuilder, SolverDiffPhD
from oracle import pd_oracle
from tests.helpers import DENSITY, golden, oracle_tet_body

pytestmark = pytest.mark.gpu

TIGHT = {"max_iterations": 3000, "abs_tol": 1.0e-12, "rel_tol": 1.0e-11}
_TET_FACES = np.array(((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)))


def _two_bodies(gap, requires_grad=False):
    """A soft 3x2x2 grid (bottom pinned) and one tetrahedron whose apex reaches ``gap`` above the grid top."""
    builder = ModelBuilder(gravity=(0.0, 0.0, 0.0))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=3, dim_y=2, dim_z=2, cell_x=0.1,
                          cell_y=0.1, cell_z=0.1, density=DENSITY, k_mu=3.0e4, k_lambda=8.0e4, k_damp=0.0,
                          fix_bottom=True)
    grid = builder.particle_count
    for point in ((0.13, 0.11, 0.2 + gap), (0.33, 0.07, 0.5), (0.05, 0.18, 0.5), (0.17, 0.02, 0.55)):
        builder.add_particle(point, (0.0, 0.0, 0.0), 1.0)
    builder.add_tetrahedron(grid, grid + 1, grid + 2, grid + 3, k_mu=3.0e4, k_lambda=8.0e4)
    model = builder.finalize("cuda", requires_grad=requires_grad)
    tets = model.tet_indices.cpu().numpy().reshape(-1, 4)
    faces = tets[:, _TET_FACES].reshape(-1, 3)
    _, first, counts = np.unique(np.sort(faces, axis=1), axis=0, return_index=True, return_counts=True)
    faces = faces[first[counts == 1]]
    return model, faces[np.all(faces < grid, axis=1)], faces[np.all(faces >= grid, axis=1)]


def test_force_matches_reference_transcription():
    g = golden("mesh_contact.npz")
    model, faces_a, faces_b = _two_bodies(-0.004)
    np.testing.assert_array_equal(model.particle_q.cpu().numpy(), g["vertices"].astype(np.float32))
    options = tuple(g["options"]) + (g["faces_a"], g["faces_b"])
    solver = SolverDiffPhD(model, density=DENSITY, mesh_contact=options)
    for trial in range(4):
        q, v = g[f"t{trial}__q"], g[f"t{trial}__v"]
        expected = g[f"t{trial}__force"]
        got = solver.mesh_contact_force(torch.as_tensor(q), torch.as_tensor(v)).cpu().numpy()
        np.testing.assert_allclose(got, expected, rtol=0.0, atol=1.0e-12 * max(np.abs(expected).max(), 1.0))


def test_step_matches_oracle_with_state_force_in_the_target():
    model, faces_a, faces_b = _two_bodies(-0.003)
    options = (0.01, 5.0e3, 5.0e4, 50.0, 0.5, faces_a, faces_b)
    solver = SolverDiffPhD(model, density=DENSITY, mesh_contact=options, **TIGHT)
    rng = np.random.default_rng(3)
    state_in, state_out = model.state(), model.state()
    free = model.particle_inv_mass.cpu().numpy() > 0
    velocity = np.where(free[:, None], 0.2 * rng.standard_normal((model.particle_count, 3)), 0.0)
    state_in.particle_qd.copy_(torch.as_tensor(velocity, dtype=torch.float32))
    dt = 0.004
    solver.step(state_in, state_out, None, None, dt)
    solver.check_status()
    assert solver.mesh_contact_pairs > 0
    q = state_in.particle_q.cpu().numpy().astype(np.float64)
    v = state_in.particle_qd.cpu().numpy().astype(np.float64)
    force = pd_oracle.mesh_contact_force(q, v, faces_a, faces_b, *options[:5])
    assert np.abs(force).max() > 0.0
    expected, _iterations, converged = pd_oracle.step(oracle_tet_body(model), q, v, force, np.zeros(3), dt,
                                                      max_iterations=3000, abs_tol=1.0e-12, rel_tol=1.0e-11)
    assert converged
    np.testing.assert_allclose(solver._x.cpu().numpy(), expected, rtol=0.0, atol=1.0e-10 * np.abs(expected).max())


def test_gradients_hold_the_state_force_fixed():
    """The reference's BackwardForce is zero: gradients equal those of the same step with
    the evaluated contact force supplied as a constant external force."""
    results = []
    for frozen in (False, True):
        model, faces_a, faces_b = _two_bodies(-0.003, requires_grad=True)
        weights = torch.as_tensor(np.random.default_rng(5).standard_normal((model.particle_count, 3)),
                                  dtype=torch.float32, device="cuda")
        options = (0.01, 5.0e3, 5.0e4, 50.0, 0.5, faces_a, faces_b)
        solver = SolverDiffPhD(model, density=DENSITY, mesh_contact=None if frozen else options, **TIGHT)
        state_in, state_out = model.state(), model.state()
        if frozen:
            q = state_in.particle_q.cpu().numpy().astype(np.float64)
            force = pd_oracle.mesh_contact_force(q, np.zeros_like(q), faces_a, faces_b, *options[:5])
            state_in.particle_f.copy_(torch.as_tensor(force, dtype=torch.float32))
        state_in.requires_grad_(True)
        state_out.requires_grad_(True)
        record = torch.zeros((model.particle_count, 3), dtype=torch.float64, device="cuda")
        solver.step(state_in, state_out, None, None, 0.004, record=record)
        solver.check_status()
        state_out.particle_q.grad.copy_(weights)
        solver.backward_step(record, 0.004, state_in, state_out)
        results.append([state_in.particle_q.grad.cpu().numpy(), state_in.particle_qd.grad.cpu().numpy(),
                        solver._x.cpu().numpy()])
    for actual, expected in zip(results[0], results[1]):
        np.testing.assert_allclose(actual, expected, rtol=0.0, atol=1.0e-6 * max(np.abs(expected).max(), 1.0))


def test_invalid_mesh_contact_is_rejected():
    model, faces_a, faces_b = _two_bodies(0.0)
    for options in (
        (0.01, 5.0e3, 5.0e4, 50.0, 0.5, faces_a),
        (-0.01, 5.0e3, 5.0e4, 50.0, 0.5, faces_a, faces_b),
        (0.01, 5.0e3, 5.0e4, 50.0, 0.5, faces_a, np.zeros((0, 3), dtype=np.int32)),
        (0.01, 5.0e3, 5.0e4, 50.0, 0.5, faces_a, faces_b + model.particle_count),
    ):
        with pytest.raises(ValueError):
            SolverDiffPhD(model, density=DENSITY, mesh_contact=options)
