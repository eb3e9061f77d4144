"""Forward step on the B200 against the reference's golden iterates and the oracle.

Mirrors tests/test_diff_phd_solver.py and tests/test_diff_phd_hex.py of the
reference: positions within 1e-10 of max|x| of the reference oracle, identical
iteration counts, Eigen SVD conventions, Dirichlet handling and status bits.
"""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import ConvergenceError, SolverDiffPhD
from oracle import pd_oracle
from tests.helpers import DENSITY, deformed_arrays, golden, oracle_tet_body, particle_model, tet_grid_model, two_cube_mesh

pytestmark = pytest.mark.gpu


def _state_from(model, q, v, f=None):
    state = model.state()
    state.particle_q.copy_(torch.as_tensor(q, dtype=torch.float32))
    state.particle_qd.copy_(torch.as_tensor(v, dtype=torch.float32))
    if f is not None:
        state.particle_f.copy_(torch.as_tensor(f, dtype=torch.float32))
    return state


@pytest.mark.parametrize("contrast,material,label", [
    (1.0, "pd", "fixed"), (1.0, "pd", "converged"), (1.0, "neo_hookean", "fixed"), (1.0, "neo_hookean", "converged"),
    (10.0, "pd", "converged"), (10.0, "neo_hookean", "converged"), (100.0, "pd", "converged"),
    (100.0, "neo_hookean", "converged"),
])
def test_forward_matches_reference_iterates(contrast, material, label):
    g = golden("tet_forward.npz")
    c = f"c{int(contrast)}"
    key = f"{c}_{material}_{label}"
    options = g[key + "__options"]
    model = tet_grid_model(contrast)
    np.testing.assert_array_equal(model.tet_materials.cpu().numpy()[:, 0].astype(np.float64), g[c + "__mu"])
    solver = SolverDiffPhD(model, density=DENSITY, material=material, max_iterations=int(options[0]),
                           abs_tol=float(options[1]), rel_tol=float(options[2]))
    state_in, state_out = _state_from(model, g[c + "__q"], g[c + "__v"]), model.state()
    solver.step(state_in, state_out, None, None, 0.004)
    if label == "fixed":
        with pytest.raises(ConvergenceError):
            solver.check_status()
    else:
        solver.check_status()
    expected = g[key + "__x"]
    np.testing.assert_allclose(solver._x.cpu().numpy(), expected, rtol=0.0, atol=1.0e-10 * np.abs(expected).max())
    assert int(solver.iterations[0]) == int(g[key + "__iterations"])
    np.testing.assert_array_equal(state_out.particle_q.cpu().numpy(), expected.astype(np.float32))


def test_muscle_activation_matches_reference():
    g = golden("tet_forward.npz")
    model = tet_grid_model()
    solver = SolverDiffPhD(model, density=DENSITY, muscle_directions=g["muscle__directions"],
                           muscle_stiffness=g["muscle__stiffness"], max_iterations=500, abs_tol=1e-11, rel_tol=1e-10)
    control = model.control()
    control.tet_activations = torch.tensor(g["muscle__contraction"], device="cuda")
    state_in, state_out = _state_from(model, g["muscle__q"], g["muscle__v"]), model.state()
    solver.step(state_in, state_out, control, None, 0.004)
    solver.check_status()
    expected = g["muscle__x"]
    np.testing.assert_allclose(solver._x.cpu().numpy(), expected, rtol=0.0, atol=1.0e-10 * np.abs(expected).max())


@pytest.mark.parametrize("material", ["pd", "neo_hookean"])
def test_hex_heterogeneous_step_with_muscles_and_planes(material):
    h = golden("hex_forward.npz")
    mesh = two_cube_mesh()
    model = particle_model(mesh.vertices, np.arange(12) < 4)
    solver = SolverDiffPhD(
        model, density=1000, hex_mesh=mesh, hex_materials=h["materials"], material=material,
        muscle_directions=[[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]], muscle_stiffness=[1000.0, 300.0],
        muscle_targets=[0.0, 0.8], planar_energies=(np.array([0, 8, 9]), 120.0, (0.0, 0.0, 2.0, -0.08)),
        anderson_window=0, max_iterations=1000, rel_tol=1e-10, abs_tol=1e-12,
    )
    assert solver.mean_volume == pytest.approx(0.001, abs=1e-16)
    assert solver.particle_mass == pytest.approx(1.0, abs=1e-13)
    state, out = _state_from(model, h["q"], h["v"], h["f"]), model.state()
    solver.step(state, out, None, None, 0.003)
    solver.check_status()
    np.testing.assert_allclose(out.particle_q.cpu().numpy(), h[material + "__x"], rtol=0, atol=2e-8)
    np.testing.assert_allclose(solver._x.cpu().numpy(), h[material + "__x"], rtol=0, atol=1e-12)
    assert int(solver.iterations[0]) == int(h[material + "__iterations"])
    # Every column of the inverse, including the eliminated pins.
    columns = torch.eye(12, dtype=torch.float64, device="cuda")
    for axis in range(0, 12, 3):
        rhs = columns[:, axis:axis + 3].contiguous()
        result = solver.apply_inverse(rhs).cpu().numpy()
        np.testing.assert_allclose(result, h[material + "__inverse"][:, axis:axis + 3], atol=2e-14, rtol=2e-12)


def test_hex_affine_patch_determinants():
    mesh = two_cube_mesh()
    model = particle_model(mesh.vertices, np.zeros(12, bool))
    solver = SolverDiffPhD(model, density=1000, hex_mesh=mesh, hex_materials=[[2e3, 5e3], [2e4, 5e4]])
    f = np.array([[1.05, 0.02, -0.03], [0.06, 0.96, 0.08], [0.0, -0.04, 1.03]])
    state = model.state()
    state.particle_q.copy_(torch.tensor(mesh.vertices @ f.T + [0.2, -0.3, 0.4], dtype=torch.float32))
    determinants = solver.deformation_determinants(state).cpu().numpy()
    assert determinants.shape == (2, 8)
    np.testing.assert_allclose(determinants, np.linalg.det(f), atol=6e-7, rtol=0)
    q = mesh.vertices.copy()
    q[:, 0] += 2.0 * q[:, 0] * q[:, 1] * q[:, 2]
    state.particle_q.copy_(torch.tensor(q, dtype=torch.float32))
    assert np.ptp(solver.deformation_determinants(state).cpu().numpy()[0]) > 0.01


def test_reflected_rest_shape_remains_stationary():
    model = tet_grid_model(fix_left=False, gravity=0.0, cell=0.125)
    state_in, state_out = model.state(), model.state()
    reflected = state_in.particle_q.clone()
    reflected[:, 0] *= -1.0
    state_in.particle_q.copy_(reflected)
    for material in ("pd", "neo_hookean"):
        solver = SolverDiffPhD(model, density=DENSITY, material=material, max_iterations=20)
        solver.step(state_in, state_out, None, None, 0.001)
        solver.check_status()
        assert torch.isfinite(state_out.particle_q).all()
        np.testing.assert_allclose(state_out.particle_q.cpu().numpy(), reflected.cpu().numpy(), rtol=0, atol=1e-12)
        np.testing.assert_allclose(state_out.particle_qd.cpu().numpy(), 0.0, rtol=0, atol=1e-10)


def test_rigid_free_fall_is_the_inertial_target():
    model = tet_grid_model(fix_left=False, cell=0.125)
    solver = SolverDiffPhD(model, density=DENSITY)
    state_in, state_out = model.state(), model.state()
    velocity = np.tile([0.25, -0.125, 0.5], (model.particle_count, 1)).astype(np.float32)
    state_in.particle_qd.copy_(torch.tensor(velocity))
    dt = 2.0**-7
    solver.step(state_in, state_out, None, None, dt)
    solver.check_status()
    gravity = model.gravity.cpu().numpy()[0].astype(np.float64)
    q0 = state_in.particle_q.cpu().numpy().astype(np.float64)
    np.testing.assert_allclose(solver._x.cpu().numpy(), q0 + dt * velocity + dt**2 * gravity, rtol=0, atol=1e-12)


@pytest.mark.parametrize("integrate", [False, True])
def test_dirichlet_particles_are_fixed_or_prescribed(integrate):
    model = tet_grid_model()
    pinned = model.particle_inv_mass.cpu().numpy() == 0
    velocity = np.zeros((model.particle_count, 3), dtype=np.float32)
    velocity[pinned] = [0.0, 0.5, 0.0]
    solver = SolverDiffPhD(model, density=DENSITY, integrate_pinned_velocities=integrate)
    state_in, state_out = model.state(), model.state()
    state_in.particle_qd.copy_(torch.tensor(velocity))
    solver.step(state_in, state_out, None, None, 0.01)
    solver.check_status()
    q0 = state_in.particle_q.cpu().numpy()[pinned]
    expected = q0 + 0.01 * velocity[pinned] if integrate else q0
    np.testing.assert_allclose(state_out.particle_q.cpu().numpy()[pinned], expected, atol=1e-7)
    targets = state_in.particle_q.clone()
    targets[torch.tensor(pinned, device="cuda")] += torch.tensor([0.0, 0.0, 0.02], device="cuda")
    solver.step(state_in, state_out, None, None, 0.01, dirichlet_positions=targets)
    solver.check_status()
    np.testing.assert_allclose(state_out.particle_q.cpu().numpy()[pinned], targets.cpu().numpy()[pinned], atol=1e-7)


def test_status_reports_nonconvergence_until_checked():
    model = tet_grid_model()
    solver = SolverDiffPhD(model, density=DENSITY, max_iterations=2, abs_tol=0.0, rel_tol=0.0)
    q, v = deformed_arrays(model.particle_q.cpu().numpy(), model.particle_inv_mass.cpu().numpy() > 0)
    state_in, state_out = _state_from(model, q, v), model.state()
    solver.step(state_in, state_out, None, None, 0.004)
    assert int(solver.iterations[0]) == 2
    with pytest.raises(ConvergenceError):
        solver.check_status()
    solver.check_status()
    solver.max_iterations, solver.abs_tol, solver.rel_tol = 3, 0.0, 0.0
    solver.notify_model_changed(0)
    solver.step(state_in, state_out, None, None, 0.004)
    assert int(solver.iterations[0]) == 3


def test_invalid_configuration_is_rejected():
    model = tet_grid_model()
    for kwargs in ({"density": 0.0}, {"density": DENSITY, "material": "linear"},
                   {"density": DENSITY, "anderson_window": 9}, {"density": DENSITY, "max_iterations": 0}):
        with pytest.raises(ValueError):
            SolverDiffPhD(model, **kwargs)
    solver = SolverDiffPhD(model, density=DENSITY)
    state = model.state()
    with pytest.raises(ValueError):
        solver.step(state, state, None, None, 0.01)
    with pytest.raises(NotImplementedError):
        solver.step(state, model.state(), None, object(), 0.01)


def test_repeated_steps_are_bitwise_deterministic():
    model = tet_grid_model(contrast=10.0)
    q, v = deformed_arrays(model.particle_q.cpu().numpy(), model.particle_inv_mass.cpu().numpy() > 0)
    results = []
    for _ in range(3):
        solver = SolverDiffPhD(model, density=DENSITY)
        state_in, state_out = _state_from(model, q, v), model.state()
        for _step in range(3):
            solver.step(state_in, state_out, None, None, 0.004)
            state_in, state_out = state_out, state_in
        results.append(solver._x.cpu().numpy().copy())
    np.testing.assert_array_equal(results[0], results[1])
    np.testing.assert_array_equal(results[0], results[2])


def test_rollout_matches_oracle_with_anderson_on_a_larger_block():
    # 6x3x3 block, heterogeneous log-uniform E, gravity, 5 steps at rel 1e-6.
    from newton_solver_diff_phd_b200 import ModelBuilder, meshes

    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0, 0, 0), rot=None, vel=(0, 0, 0), dim_x=6, dim_y=3, dim_z=3, cell_x=0.01, cell_y=0.01,
                          cell_z=0.01, density=DENSITY, k_mu=1.0, k_lambda=1.0, k_damp=0.0, fix_left=True)
    model = builder.finalize("cuda")
    rng = np.random.default_rng(0)
    young = np.exp(rng.uniform(np.log(1e5), np.log(1e7), model.tet_count))
    mu, lam = meshes.lame_from_young(young, 0.4)
    model.tet_materials.copy_(torch.tensor(np.column_stack((mu, lam, np.zeros_like(mu))), dtype=torch.float32))
    solver = SolverDiffPhD(model, density=DENSITY, rel_tol=1e-6)
    body = oracle_tet_body(model)
    state_in, state_out = model.state(), model.state()
    q = state_in.particle_q.cpu().numpy().astype(np.float64)
    v = np.zeros_like(q)
    gravity = model.gravity.cpu().numpy()[0].astype(np.float64)
    for _ in range(5):
        solver.step(state_in, state_out, None, None, 5e-3)
        solver.check_status()
        x, iterations, converged = pd_oracle.step(body, q, v, np.zeros_like(q), gravity, 5e-3, max_iterations=10000,
                                                  abs_tol=1e-9, rel_tol=1e-6)
        assert converged
        gpu = solver._x.cpu().numpy()
        np.testing.assert_allclose(gpu, x, rtol=0, atol=1e-6 * np.abs(x).max())
        assert abs(int(solver.iterations[0]) - iterations) <= 1
        q_next = state_out.particle_q.cpu().numpy().astype(np.float64)
        v = state_out.particle_qd.cpu().numpy().astype(np.float64)
        q = q_next
        state_in, state_out = state_out, state_in


@pytest.mark.parametrize("precision", ["fp64", "fp32+refine"])
def test_streamed_factor_matches_the_resident_one(precision):
    """A factor left in global memory (padded streaming layout) steps like the
    one kept in shared memory; the adjoint as well."""
    from newton_solver_diff_phd_b200 import ModelBuilder, meshes

    results = []
    for resident in (True, False):
        builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
        builder.add_soft_grid(pos=(0, 0, 0), rot=None, vel=(0, 0, 0), dim_x=8, dim_y=3, dim_z=3, cell_x=0.01,
                              cell_y=0.01, cell_z=0.01, density=DENSITY, k_mu=1.0, k_lambda=1.0, k_damp=0.0,
                              fix_left=True)
        model = builder.finalize("cuda")
        rng = np.random.default_rng(0)
        young = np.exp(rng.uniform(np.log(1e5), np.log(1e7), model.tet_count))
        mu, lam = meshes.lame_from_young(young, 0.4)
        model.tet_materials.copy_(torch.tensor(np.column_stack((mu, lam, np.zeros_like(mu))), dtype=torch.float32))
        solver = SolverDiffPhD(model, density=DENSITY, rel_tol=1e-8, abs_tol=1e-12, precision=precision,
                               resident=resident, adjoint="exact", blocks=4)
        state_in, state_out = model.state(), model.state()
        record = torch.zeros((model.particle_count, 3), dtype=torch.float64, device="cuda")
        iterations = []
        for _ in range(3):
            solver.step(state_in, state_out, None, None, 5e-3, record=record)
            iterations.append(int(solver.iterations[0]))
            state_in, state_out = state_out, state_in
        solver.check_status()
        state_in.requires_grad_(True)
        state_out.requires_grad_(True)
        state_in.particle_q.grad.normal_(generator=torch.Generator(device="cuda").manual_seed(3))
        solver.backward_step(record, 5e-3, state_out, state_in)
        results.append((solver._x.clone(), iterations, state_out.particle_q.grad.clone()))
    (x_r, it_r, g_r), (x_s, it_s, g_s) = results
    assert max(abs(a - b) for a, b in zip(it_r, it_s)) <= 1
    assert float((x_r - x_s).abs().max()) <= 1e-7 * float(x_r.abs().max())
    assert float((g_r - g_s).abs().max()) <= 1e-5 * float(g_r.abs().max())
