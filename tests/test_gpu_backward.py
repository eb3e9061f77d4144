"""Backward pass on the B200: the reference adjoint's outputs, and finite differences.

Mirrors tests/test_diff_phd_adjoint.py of the reference. ``adjoint="reference"``
reproduces the reference's mean-weight adjoint (checked against the golden
vectors of reference_backward); ``adjoint="exact"`` is the derivative of the
forward map and is checked by central differences, including Hex8 cells.
"""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import SolverDiffPhD, Tape
from oracle import pd_oracle
from tests.helpers import DENSITY, deformed_arrays, golden, oracle_tet_body, particle_model, tet_grid_model, two_cube_mesh

pytestmark = pytest.mark.gpu

TIGHT = {"max_iterations": 3000, "abs_tol": 1.0e-12, "rel_tol": 1.0e-12}


def _state(model, q, v, requires_grad=True):
    state = model.state(requires_grad=False)
    state.particle_q.copy_(torch.as_tensor(q, dtype=torch.float32))
    state.particle_qd.copy_(torch.as_tensor(v, dtype=torch.float32))
    if requires_grad:
        state.requires_grad_(True)
    return state


@pytest.mark.parametrize("key", ["c2_pd", "c1_pd", "c1_neo_hookean"])
def test_reference_adjoint_matches_reference_backward(key):
    b = golden("tet_backward.npz")
    contrast = float(key.split("_")[0][1:])
    material = key.split("_", 1)[1]
    model = tet_grid_model(contrast, requires_grad=True)
    solver = SolverDiffPhD(model, density=DENSITY, material=material, **TIGHT)
    state_in = _state(model, b[key + "__q"], b[key + "__v"])
    state_out = model.state(requires_grad=True)
    with Tape() as tape:
        solver.step(state_in, state_out, None, None, 0.004)
    np.testing.assert_allclose(solver._x.cpu().numpy(), b[key + "__x"], rtol=0, atol=1e-9 * np.abs(b[key + "__x"]).max())
    tape.backward(grads={state_out.particle_q: torch.tensor(b[key + "__gq"], dtype=torch.float32, device="cuda"),
                         state_out.particle_qd: torch.tensor(b[key + "__gv"], dtype=torch.float32, device="cuda")})
    bits = solver.read_status()
    assert bits & 8 == 0
    free = model.particle_inv_mass.cpu().numpy() > 0
    for name, tensor in (("q", state_in.particle_q), ("qd", state_in.particle_qd), ("f", state_in.particle_f)):
        expected = b[key + "__out_" + name]
        np.testing.assert_allclose(tensor.grad.cpu().numpy()[free], expected[free], rtol=2e-5,
                                   atol=2e-5 * np.abs(expected).max())
    # Pinned particles also receive the Dirichlet value gradient g_D - (A - K)_DF mu_F, which
    # the reference solver adds (adjoint.py:32-33) and reference_backward omits.
    body = oracle_tet_body(model, material)
    out = pd_oracle.backward(body, solver._x.cpu().numpy(), 0.004, b[key + "__gq"], b[key + "__gv"], mode="reference")
    expected = (out["q"] + out["dirichlet"])[~free]
    np.testing.assert_allclose(state_in.particle_q.grad.cpu().numpy()[~free], expected, rtol=0,
                               atol=2e-5 * np.abs(expected).max())
    expected = b[key + "__out_materials"]
    actual = model.tet_materials.grad.cpu().numpy()[:, :2]
    np.testing.assert_allclose(actual, expected, rtol=0, atol=1e-5 * np.abs(expected).max())


def _gradient_check(material, adjoint, contrast=1.0, muscles=False, integrate=False, material_checks=True):
    model = tet_grid_model(contrast, requires_grad=True)
    rng = np.random.default_rng(21)
    options = dict(TIGHT, density=DENSITY, material=material, adjoint=adjoint, integrate_pinned_velocities=integrate)
    if muscles:
        options["muscle_directions"] = rng.standard_normal((model.tet_count, 3))
        options["muscle_stiffness"] = 4.0e4
    solver = SolverDiffPhD(model, **options)
    dt = 0.004
    free = model.particle_inv_mass.cpu().numpy() > 0
    q, v = deformed_arrays(model.particle_q.cpu().numpy(), free, stretch=(1.2, 0.85, 1.05), speed=0.3)
    state_in = _state(model, q, v)
    with torch.no_grad():
        state_in.particle_f.copy_(torch.tensor(rng.uniform(-1.0, 1.0, (model.particle_count, 3)), dtype=torch.float32))
    state_out = model.state(requires_grad=True)
    control = model.control()
    contraction = rng.uniform(-0.2, 0.3, model.tet_count).astype(np.float32)
    if muscles:
        control.tet_activations = torch.tensor(contraction, device="cuda")
        control.tet_activations.grad = torch.zeros_like(control.tet_activations)
    q_weight = rng.standard_normal((model.particle_count, 3))
    qd_weight = 0.01 * rng.standard_normal((model.particle_count, 3))
    with Tape() as tape:
        solver.step(state_in, state_out, control, None, dt)
    tape.backward(grads={state_out.particle_q: torch.tensor(q_weight, dtype=torch.float32, device="cuda"),
                         state_out.particle_qd: torch.tensor(qd_weight, dtype=torch.float32, device="cuda")})
    solver.check_status()
    q_weight32 = q_weight.astype(np.float32).astype(np.float64)
    qd_weight32 = qd_weight.astype(np.float32).astype(np.float64)

    def objective():
        scratch = model.state()
        solver.step(state_in, scratch, control, None, dt)
        solver.check_status()
        x = solver._x.cpu().numpy()
        q0 = state_in.particle_q.detach().cpu().numpy().astype(np.float64)
        return float(np.sum(x * q_weight32) + np.sum((x - q0) / dt * qd_weight32))

    def central(tensor, index, step, rebuild=False):
        with torch.no_grad():
            original = tensor[index].item()
            results, deltas = [], []
            for sign in (1.0, -1.0):
                tensor[index] = original + sign * step
                deltas.append(tensor[index].item())
                if rebuild:
                    solver.notify_model_changed(0)
                results.append(objective())
            tensor[index] = original
            if rebuild:
                solver.notify_model_changed(0)
        return (results[0] - results[1]) / (deltas[0] - deltas[1])

    checks = []
    nodes = np.flatnonzero(free)[[0, 7, 15]]
    pinned = np.flatnonzero(~free)[[0, -1]]
    for name, step in (("particle_q", 1.0e-4), ("particle_qd", 1.0e-3), ("particle_f", 1.0e-2)):
        tensor = getattr(state_in, name)
        analytic = tensor.grad.cpu().numpy()
        for node in (np.concatenate((nodes, pinned)) if name != "particle_f" else nodes):
            for axis in (0, 2):
                checks.append((name, analytic[node, axis], central(tensor, (int(node), axis), step)))
    if material_checks and material == "pd":
        gradient = model.tet_materials.grad.cpu().numpy()
        for element in (0, 11, 37):
            for column, step in ((0, 20.0), (1, 50.0)):
                checks.append(("tet_materials", gradient[element, column],
                               central(model.tet_materials, (element, column), step, rebuild=True)))
    if muscles:
        gradient = control.tet_activations.grad.cpu().numpy()
        for element in (2, 19):
            checks.append(("activation", gradient[element], central(control.tet_activations, element, 1.0e-3)))
    for name, analytic, numeric in checks:
        assert abs(analytic - numeric) <= 2.0e-4 * max(abs(numeric), 1.0e-3), (name, analytic, numeric)


def test_pd_state_and_material_gradients_match_finite_differences():
    _gradient_check("pd", "reference")


def test_neo_hookean_state_gradients_match_finite_differences():
    _gradient_check("neo_hookean", "reference", material_checks=False)


def test_activation_gradients_match_finite_differences():
    _gradient_check("pd", "reference", muscles=True)


def test_integrated_dirichlet_gradients_match_finite_differences():
    _gradient_check("neo_hookean", "reference", muscles=True, integrate=True, material_checks=False)


def test_exact_adjoint_matches_finite_differences_on_heterogeneous_materials():
    # The reference adjoint uses mean weights in K; the exact mode differentiates the forward map.
    _gradient_check("pd", "exact", contrast=4.0)


def test_exact_adjoint_matches_dense_oracle():
    model = tet_grid_model(3.0, requires_grad=True)
    solver = SolverDiffPhD(model, density=DENSITY, adjoint="exact", **TIGHT)
    free = model.particle_inv_mass.cpu().numpy() > 0
    q, v = deformed_arrays(model.particle_q.cpu().numpy(), free, stretch=(1.2, 0.85, 1.05), speed=0.3)
    state_in = _state(model, q, v)
    state_out = model.state(requires_grad=True)
    rng = np.random.default_rng(3)
    gq = rng.standard_normal((model.particle_count, 3)).astype(np.float32)
    with Tape() as tape:
        solver.step(state_in, state_out, None, None, 0.004)
    tape.backward(grads={state_out.particle_q: torch.tensor(gq, device="cuda")})
    solver.check_status()
    body = oracle_tet_body(model)
    out = pd_oracle.backward(body, solver._x.cpu().numpy(), 0.004, gq.astype(np.float64), np.zeros_like(gq, float), mode="exact")
    np.testing.assert_allclose(state_in.particle_f.grad.cpu().numpy(), out["f"], rtol=0, atol=2e-5 * np.abs(out["f"]).max())
    np.testing.assert_allclose(model.tet_materials.grad.cpu().numpy()[:, :2], out["materials"], rtol=0,
                               atol=1e-5 * np.abs(out["materials"]).max())


@pytest.mark.parametrize("adjoint", ["reference", "exact"])
def test_hex_adjoint_matches_dense_oracle_and_finite_differences(adjoint):
    mesh = two_cube_mesh()
    pinned = np.arange(12) < 4
    model = particle_model(mesh.vertices, pinned, requires_grad=True)
    materials = torch.tensor([[2000.0, 4000.0], [20000.0, 40000.0]], dtype=torch.float64, device="cuda")
    materials.grad = torch.zeros_like(materials)
    solver = SolverDiffPhD(model, density=1000, hex_mesh=mesh, hex_materials=materials, adjoint=adjoint, **TIGHT)
    q = mesh.vertices.copy()
    q[4:, 0] *= 1.04
    q[4:, 2] += 0.01 * q[4:, 0]
    v = np.random.default_rng(4).normal(0, 0.03, q.shape)
    v[:4] = 0
    state_in = _state(model, q, v)
    state_out = model.state(requires_grad=True)
    rng = np.random.default_rng(8)
    gq = rng.standard_normal((12, 3)).astype(np.float32)
    dt = 0.003
    with Tape() as tape:
        solver.step(state_in, state_out, None, None, dt)
    tape.backward(grads={state_out.particle_q: torch.tensor(gq, device="cuda")})
    solver.check_status()
    body = pd_oracle.Body.hex(mesh.vertices, mesh.indices, ~pinned, [2000.0, 20000.0], [4000.0, 40000.0], 1000.0)
    x = solver._x.cpu().numpy()
    out = pd_oracle.backward(body, x, dt, gq.astype(np.float64), np.zeros((12, 3)), mode=adjoint)
    np.testing.assert_allclose(state_in.particle_f.grad.cpu().numpy(), out["f"], rtol=0, atol=2e-5 * np.abs(out["f"]).max())
    np.testing.assert_allclose(materials.grad.cpu().numpy(), out["materials"], rtol=0,
                               atol=1e-5 * np.abs(out["materials"]).max())
    if adjoint == "exact":
        for element, column, step in ((0, 0, 20.0), (1, 1, 400.0)):
            values = []
            for sign in (1.0, -1.0):
                with torch.no_grad():
                    materials[element, column] += sign * step
                solver.notify_model_changed(0)
                solver.step(state_in, model.state(), None, None, dt)
                values.append(float(np.sum(solver._x.cpu().numpy() * gq.astype(np.float64))))
                with torch.no_grad():
                    materials[element, column] -= sign * step
            solver.notify_model_changed(0)
            numeric = (values[0] - values[1]) / (2 * step)
            analytic = materials.grad.cpu().numpy()[element, column]
            assert abs(analytic - numeric) <= 2e-4 * max(abs(numeric), 1e-3), (element, column, analytic, numeric)


def test_zero_volume_energy_suppresses_whole_material_gradient():
    model = tet_grid_model(requires_grad=True)
    with torch.no_grad():
        model.tet_materials[:, 1] = 0.0
    solver = SolverDiffPhD(model, density=DENSITY, **TIGHT)
    free = model.particle_inv_mass.cpu().numpy() > 0
    q, v = deformed_arrays(model.particle_q.cpu().numpy(), free, stretch=(1.2, 0.85, 1.05), speed=0.3)
    state_in = _state(model, q, v)
    state_out = model.state(requires_grad=True)
    seed = torch.tensor(np.random.default_rng(40).standard_normal((model.particle_count, 3)), dtype=torch.float32, device="cuda")
    with Tape() as tape:
        solver.step(state_in, state_out, None, None, 0.004)
    tape.backward(grads={state_out.particle_q: seed})
    assert solver.read_status() == 16
    np.testing.assert_array_equal(model.tet_materials.grad.cpu().numpy(), 0.0)
    assert torch.linalg.norm(state_in.particle_q.grad) > 0


def test_backbone_clip_suppresses_unreliable_contributions():
    model = tet_grid_model(fix_left=False, requires_grad=True)
    solver = SolverDiffPhD(model, density=DENSITY, **TIGHT)
    state_in, state_out = model.state(requires_grad=True), model.state(requires_grad=True)
    with Tape() as tape:
        solver.step(state_in, state_out, None, None, 0.004)
    seed = torch.zeros((model.particle_count, 3), dtype=torch.float32, device="cuda")
    seed[:, 0] = 1e12
    tape.backward(grads={state_out.particle_q: seed})
    assert solver.read_status() & 16
    for tensor in (state_in.particle_q, state_in.particle_qd, state_in.particle_f, model.tet_materials):
        np.testing.assert_array_equal(tensor.grad.cpu().numpy(), 0.0)
