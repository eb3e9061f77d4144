"""The frictional boundary on the B200 (tests/test_diff_phd_contact.py and
tests/test_diff_phd_mesh_boundary.py of the reference).

Every rollout steps the solver with the per-step states of the reference
transcription's rollout (tests/golden/frictional_contact.npz) and compares
positions (1e-9 absolute, the reference tests' bound), multipliers, iteration
counts, status and mesh candidates; the oracle restatement covers variants
without a fixture.
"""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import ConvergenceError, ModelBuilder, SolverDiffPhD
from oracle import pd_oracle
from tests.helpers import DENSITY, golden, oracle_tet_body, tet_grid_model

pytestmark = pytest.mark.gpu

GRID_CASES = ["plane", "stick", "slide", "sphere", "chatter", "restitution"]
MESH_CASES = ["mesh", "mesh_stick", "mesh_restitution", "mesh_two_sided"]


def _options(g, name):
    options = g[f"{name}__options"]
    return {"max_iterations": int(options[0]), "abs_tol": float(options[1]), "rel_tol": float(options[2])}


def _state(model, q, v):
    state = model.state()
    state.particle_q.copy_(torch.as_tensor(q, dtype=torch.float32))
    state.particle_qd.copy_(torch.as_tensor(v, dtype=torch.float32))
    return state


def _blocks_model(g):
    """The two soft blocks of the mesh boundary tests from the fixture's arrays."""
    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    for point, free in zip(g["blocks__vertices"], g["blocks__free"]):
        builder.add_particle(point, (0.0, 0.0, 0.0), 1.0 if free else 0.0)
    for tet in g["blocks__tets"]:
        builder.add_tetrahedron(*map(int, tet), k_mu=2.0e4, k_lambda=5.0e4)
    return builder.finalize("cuda")


def _steps(g, name):
    return sum(1 for key in g.files if key.startswith(f"{name}__s") and key.endswith("__x"))


def _rollout(g, name, solver, model, mesh):
    for t in range(_steps(g, name)):
        key = f"{name}__s{t}"
        state_in, state_out = _state(model, g[key + "__q"], g[key + "__v"]), model.state()
        solver.step(state_in, state_out, None, None, 0.004)
        assert int(solver.iterations[0]) == int(g[key + "__iterations"])
        converged = bool(g[key + "__converged"])
        assert (solver.read_status() == 0) == converged
        if not converged:
            continue
        np.testing.assert_allclose(solver._x.cpu().numpy(), g[key + "__x"], rtol=0.0, atol=1.0e-9)
        if mesh:
            candidate = solver.frictional_state()[3].cpu().numpy()
            np.testing.assert_array_equal(candidate, g[key + "__candidate"])
        if name != "mesh_two_sided":
            tolerance = {"rtol": 1.0e-5, "atol": 1.0e-6} if mesh else {"rtol": 1.0e-6, "atol": 1.0e-9}
            np.testing.assert_allclose(solver.contact_multipliers.cpu().numpy(), g[key + "__multiplier"], **tolerance)


@pytest.mark.parametrize("name", GRID_CASES)
def test_grid_against_plane_and_sphere_matches_reference(name):
    g = golden("frictional_contact.npz")
    model = tet_grid_model(fix_left=False)
    options = g[f"{name}__options"]
    kind = "spherical" if name in ("sphere", "chatter") else "planar"
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=(kind, g[f"{name}__parameters"]),
                           frictional_vertices=g["grid__nodes"], friction=float(options[3]),
                           restitution=float(options[4]), **_options(g, name))
    _rollout(g, name, solver, model, mesh=False)
    if name == "plane":
        # Converged complementarity: lambda >= 0 and zero gap where active.
        multiplier = solver.contact_multipliers.cpu().numpy()
        gaps = solver._x.cpu().numpy()[g["grid__nodes"], 2]
        assert multiplier.max() > 0.0 and np.all(multiplier >= 0.0)
        np.testing.assert_allclose(gaps[multiplier > 0], 0.0, atol=1.0e-9)
        assert gaps.min() > -1.0e-9


@pytest.mark.parametrize("name", MESH_CASES)
def test_soft_blocks_mesh_boundary_matches_reference(name):
    g = golden("frictional_contact.npz")
    model = _blocks_model(g)
    options = g[f"{name}__options"]
    boundary = ("mesh", (float(options[5]), int(g["blocks__split"]), g["blocks__faces_left"], g["blocks__faces_right"]))
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=boundary, frictional_vertices=g[f"{name}__nodes"],
                           friction=float(options[3]), restitution=float(options[4]), **_options(g, name))
    _rollout(g, name, solver, model, mesh=True)


def test_chatter_raises_convergence_error():
    g = golden("frictional_contact.npz")
    model = tet_grid_model(fix_left=False)
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("spherical", g["chatter__parameters"]),
                           friction=0.4, **_options(g, "chatter"))
    for t in range(2):
        key = f"chatter__s{t}"
        solver.step(_state(model, g[key + "__q"], g[key + "__v"]), model.state(), None, None, 0.004)
        if t == 0:
            solver.check_status()
    with pytest.raises(ConvergenceError):
        solver.check_status()


def test_fp32_refine_reaches_the_fp64_contact_solution():
    """FP32 factor products with FP64 refinement keep the contact fixed point."""
    g = golden("frictional_contact.npz")
    model = tet_grid_model(fix_left=False)
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("planar", g["stick__parameters"]),
                           frictional_vertices=g["grid__nodes"], friction=2.0, precision="fp32+refine",
                           **_options(g, "stick"))
    key = "stick__s0"
    solver.step(_state(model, g[key + "__q"], g[key + "__v"]), model.state(), None, None, 0.004)
    solver.check_status()
    np.testing.assert_allclose(solver._x.cpu().numpy(), g[key + "__x"], rtol=0.0, atol=1.0e-9)


def test_fp32_contact_solution_stays_within_the_fp32_shift():
    """FP32 local projections move the fixed point by about cond(A) x 6e-8; the
    gate is the reference example's (1e-9 absolute, 1e-6 relative)."""
    g = golden("frictional_contact.npz")
    model = tet_grid_model(fix_left=False)
    options = {"max_iterations": 2000, "abs_tol": 1.0e-9, "rel_tol": 1.0e-6}
    results = []
    for precision in ("fp64", "fp32"):
        solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("planar", g["stick__parameters"]),
                               frictional_vertices=g["grid__nodes"], friction=2.0, precision=precision, **options)
        key = "stick__s0"
        solver.step(_state(model, g[key + "__q"], g[key + "__v"]), model.state(), None, None, 0.004)
        solver.check_status()
        results.append(solver._x.cpu().numpy())
    np.testing.assert_allclose(results[1], results[0], rtol=0.0, atol=1.0e-5 * np.abs(results[0]).max())


def test_edited_sphere_parameters_match_the_oracle():
    """boundary_parameters aliases the device array the kernel reads at every step."""
    g = golden("frictional_contact.npz")
    model = tet_grid_model(fix_left=False)
    center = g["sphere__parameters"]
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("spherical", center), friction=0.4,
                           max_iterations=2000, abs_tol=1.0e-9, rel_tol=1.0e-6)
    nodes = solver.frictional_vertices
    body = oracle_tet_body(model)
    boundary = pd_oracle.FrictionalBoundary("spherical", center, nodes, friction=0.4)
    q, v = g["sphere__s1__q"], g["sphere__s1__v"]
    for offset in (0.0, 0.01, 0.02):
        parameters = np.array([center[0] + offset, center[1], center[2] + offset, center[3]])
        solver.boundary_parameters.copy_(torch.as_tensor(parameters[None]))
        boundary.parameters = parameters
        # Same multiplier warm start for both.
        boundary.multiplier = solver.contact_multipliers.cpu().numpy().copy()
        solver.step(_state(model, q, v), model.state(), None, None, 0.004)
        solver.check_status()
        expected, iterations, converged = pd_oracle.step(body, q, v, np.zeros_like(q), model.gravity[0].cpu().numpy(),
                                                         0.004, contact=boundary, max_iterations=2000, abs_tol=1.0e-9,
                                                         rel_tol=1.0e-6)
        assert converged and int(solver.iterations[0]) == iterations
        np.testing.assert_allclose(solver._x.cpu().numpy(), expected, rtol=0.0, atol=1.0e-9)


def test_default_vertices_are_the_tetrahedral_surface():
    model = tet_grid_model(fix_left=False)
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("planar", (0.0, 0.0, 1.0, 0.0)))
    assert np.array_equal(solver.frictional_vertices, golden("frictional_contact.npz")["grid__nodes"])
    assert solver.contact_multipliers.shape == (len(solver.frictional_vertices),)


def test_invalid_frictional_boundaries_are_rejected():
    model = tet_grid_model(fix_left=False)
    for kwargs in (
        {"frictional_boundary": ("cylinder", (0.0, 0.0, 1.0, 0.0))},
        {"frictional_boundary": ("planar", (0.0, 0.0, 0.0, 0.0))},
        {"frictional_boundary": ("planar", (0.0, 0.0, 1.0, np.nan))},
        {"frictional_boundary": ("planar", (0.0, 0.0, 1.0, 0.0)), "frictional_vertices": [0, 0]},
        {"frictional_boundary": ("planar", (0.0, 0.0, 1.0, 0.0)), "frictional_vertices": [model.particle_count]},
        {"frictional_boundary": ("planar", (0.0, 0.0, 1.0, 0.0)), "friction": -1.0},
        {"frictional_boundary": ("planar", (0.0, 0.0, 1.0, 0.0)), "restitution": np.inf},
        {"frictional_boundary": ("mesh", (-0.01, 0, [[0, 1, 2]], [[3, 4, 5]]))},
        {"frictional_boundary": ("mesh", (0.01, 0, [[0, 1, model.particle_count]], [[3, 4, 5]]))},
        {"friction": 0.5},
    ):
        with pytest.raises(ValueError):
            SolverDiffPhD(model, density=DENSITY, **kwargs)


@pytest.mark.parametrize("key", ["f0", "f5"])
def test_contact_woodbury_projection_matches_reference(key):
    """Parameter gradients through the contact projection (tests/test_diff_phd_adjoint.py:339-416):
    against the reference's reference_backward outputs and against the oracle on the
    solver's own recorded contact state; state gradients use mu."""
    from newton_solver_diff_phd_b200 import Tape

    g = golden("woodbury.npz")
    friction = 0.5 if key == "f5" else 0.0
    model = tet_grid_model(fix_left=False, requires_grad=True)
    directions = g[key + "__directions"]
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("planar", (0.0, 0.0, 1.0, 0.0)),
                           frictional_vertices=g["nodes"], friction=friction, muscle_directions=directions,
                           muscle_stiffness=4.0e4, max_iterations=2000, abs_tol=1.0e-12, rel_tol=1.0e-11)
    control = model.control()
    contraction = g[key + "__contraction"]
    control.tet_activations = torch.tensor(contraction, device="cuda")
    control.tet_activations.grad = torch.zeros_like(control.tet_activations)
    q = model.particle_q.cpu().numpy().astype(np.float64)
    q[:, 2] += 0.001 - q[:, 2].min()
    states = [_state(model, q, np.tile([0.3, 0.0, -1.0], (model.particle_count, 1)))]
    states += [model.state(requires_grad=True) for _ in range(3)]
    for i in range(2):
        solver.step(states[i], states[i + 1], control, None, 0.004)
    state_in, state_out = states[2], states[3]
    state_in.requires_grad_(True)
    with Tape() as tape:
        solver.step(state_in, state_out, control, None, 0.004)
    np.testing.assert_allclose(solver._x.cpu().numpy(), g[key + "__x"], rtol=0.0, atol=1.0e-8)
    tape.backward(grads={state_out.particle_q: torch.tensor(g[key + "__gq"], dtype=torch.float32, device="cuda"),
                         state_out.particle_qd: torch.tensor(g[key + "__gv"], dtype=torch.float32, device="cuda")})
    solver.check_status()
    multiplier, omega, normal, _ = solver.frictional_state()
    assert int((multiplier > 0).sum()) > 0
    body = oracle_tet_body(model, muscle_directions=directions, muscle_stiffness=np.full(model.tet_count, 4.0e4))
    oracle = pd_oracle.backward(body, solver._x.cpu().numpy(), 0.004, g[key + "__gq"], g[key + "__gv"],
                                targets=1.0 - contraction.astype(np.float64),
                                contact=(g["nodes"], multiplier.cpu().numpy(), omega.cpu().numpy(),
                                         normal.cpu().numpy(), friction))
    pairs = (
        ("q", state_in.particle_q.grad), ("qd", state_in.particle_qd.grad), ("f", state_in.particle_f.grad),
        ("materials", model.tet_materials.grad[:, :2]), ("activations", control.tet_activations.grad),
    )
    for name, tensor in pairs:
        actual = tensor.detach().cpu().numpy()
        for expected in (oracle[name], g[f"{key}__out_{name}"]):
            scale = max(np.abs(expected).max(), 1.0e-30)
            np.testing.assert_allclose(actual, expected, rtol=0.0, atol=1.0e-5 * scale, err_msg=name)


def test_large_contact_set_on_the_team_path_matches_the_oracle():
    """A 8x6x2 block: 63 floor contacts plus 200 registered surface vertices, so
    the Newton step runs across the team with the panelled Cholesky (two panels)."""
    from newton_solver_diff_phd_b200 import ModelBuilder

    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=8, dim_y=6, dim_z=2, cell_x=0.05,
                          cell_y=0.05, cell_z=0.05, density=DENSITY, k_mu=2.0e4, k_lambda=5.0e4, k_damp=0.0)
    model = builder.finalize("cuda")
    options = {"max_iterations": 2000, "abs_tol": 1.0e-12, "rel_tol": 1.0e-11}
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("planar", (0.0, 0.0, 1.0, 0.0)),
                           friction=0.5, **options)
    nodes = solver.frictional_vertices
    assert len(nodes) > 32
    body = oracle_tet_body(model)
    boundary = pd_oracle.FrictionalBoundary("planar", (0.0, 0.0, 1.0, 0.0), nodes, friction=0.5)
    q = model.particle_q.cpu().numpy().astype(np.float64)
    q[:, 2] += 0.0005
    q = q.astype(np.float32).astype(np.float64)
    v = np.tile(np.array([0.2, 0.0, -1.0], dtype=np.float32), (model.particle_count, 1)).astype(np.float64)
    gravity = model.gravity[0].cpu().numpy().astype(np.float64)
    for _ in range(2):
        solver.step(_state(model, q, v), model.state(), None, None, 0.004)
        solver.check_status()
        expected, iterations, converged = pd_oracle.step(body, q, v, np.zeros_like(q), gravity, 0.004,
                                                         contact=boundary, **options)
        assert converged and int(solver.iterations[0]) == iterations
        np.testing.assert_allclose(solver._x.cpu().numpy(), expected, rtol=0.0, atol=1.0e-9)
        np.testing.assert_allclose(solver.contact_multipliers.cpu().numpy(), boundary.multiplier, rtol=1.0e-6,
                                   atol=1.0e-9)
        assert int((boundary.multiplier > 0).sum()) > 32
        x = solver._x.cpu().numpy()
        q, v = x.astype(np.float32).astype(np.float64), ((x - q) / 0.004).astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("friction", [0.0, 0.5])
def test_woodbury_columns_on_lanes_match_one_launch_per_column(friction):
    """The contact projection of a 8x6x2 block resting on the floor (63 contacts,
    189 rows with friction): the parameter and state gradients with the columns
    side by side on lanes (automatic team: one launch; teams of 4 blocks: 74
    lanes, so three launches with friction) equal those of one launch per
    column, and the lanes' material gradients agree with the oracle's Woodbury
    projection."""
    from newton_solver_diff_phd_b200 import Tape
    from newton_solver_diff_phd_b200 import _lib

    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=8, dim_y=6, dim_z=2, cell_x=0.05,
                          cell_y=0.05, cell_z=0.05, density=DENSITY, k_mu=2.0e4, k_lambda=5.0e4, k_damp=0.0)
    model = builder.finalize("cuda", requires_grad=True)
    solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("planar", (0.0, 0.0, 1.0, 0.0)),
                           friction=friction, max_iterations=2000, abs_tol=1.0e-12, rel_tol=1.0e-11)
    q = model.particle_q.cpu().numpy().astype(np.float64)
    q[:, 2] += 0.0002
    v = np.tile([0.1, 0.0, -0.5], (model.particle_count, 1))
    rng = np.random.default_rng(7)
    gq = rng.standard_normal((model.particle_count, 3)).astype(np.float32)
    gv = rng.standard_normal((model.particle_count, 3)).astype(np.float32)
    for invalid in (-1, 3, 128):
        assert solver._lib.pd_set_woodbury_team(solver._handle, invalid) != 0
    results = []
    for lanes, team in ((1, 0), (1, 4), (0, 0)):
        _lib.check(solver._lib.pd_set_woodbury_lanes(solver._handle, lanes))
        _lib.check(solver._lib.pd_set_woodbury_team(solver._handle, team))
        model.tet_materials.grad = torch.zeros_like(model.tet_materials)
        state_in = _state(model, q, v)
        state_in.requires_grad_(True)
        state_out = model.state(requires_grad=True)
        with Tape() as tape:
            solver.step(state_in, state_out, None, None, 0.004)
        solver.check_status()
        tape.backward(grads={state_out.particle_q: torch.tensor(gq, device="cuda"),
                             state_out.particle_qd: torch.tensor(gv, device="cuda")})
        results.append({"materials": model.tet_materials.grad[:, :2].double().cpu().numpy(),
                        "q": state_in.particle_q.grad.double().cpu().numpy(),
                        "qd": state_in.particle_qd.grad.double().cpu().numpy()})
    multiplier, omega, normal, _ = solver.frictional_state()
    assert int(((multiplier > 0) & (omega >= 0.5)).sum()) > 32
    for result in results[:2]:
        for name in result:
            scale = max(np.abs(results[2][name]).max(), 1.0e-30)
            np.testing.assert_allclose(result[name], results[2][name], rtol=0.0, atol=1.0e-9 * scale, err_msg=name)
    body = oracle_tet_body(model)
    oracle = pd_oracle.backward(body, solver._x.cpu().numpy(), 0.004, gq.astype(np.float64), gv.astype(np.float64),
                                contact=(solver.frictional_vertices, multiplier.cpu().numpy(), omega.cpu().numpy(),
                                         normal.cpu().numpy(), friction))
    # The columns are fixed points capped at 120 iterations, the oracle's are direct solves.
    scale = max(np.abs(oracle["materials"]).max(), 1.0e-30)
    np.testing.assert_allclose(results[0]["materials"], oracle["materials"], rtol=0.0, atol=1.0e-4 * scale)


def test_young_and_poisson_gradients_through_the_contact_projection_match_central_differences():
    """dL/dE and dL/dnu of one contact step (an 8x6x2 block pressed onto the frictionless floor,
    63 active contacts) through the Woodbury projection, against central differences of the
    float64 step result. E and nu are global; the tape's per-tet dL/d(mu, lambda) is contracted
    with the float32 Lame parameters each perturbed model actually holds. Both perturbed steps
    keep the base step's active contact set (checked), inside which the contact solution is
    smooth. With friction the reference's projection holds both tangent directions of every
    active contact fixed (adjoint.py:21-25), which is not the derivative of a sliding contact
    (measured 11 % off on this block), so the finite-difference check is frictionless."""
    friction = 0.0
    from newton_solver_diff_phd_b200 import Tape, meshes

    young, poisson, dt = 5.0e4, 0.35, 0.004
    rng = np.random.default_rng(11)

    def step(young_value, poisson_value, taped):
        mu, lam = meshes.lame_from_young(young_value, poisson_value)
        builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
        builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=8, dim_y=6, dim_z=2,
                              cell_x=0.05, cell_y=0.05, cell_z=0.05, density=DENSITY, k_mu=float(mu),
                              k_lambda=float(lam), k_damp=0.0)
        model = builder.finalize("cuda", requires_grad=taped)
        solver = SolverDiffPhD(model, density=DENSITY, frictional_boundary=("planar", (0.0, 0.0, 1.0, 0.0)),
                               friction=friction, max_iterations=4000, abs_tol=1.0e-13, rel_tol=1.0e-12)
        q = model.particle_q.cpu().numpy().astype(np.float64)
        q[:, 2] += 0.0002
        v = np.tile([0.1, 0.0, -0.5], (model.particle_count, 1))
        state_in, state_out = _state(model, q, v), model.state(requires_grad=taped)
        if taped:
            model.tet_materials.grad = torch.zeros_like(model.tet_materials)
            state_in.requires_grad_(True)
            with Tape() as tape:
                solver.step(state_in, state_out, None, None, dt)
            tape.backward(grads={state_out.particle_q: torch.tensor(gq, dtype=torch.float32, device="cuda"),
                                 state_out.particle_qd: torch.tensor(gv, dtype=torch.float32, device="cuda")})
        else:
            solver.step(state_in, state_out, None, None, dt)
        solver.check_status()
        x = solver._x.cpu().numpy()
        q_in = state_in.particle_q.detach().double().cpu().numpy()
        loss = float(np.sum(gq * x) + np.sum(gv * (x - q_in) / dt))
        active = (solver.contact_multipliers.cpu().numpy() > 0).copy()
        lame = model.tet_materials[:, :2].detach().double().cpu().numpy()
        grad = model.tet_materials.grad[:, :2].double().cpu().numpy() if taped else None
        return loss, active, lame, grad

    builder_count = 9 * 7 * 3
    gq = rng.standard_normal((builder_count, 3))
    gv = rng.standard_normal((builder_count, 3))
    _, base_active, _, grad = step(young, poisson, True)
    assert base_active.sum() > 32
    for name, eps in (("young", 1.0e-4 * young), ("poisson", 1.0e-4)):
        results = []
        for sign in (1.0, -1.0):
            e = young + sign * eps if name == "young" else young
            nu = poisson + sign * eps if name == "poisson" else poisson
            results.append(step(e, nu, False))
        (loss_p, active_p, lame_p, _), (loss_m, active_m, lame_m, _) = results
        np.testing.assert_array_equal(active_p, base_active)
        np.testing.assert_array_equal(active_m, base_active)
        measured = loss_p - loss_m
        predicted = float(np.sum(grad * (lame_p - lame_m)))
        assert abs(predicted - measured) <= 1.0e-3 * abs(measured), (name, predicted, measured)
