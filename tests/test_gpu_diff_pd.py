"""The DiffPD ``pd_eigen`` forward step on the B200 path against the reference's own oracle.

``tests/golden/diff_pd.npz`` holds the reference's ``tests/reference_oracle_diff_pd.py``
run on the scenes of its ``tests/test_diff_pd_solver.py`` (free fall of a
deformed block, a pinned cantilever, planar and arc penalty contacts, a long
step whose L-BFGS history wraps and whose line search halves, external
forces). As in the reference test, every step starts from the same float32
state on both sides, so the iteration counts must be equal and the float64
positions agree to rounding: within 1e-10 m, since the device sums in a
different order and the long step's 160 L-BFGS iterations carry those
roundings along (1.1e-11 m measured).
"""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import ModelBuilder, SolverDiffPD, Tape
from newton_solver_diff_phd_b200.solver import ConvergenceError
from tests.helpers import golden

DENSITY, COROTATED, VOLUME, DT = 1000.0, 4.0e4, 5.0e4, 1.0e-2
GRAVITY = (0.0, 0.0, -9.81)
POSITION_TOL = 1.0e-10
ARC_START = (np.sin(np.radians(30.0)), 0.0, -np.cos(np.radians(30.0)))
SCENES = {
    "free_fall": ((0.0, 0.0, 1.0), False, []),
    "pinned": ((0.0, 0.0, 1.0), True, []),
    "planar": ((-0.15, -0.1, -0.005), False, [("planar_contact", [0.0, 0.0, 2.0, 0.0, 3, 1.0e6, 1.0, 0.1])]),
    "arc": ((-0.15, -0.1, -0.005), False,
            [("arc_contact", [0.0, 0.0, 1.0, 0.0, 2.0, 0.0, *ARC_START, 1.0, np.radians(32.0), 3, 1.0e6, 1.0, 0.1])]),
    "history": ((0.0, 0.0, 1.0), False, []),
    "external": ((0.0, 0.0, 1.0), False, []),
}


def grid(origin=(0.0, 0.0, 1.0), fix_left=False, device="cuda"):
    builder = ModelBuilder(gravity=GRAVITY)
    builder.add_soft_grid(pos=origin, rot=None, vel=(0.0, 0.0, 0.0), dim_x=3, dim_y=2, dim_z=2, cell_x=0.1, cell_y=0.1,
                          cell_z=0.1, density=DENSITY, k_mu=2.0e4, k_lambda=5.0e4, k_damp=0.0, fix_left=fix_left)
    return builder.finalize(device)


@pytest.mark.gpu
@pytest.mark.parametrize("scene", list(SCENES))
def test_steps_match_the_reference_oracle(scene):
    g = golden("diff_pd.npz")
    key = scene + "__"
    origin, fix_left, forces = SCENES[scene]
    model = grid(origin, fix_left)
    np.testing.assert_array_equal(model.tet_indices.cpu().numpy().reshape(-1, 4), g[key + "tets"])
    solver = SolverDiffPD(model, density=DENSITY, corotated_stiffness=COROTATED, volume_stiffness=VOLUME,
                          state_forces=forces, gravity=GRAVITY)
    dt = float(g[key + "dt"])
    state_in, state_out = model.state(), model.state()
    for t in range(len(g[key + "iterations"])):
        state_in.particle_q.copy_(torch.as_tensor(g[key + "q_in"][t]))
        state_in.particle_qd.copy_(torch.as_tensor(g[key + "v_in"][t]))
        state_in.particle_f.copy_(torch.as_tensor(g[key + "f"][t]))
        solver.step(state_in, state_out, None, None, dt)
        status = solver.read_status()
        assert status & ~4 == 0, status  # bit 4 (all halvings used) is informational
        assert int(solver.iterations[0]) == int(g[key + "iterations"][t]), t
        np.testing.assert_allclose(solver.positions.cpu().numpy(), g[key + "q_out"][t], rtol=0.0, atol=POSITION_TOL)
        np.testing.assert_allclose(solver.velocities.cpu().numpy(), g[key + "v_out"][t], rtol=0.0,
                                   atol=POSITION_TOL / dt)
        expected = g[key + "q_out"][t].astype(np.float32)
        np.testing.assert_array_max_ulp(state_out.particle_q.cpu().numpy(), expected, maxulp=1)


@pytest.mark.gpu
def test_pinned_particles_keep_their_positions():
    model = grid(fix_left=True)
    solver = SolverDiffPD(model, density=DENSITY, corotated_stiffness=COROTATED, volume_stiffness=VOLUME)
    pinned = model.particle_inv_mass.cpu().numpy() == 0
    start = model.particle_q.cpu().numpy()
    states = [model.state(), model.state()]
    for _ in range(3):
        solver.step(states[0], states[1], None, None, DT)
        states.reverse()
    solver.check_status()
    q = states[0].particle_q.cpu().numpy()
    np.testing.assert_array_equal(q[pinned], start[pinned])
    np.testing.assert_array_equal(states[0].particle_qd.cpu().numpy()[pinned], 0.0)
    assert q[~pinned, 2].min() < start[~pinned, 2].min()


@pytest.mark.gpu
def test_max_pd_iter_raises_convergence_error():
    g = golden("diff_pd.npz")
    model = grid()
    solver = SolverDiffPD(model, density=DENSITY, corotated_stiffness=COROTATED, volume_stiffness=VOLUME,
                          gravity=GRAVITY, max_pd_iter=1)
    state = model.state()
    state.particle_q.copy_(torch.as_tensor(g["free_fall__q_in"][0]))
    solver.step(state, model.state(), None, None, DT)
    with pytest.raises(ConvergenceError):
        solver.check_status()
    solver.check_status()


@pytest.mark.gpu
def test_singular_deformation_gradient_raises():
    model = grid()
    solver = SolverDiffPD(model, density=DENSITY, corotated_stiffness=COROTATED, volume_stiffness=VOLUME)
    state = model.state()
    state.particle_q[:, 2] = 1.0
    solver.step(state, model.state(), None, None, DT)
    assert int(solver.iterations[0]) == 0
    with pytest.raises(ValueError, match="Singular F"):
        solver.check_status()


@pytest.mark.gpu
def test_tape_and_contacts_are_rejected():
    model = grid()
    solver = SolverDiffPD(model, density=DENSITY, corotated_stiffness=COROTATED)
    with Tape(), pytest.raises(NotImplementedError):
        solver.step(model.state(), model.state(), None, None, DT)
    with pytest.raises(NotImplementedError):
        solver.step(model.state(), model.state(), None, object(), DT)
    state = model.state()
    with pytest.raises(ValueError):
        solver.step(state, state, None, None, DT)
    for dt in (0.0, -1.0, np.nan):
        with pytest.raises(ValueError):
            solver.step(state, model.state(), None, None, dt)


def test_invalid_configurations_are_rejected():
    model = grid(device="cpu")
    invalid = [
        {"density": 0.0},
        {"density": np.nan},
        {"corotated_stiffness": -1.0},
        {"volume_stiffness": np.inf},
        {"max_pd_iter": 0},
        {"max_ls_iter": 0},
        {"max_ls_iter": 2.5},
        {"bfgs_history_size": 1},
        {"abs_tol": -1.0},
        {"rel_tol": np.nan},
        {"gravity": (0.0, 1.0)},
        {"rest_positions": np.zeros((2, 3))},
        {"state_forces": [("hydrodynamics", [0.0] * 8)]},
        {"state_forces": [("planar_contact", [0.0] * 7)]},
        {"state_forces": [("planar_contact", [0.0, 0.0, 1.0e-6, 0.0, 3, 1.0, 1.0, 1.0])]},
        {"state_forces": [("arc_contact", [0.0] * 15)]},
        {"state_forces": [("planar_contact",)]},
    ]
    for options in invalid:
        arguments = {"density": DENSITY, **options}
        with pytest.raises(ValueError):
            SolverDiffPD(model, **arguments)


@pytest.mark.gpu
def test_a_streamed_factor_with_a_staged_vector_gives_the_same_steps():
    """96 blocks instead of 148 on the 32x8x8 block: the larger slices of S and S^T no longer fit
    in shared memory, so the products stream the factor and stage their input vector with
    16-byte loads (every DiffPD vector starts on a 256-byte boundary for that; with the vectors
    packed 3n doubles apart this launch stopped on a misaligned address); the steps follow the
    default launch's within rounding."""
    results = []
    for blocks in (0, 96):
        builder = ModelBuilder(gravity=GRAVITY)
        builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=32, dim_y=8, dim_z=8,
                              cell_x=0.01, cell_y=0.01, cell_z=0.01, density=DENSITY, k_mu=2.0e4, k_lambda=5.0e4,
                              k_damp=0.0, fix_left=True)
        model = builder.finalize("cuda")
        solver = SolverDiffPD(model, density=DENSITY, corotated_stiffness=COROTATED, volume_stiffness=VOLUME,
                              gravity=GRAVITY, blocks=blocks)
        states = [model.state(), model.state()]
        iterations = []
        for _ in range(3):
            solver.step(states[0], states[1], None, None, DT)
            solver.check_status()
            iterations.append(int(solver.iterations[0]))
            states.reverse()
        results.append((solver.positions.cpu().numpy().copy(), iterations))
    assert all(abs(a - b) <= 1 for a, b in zip(results[0][1], results[1][1]))
    np.testing.assert_allclose(results[1][0], results[0][0], rtol=0.0, atol=1.0e-8)
