"""Multi-step rollouts: checkpointing and gradients through the autograd boundary.

The Young's-modulus gradient of a rollout loss is checked against central
finite differences on a small heterogeneous block with float64 states (float32
states round positions to ~2e-9 m between steps, far above the response to a
small change of E). The step is 1e-3 of E: at 1e-4 the solver's own
convergence noise is a few 1e-4 of the difference.
"""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import ModelBuilder, SolverDiffPhD, meshes
from newton_solver_diff_phd_b200.rollout import Rollout, rollout

pytestmark = pytest.mark.gpu

TIGHT = {"max_iterations": 5000, "abs_tol": 1e-13, "rel_tol": 1e-12}


def _block(seed=0, nx=4, ny=2, nz=2):
    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0, 0, 0), rot=None, vel=(0, 0, 0), dim_x=nx, dim_y=ny, dim_z=nz, cell_x=0.01, cell_y=0.01,
                          cell_z=0.01, density=1000.0, k_mu=1.0, k_lambda=1.0, k_damp=0.0, fix_left=True)
    model = builder.finalize("cuda")
    rng = np.random.default_rng(seed)
    young = np.exp(rng.uniform(np.log(1e5), np.log(1e7), model.tet_count))
    return model, young


def _set_young(model, young, nu=0.4):
    mu, lam = meshes.lame_from_young(young, nu)
    with torch.no_grad():
        model.tet_materials.copy_(torch.tensor(np.column_stack((mu, lam, np.zeros_like(mu))), dtype=torch.float32))
    # The solver reads float32 materials, as Newton stores them.
    stored = model.tet_materials.cpu().numpy().astype(np.float64)
    return stored[:, 0], stored[:, 1]


def test_checkpointed_rollout_is_bitwise_equal_to_the_plain_one():
    model, young = _block()
    _set_young(model, young)
    results = []
    for every in (1, 3):
        solver = SolverDiffPhD(model, density=1000.0, adjoint="exact", rel_tol=1e-8)
        driver = Rollout(solver, 7, 5e-3, checkpoint_every=every)
        q0 = model.particle_q.clone()
        final = driver.forward(q0, torch.zeros_like(q0))
        gq = torch.ones_like(q0)
        gq0, gqd0, gforces, gmaterials = driver.backward(gq)
        solver.check_status()
        results.append((final.particle_q.clone(), gq0.clone(), gforces.clone(), gmaterials.clone()))
    for a, b in zip(results[0], results[1]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("adjoint_solver", ["cg", "fixed_point"])
def test_young_modulus_gradient_matches_finite_differences(adjoint_solver):
    model, young = _block()
    steps, dt, nu = 5, 5e-3, 0.4
    rng = np.random.default_rng(3)
    target = model.particle_q.cpu().numpy().astype(np.float64) + rng.normal(0.0, 1e-3, (model.particle_count, 3))
    target_t = torch.tensor(target, device="cuda")

    def loss_of(young_values, with_grad):
        mu, lam = _set_young(model, young_values, nu)
        # float64 states: a 1e-4 relative change of E moves positions by ~1e-10 m,
        # far below the float32 state rounding (~2e-9 m) between steps.
        solver = SolverDiffPhD(model, density=1000.0, adjoint="exact", adjoint_solver=adjoint_solver,
                               state_dtype=torch.float64, **TIGHT)
        driver = Rollout(solver, steps, dt)
        q0 = model.particle_q.double()
        e = torch.tensor(young_values, dtype=torch.float64, device="cuda", requires_grad=with_grad)
        mu_t = e / (2.0 * (1.0 + nu))
        lam_t = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        q_t, _ = rollout(driver, q0, torch.zeros_like(q0), None, torch.stack((mu_t, lam_t), dim=1))
        # Loss on the float64 recorded positions of the last step (no float32 output rounding).
        loss = ((q_t - target_t) ** 2).sum()
        if with_grad:
            loss.backward()
        solver.check_status()
        return float(loss.detach()), (e.grad.cpu().numpy() if with_grad else None)

    _, grad = loss_of(young, True)
    scale = np.abs(grad).max()
    largest = np.argsort(-np.abs(grad))[:4]
    random = np.random.default_rng(5).choice(len(young), 4, replace=False)
    for element in np.concatenate((largest, random)):
        eps = 1e-3 * young[element]
        plus, minus = young.copy(), young.copy()
        plus[element] += eps
        minus[element] -= eps
        numeric = (loss_of(plus, False)[0] - loss_of(minus, False)[0]) / (2 * eps)
        # The reference's FD tolerance, 2e-4 relative, for the dominant entries;
        # small entries sit at the FD noise floor of a 1e-12-converged solve, so
        # they get an absolute floor of 2e-4 of the largest entry.
        assert abs(grad[element] - numeric) <= 2e-4 * max(abs(numeric), scale * (element not in largest)), (
            element, grad[element], numeric)


def test_cg_and_fixed_point_adjoints_agree():
    model, young = _block(seed=1)
    _set_young(model, young)
    grads = []
    for adjoint_solver in ("cg", "fixed_point"):
        solver = SolverDiffPhD(model, density=1000.0, adjoint="exact", adjoint_solver=adjoint_solver, **TIGHT)
        driver = Rollout(solver, 4, 5e-3)
        q0 = model.particle_q.clone()
        driver.forward(q0, torch.zeros_like(q0))
        gq0, _, _, gmaterials = driver.backward(torch.ones_like(q0))
        solver.check_status()
        grads.append((gq0.cpu().numpy().astype(np.float64), gmaterials.cpu().numpy()))
    np.testing.assert_allclose(grads[0][0], grads[1][0], rtol=0, atol=1e-6 * np.abs(grads[1][0]).max())
    np.testing.assert_allclose(grads[0][1], grads[1][1], rtol=0, atol=1e-6 * np.abs(grads[1][1]).max())
