"""Parity of the Tet4 block workload at its full size against the CPU oracle.

The workload is the benchmark's: a 32 x 8 x 8 block of 0.01 m cubes in five
tetrahedra each (10,240 Tet4, 2,673 particles), per-tet E log-uniform in
[1e5, 1e7] Pa, nu 0.4, gravity, the x = 0 face pinned, 50 steps of dt 5e-3 at
rel 1e-6, and the loss ``|q_50 - target|^2``. ``tests/golden/tet_block_rollout.npz``
holds the oracle's rollout (``tests/golden/make_tet_block_rollout.py``: the
reference algorithm on the CPU with the reference's exact inverse factor):
the state every second step, every step's iteration count, the final
positions and dL/dE of every tet.

Tolerances (the precision contract of the path): positions within 1e-6
relative in the norm of the solver's own stop rule (|x - x_ref| / |x_ref|,
2-norm over all particles), gradients within 1e-4 relative (2-norm over all
tets); the finite-difference check uses central differences at eps = 1e-4 E
on 16 seeded tets.
"""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import ModelBuilder, SolverDiffPhD, meshes
from newton_solver_diff_phd_b200.rollout import Rollout
from tests.helpers import golden

pytestmark = pytest.mark.gpu

NX, NY, NZ, EDGE, DT, STEPS = 32, 8, 8, 0.01, 5.0e-3, 50


def block(state_dtype=torch.float32, precision="fp64", rel_tol=1.0e-6, abs_tol=1.0e-9, young=None):
    vertices, tets, _ = meshes.tet_grid(NX, NY, NZ, EDGE)
    rng = np.random.default_rng(0)
    seeded = np.exp(rng.uniform(np.log(1.0e5), np.log(1.0e7), len(tets)))
    target = vertices + rng.normal(0.0, 1.0e-3, vertices.shape)
    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=NX, dim_y=NY, dim_z=NZ,
                          cell_x=EDGE, cell_y=EDGE, cell_z=EDGE, density=1000.0, k_mu=1.0, k_lambda=1.0, k_damp=0.0,
                          fix_left=True)
    model = builder.finalize("cuda")
    mu, lam = meshes.lame_from_young(seeded if young is None else young, 0.4)
    with torch.no_grad():
        model.tet_materials.copy_(torch.tensor(np.column_stack((mu, lam, np.zeros_like(mu))), dtype=torch.float32))
    solver = SolverDiffPhD(model, density=1000.0, rel_tol=rel_tol, abs_tol=abs_tol, adjoint="exact",
                           precision=precision, state_dtype=state_dtype)
    return model, solver, torch.tensor(target.astype(np.float32), device="cuda"), seeded


def run(model, solver, target, with_gradient=True):
    """Rollout, loss and dL/d(mu, lambda) per tet; the positions after every step."""
    driver = Rollout(solver, STEPS, DT)
    dtype = solver.state_dtype
    q0 = model.particle_q.to(dtype)
    final = driver.forward(q0, torch.zeros_like(q0))
    positions = [driver.checkpoints[t + 1].particle_q.double().cpu().numpy() for t in range(STEPS)]
    diff = final.particle_q.double() - target.double()
    loss = float((diff ** 2).sum())
    if not with_gradient:
        solver.check_status()
        return positions, loss, None
    _, _, _, gml = driver.backward((2.0 * diff).to(dtype).contiguous())
    solver.check_status()
    return positions, loss, gml.cpu().numpy()


def relative(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def young_gradient(gml):
    dmu, dlam = 1.0 / (2.0 * 1.4), 0.4 / (1.4 * 0.2)
    return gml[:, 0] * dmu + gml[:, 1] * dlam


def test_fp64_rollout_and_gradient_match_the_oracle_at_full_size():
    g = golden("tet_block_rollout.npz")
    model, solver, target, _ = block()
    iterations = []
    driver = Rollout(solver, STEPS, DT)
    # Per-step iteration counts: step the rollout's states one at a time.
    states = driver.checkpoints
    states[0].particle_q.copy_(model.particle_q)
    states[0].particle_qd.zero_()
    for t in range(STEPS):
        states[t].particle_f.zero_()
        solver.step(states[t], states[t + 1], None, None, DT, record=driver.records[t])
        iterations.append(int(solver.iterations[0]))
    solver.check_status()
    expected_iterations = g["iterations"]
    difference = np.array(iterations) - expected_iterations
    errors = {int(t): relative(states[t].particle_q.double().cpu().numpy(), g["q_in"][k + 1])
              for k, t in enumerate(g["steps"][1:])}
    final = states[STEPS].particle_q.double().cpu().numpy()
    errors[STEPS] = relative(final, g["q_final"])
    # Positions: within 1e-6 of the oracle at every recorded step. The
    # iteration counts agree step by step except in the few steps whose stop
    # test sits at its bound for many iterations (the beam's swing-back
    # bursts); the totals agree within one percent.
    assert max(errors.values()) <= 1e-6, errors
    assert np.count_nonzero(difference) <= 5, difference.tolist()
    assert abs(int(np.sum(iterations)) - int(np.sum(expected_iterations))) <= 0.01 * np.sum(expected_iterations)
    diff = states[STEPS].particle_q.double() - target.double()
    _, _, _, gml = driver.backward((2.0 * diff).float().contiguous())
    solver.check_status()
    grad_e = young_gradient(gml.cpu().numpy())
    assert relative(grad_e, g["grad_young"]) <= 1e-4


def test_fp32_refine_matches_fp64_at_full_size():
    model, solver64, target, _ = block()
    x64, _, g64 = run(model, solver64, target)
    model32, solver32, target32, _ = block(precision="fp32+refine")
    x32, _, g32 = run(model32, solver32, target32)
    errors = [relative(a, b) for a, b in zip(x32, x64)]
    assert max(errors) <= 1e-6, errors
    assert relative(young_gradient(g32), young_gradient(g64)) <= 1e-4


def test_gradient_wrt_young_matches_central_differences_on_16_tets():
    # float64 states (float32 state rounding between steps would swamp a
    # 1e-4 perturbation) and a tight stop rule on both passes. The materials
    # the solver reads are float32 (Newton's tet_materials), so the
    # difference of the two perturbed losses is compared with the adjoint's
    # prediction for the perturbation those float32 values actually make.
    # The losses carry the forward solve's stopping error, measured here as
    # the loss change from rel 1e-12 to rel 1e-13; each tet must agree to
    # 1e-4 relative above twice that noise.
    options = dict(state_dtype=torch.float64, rel_tol=1.0e-12, abs_tol=1.0e-14)
    model, solver, target, young = block(**options)
    _, base_loss, gml = run(model, solver, target)
    del solver
    m, s, t, _ = block(state_dtype=torch.float64, rel_tol=1.0e-13, abs_tol=1.0e-15)
    _, tight_loss, _ = run(m, s, t, with_gradient=False)
    noise = abs(tight_loss - base_loss)
    del s
    rng = np.random.default_rng(7)
    chosen = rng.choice(len(young), 16, replace=False)
    measured, predicted = [], []
    for e in chosen:
        losses, lame = [], []
        for sign in (1.0, -1.0):
            perturbed = young.copy()
            perturbed[e] *= 1.0 + sign * 1.0e-4
            m, s, t, _ = block(young=perturbed, **options)
            _, loss, _ = run(m, s, t, with_gradient=False)
            losses.append(loss)
            lame.append(m.tet_materials[e, :2].double().cpu().numpy())
            del s
        measured.append(losses[0] - losses[1])
        predicted.append(float(gml[e] @ (lame[0] - lame[1])))
    measured, predicted = np.array(measured), np.array(predicted)
    bound = 1e-4 * np.abs(measured) + 2.0 * noise
    assert np.all(np.abs(predicted - measured) <= bound), (predicted, measured, noise)
