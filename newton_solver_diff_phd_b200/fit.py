"""Material calibration through the differentiable step: rollout, loss, adjoint, optimizer.

``MaterialFit`` is the reference's two-tetrahedron calibration fixture
(``tests/material_fit_demo.py:46-95``) on this solver: two connected
tetrahedra with Poisson ratio 1/3 and independent log stiffness scales,
recovered from a four-frame trajectory by the rollout adjoint and a
backtracking descent (``optimize``, ``tests/material_fit_demo.py:98-131``).

``CantileverFit`` calibrates the Young's moduli of a batch of Hex8
cantilevers from their final positions: every optimizer iteration is one
batched rollout and one batched adjoint (each one graph launch), the loss and
the chain rule ``dL/dE = dL/dmu dmu/dE + dL/dlambda dlambda/dE`` on the
device, and a PyTorch optimizer on ``log E``.
"""

from __future__ import annotations

from contextlib import nullcontext

import numpy as np
import torch

from . import meshes
from .batch import BatchedSolver
from .model import ModelBuilder
from .scenes import Cantilever, cantilever_model
from .solver import SolverDiffPhD, Tape


class MaterialFit:
    """Five particles, two tetrahedra; particles 0-2 pinned, unit mass on the two free ones."""

    def __init__(self, device="cuda"):
        builder = ModelBuilder(gravity=(0.0, 0.0, 0.0))
        points = ((0, 0, 0), (0.4, 0, 0), (0, 0.4, 0), (0, 0, 0.4), (0.4, 0.4, 0.4))
        for index, point in enumerate(points):
            builder.add_particle(point, (0.0, 0.0, 0.0), 0.0 if index < 3 else 1.0)
        builder.add_tetrahedron(0, 1, 2, 3, k_mu=1200.0, k_lambda=2400.0, k_damp=0.0)
        builder.add_tetrahedron(1, 2, 3, 4, k_mu=1200.0, k_lambda=2400.0, k_damp=0.0)
        self.model = builder.finalize(device, requires_grad=True)
        self.device = self.model.device
        # Unit mass for the free nodes: density times the mean volume (0.016 m^3).
        self.solver = SolverDiffPhD(self.model, density=62.5, material="pd", abs_tol=1e-12, rel_tol=1e-11,
                                    max_iterations=5000)
        initial = self.model.particle_q.detach().cpu().numpy().astype(np.float64)
        initial[3] += [0.025, -0.02, 0.05]
        initial[4] += [-0.04, 0.03, -0.025]
        self.initial = torch.as_tensor(initial, dtype=torch.float32, device=self.device)
        self.reference_scales = np.array([0.7, 2.5], dtype=np.float32)
        self.target = None
        self.target = self.rollout(np.log(self.reference_scales))[0]

    def rollout(self, log_scales, *, gradient=False):
        """``(positions of frames 1..4, loss, dL/dlog_scales or None)``."""
        scales = np.exp(np.asarray(log_scales, dtype=np.float32))
        materials = torch.tensor([[1200.0 * s, 2400.0 * s, 0.0] for s in scales], dtype=torch.float32,
                                 device=self.device)
        with torch.no_grad():
            self.model.tet_materials.copy_(materials)
        self.model.tet_materials.grad = torch.zeros_like(self.model.tet_materials)
        # The solver keeps its weights and factor until told that materials changed.
        self.solver.notify_model_changed()
        states = [self.model.state(requires_grad=gradient) for _ in range(5)]
        with torch.no_grad():
            states[0].particle_q.copy_(self.initial)
        tape = Tape() if gradient else None
        with tape if tape is not None else nullcontext():
            for frame in range(4):
                self.solver.step(states[frame], states[frame + 1], None, None, 0.035)
        # The forward must have converged; the backward's safeguards act silently
        # as in the reference demo, which reads no status.
        if self.solver.read_status() & 7:
            raise RuntimeError("the calibration rollout did not converge")
        outputs = [s.particle_q.detach().clone() for s in states[1:]]
        loss, grad = 0.0, None
        if self.target is not None:
            errors = [(q.double() - t.double()) for q, t in zip(outputs, self.target)]
            loss = float(sum(10000.0 * (e * e).sum() for e in errors))
            if gradient:
                tape.backward(grads={states[frame + 1].particle_q: (20000.0 * errors[frame]).float()
                                     for frame in range(4)})
                # m = c exp(s): dL/ds = sum_k dL/dm_k m_k over mu and lambda.
                dm = self.model.tet_materials.grad[:, :2].double()
                grad = (dm * materials[:, :2].double()).sum(dim=1).cpu().numpy()
        return outputs, loss, grad


def optimize(device="cuda", iterations=15):
    """Backtracking descent on the log scales (``tests/material_fit_demo.py:98-131``)."""
    if iterations < 1:
        raise ValueError("iterations must be positive")
    problem = MaterialFit(device)
    parameters = np.log([1.6, 0.8])
    history = []
    for _ in range(iterations):
        _, loss, gradient = problem.rollout(parameters, gradient=True)
        history.append(loss)
        if loss < 1e-9:
            break
        direction = -gradient / max(1.0, float(np.linalg.norm(gradient)))
        accepted = False
        for step_size in (1.0, 0.5, 0.25, 0.125, 0.0625, 0.03125):
            proposal = parameters + step_size * direction
            _, candidate_loss, _ = problem.rollout(proposal)
            if candidate_loss < loss:
                parameters = proposal
                accepted = True
                break
        if not accepted:
            break
    _, final_loss, _ = problem.rollout(parameters)
    return {"initial_loss": history[0], "final_loss": final_loss, "stiffness_scales": np.exp(parameters).tolist(),
            "reference_scales": problem.reference_scales.tolist(), "iterations": len(history)}


class CantileverFit:
    """Young's moduli of a batch of cantilevers from their final positions.

    ``specs``: the instances (their ``young`` is the ground truth that makes the
    targets); the fit starts from ``young * start_factor`` and runs ``steps``
    steps of ``dt`` per rollout in ``precision``.
    """

    def __init__(self, specs: list[Cantilever], *, steps=5, dt=0.01, start_factor=2.0, precision="fp32+refine",
                 device="cuda"):
        self.specs = list(specs)
        self.steps, self.dt, self.device = int(steps), float(dt), torch.device(device)
        self.parts = [cantilever_model(spec, device=self.device) for spec in self.specs]
        self.solvers = [SolverDiffPhD(model, density=1000.0, hex_mesh=mesh, hex_materials=materials,
                                      precision=precision, adjoint="exact", rel_tol=1e-9, abs_tol=1e-12,
                                      max_iterations=5000)
                        for model, mesh, materials, _ in self.parts]
        self.poisson = np.array([spec.poisson for spec in self.specs])
        self.log_young = torch.tensor(np.log([spec.young for spec in self.specs]) + np.log(start_factor),
                                      dtype=torch.float64, device=self.device, requires_grad=True)
        truth = torch.tensor(np.log([spec.young for spec in self.specs]), dtype=torch.float64, device=self.device)
        self.target = self._final(truth).detach()

    def _set_young(self, log_young: torch.Tensor):
        young = torch.exp(log_young.detach()).cpu().numpy()
        for solver, e, nu in zip(self.solvers, young, self.poisson):
            mu, lam = meshes.lame_from_young(e, nu)
            solver.hex_materials[:, 0] = float(mu)
            solver.hex_materials[:, 1] = float(lam)
            solver.notify_model_changed()

    def _batch(self, log_young):
        self._set_young(log_young)
        batch = BatchedSolver(self.solvers, self.dt)
        q0 = batch.concat([model.particle_q for model, _, _, _ in self.parts])
        forces = batch.concat([torch.as_tensor(f, device=self.device) for _, _, _, f in self.parts])
        return batch, q0, forces

    def _final(self, log_young):
        batch, q0, forces = self._batch(log_young)
        q, _, _ = batch.rollout(q0, torch.zeros_like(q0), forces, self.steps)
        return q[-1].double()

    def step(self, optimizer: torch.optim.Optimizer) -> float:
        """One optimizer iteration: batched rollout, loss, batched adjoint, dL/dlog E, optimizer step."""
        batch, q0, forces = self._batch(self.log_young)
        q, _, x = batch.rollout(q0, torch.zeros_like(q0), forces, self.steps)
        error = q[-1].double() - self.target
        loss = float((error * error).sum())
        _, _, _, gm, _ = batch.backward(x, (2.0 * error).to(q.dtype))
        eo = batch.element_offsets
        nu = torch.as_tensor(self.poisson, dtype=torch.float64, device=self.device)
        young = torch.exp(self.log_young.detach())
        dmu = 1.0 / (2.0 * (1.0 + nu))
        dlam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        index = torch.as_tensor(np.repeat(np.arange(batch.count), np.diff(eo)), device=self.device)
        per_element = gm[:, 0] * dmu[index] + gm[:, 1] * dlam[index]
        grad_e = torch.zeros(batch.count, dtype=torch.float64, device=self.device).index_add_(0, index, per_element)
        optimizer.zero_grad()
        self.log_young.grad = grad_e * young
        optimizer.step()
        return loss
