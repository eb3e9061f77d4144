"""Multi-step rollouts with gradients: the ``torch.autograd.Function`` boundary.

The reference differentiates rollouts by recording every step on a
``wp.Tape`` (``tests/material_fit_demo.py:70-96``): one ``StepRecord`` per step
(``adjoint.py:809-841``) and a reverse replay of the per-step backward passes.
:class:`Rollout` does the same with preallocated device buffers (no host
synchronization inside a rollout), and optional step checkpointing: with
``checkpoint_every = k`` only every k-th state is kept and each segment's
forward steps are recomputed during the backward pass. The forward is
bitwise deterministic, so recomputed positions equal the recorded ones.

:func:`rollout` wraps it as a ``torch.autograd.Function`` mapping
``(q0, qd0, forces, mu_lambda)`` to the final positions, with gradients for
the initial state, the applied forces and the per-element Lame parameters
(and hence Young's modulus and Poisson ratio through torch).
"""

from __future__ import annotations

import torch

from .model import State


class Rollout:
    """Preallocated buffers of a ``steps``-long rollout of one solver at a fixed ``dt``."""

    def __init__(self, solver, steps: int, dt: float, checkpoint_every: int = 1):
        if steps < 1 or checkpoint_every < 1:
            raise ValueError("steps and checkpoint_every must be positive")
        self.solver = solver
        self.steps = int(steps)
        self.dt = float(dt)
        self.every = int(checkpoint_every)
        n = solver._n
        device = solver.device
        dtype = solver.state_dtype
        kept = self.steps + 1 if self.every == 1 else self.steps // self.every + 2

        def state():
            s = State(
                torch.zeros((n, 3), dtype=dtype, device=device),
                torch.zeros((n, 3), dtype=dtype, device=device),
                torch.zeros((n, 3), dtype=dtype, device=device),
            )
            for tensor in (s.particle_q, s.particle_qd, s.particle_f):
                tensor.grad = torch.zeros_like(tensor)
            return s

        self.checkpoints = [state() for _ in range(kept)]
        # Records of the converged positions: all steps, or one segment when checkpointing.
        self.records = torch.zeros((self.steps if self.every == 1 else self.every, n, 3), dtype=torch.float64,
                                   device=device)
        self.segment = [state() for _ in range(self.every + 1)] if self.every > 1 else None
        self.force_grad = torch.zeros((self.steps, n, 3), dtype=dtype, device=device)
        self.material_grad = torch.zeros((solver._element_count, 2), dtype=torch.float64, device=device)
        self._forces = None

    def _force(self, t):
        forces = self._forces
        if forces is None:
            return None
        return forces[t] if forces.dim() == 3 else forces

    def forward(self, q0: torch.Tensor, qd0: torch.Tensor, forces: torch.Tensor | None = None) -> State:
        """Run all steps; returns the final state. ``forces`` is ``(N,3)`` or ``(steps,N,3)`` in the state dtype."""
        self._forces = forces
        first = self.checkpoints[0]
        first.particle_q.copy_(q0)
        first.particle_qd.copy_(qd0)
        current = first
        for t in range(self.steps):
            force = self._force(t)
            current.particle_f.copy_(force) if force is not None else current.particle_f.zero_()
            if self.every == 1:
                target = self.checkpoints[t + 1]
                record = self.records[t]
            else:
                k = (t + 1) // self.every if (t + 1) % self.every == 0 else None
                target = self.checkpoints[k] if k is not None else self.segment[(t % self.every) + 1]
                record = self.records[t % self.every]
            self.solver.step(current, target, None, None, self.dt, record=record)
            current = target
        if self.every > 1 and self.steps % self.every:
            last = self.checkpoints[-1]
            last.particle_q.copy_(current.particle_q)
            last.particle_qd.copy_(current.particle_qd)
            current = last
        return current

    def backward(self, grad_q: torch.Tensor, grad_qd: torch.Tensor | None = None, materials: bool = True):
        """Reverse pass seeded with the gradients of the final positions (and velocities).

        Returns ``(dL/dq0, dL/dqd0, dL/dforces (steps,N,3), dL/d[mu,lambda] (E,2))``.
        """
        solver = self.solver
        self.material_grad.zero_()
        material = _MaterialSink(self.material_grad) if materials else None
        if self.every == 1:
            states = self.checkpoints
            for s in states:
                s.particle_q.grad.zero_()
                s.particle_qd.grad.zero_()
                s.particle_f.grad.zero_()
            states[-1].particle_q.grad.copy_(grad_q)
            if grad_qd is not None:
                states[-1].particle_qd.grad.copy_(grad_qd)
            for t in reversed(range(self.steps)):
                solver.backward_step(self.records[t], self.dt, states[t], states[t + 1], materials=material)
                self.force_grad[t].copy_(states[t].particle_f.grad)
            first = states[0]
            return first.particle_q.grad, first.particle_qd.grad, self.force_grad, self.material_grad
        # Checkpointed: recompute each segment forward from its checkpoint, then reverse it.
        segments = [(s, min(s + self.every, self.steps)) for s in range(0, self.steps, self.every)]
        carry_q = grad_q.clone()
        carry_qd = torch.zeros_like(grad_q) if grad_qd is None else grad_qd.clone()
        for index in reversed(range(len(segments))):
            start, stop = segments[index]
            chain = [self.checkpoints[index]] + self.segment[1:stop - start + 1]
            for t in range(start, stop):
                state = chain[t - start]
                force = self._force(t)
                state.particle_f.copy_(force) if force is not None else state.particle_f.zero_()
                solver.step(state, chain[t - start + 1], None, None, self.dt, record=self.records[t - start])
            for s in chain:
                s.particle_q.grad.zero_()
                s.particle_qd.grad.zero_()
                s.particle_f.grad.zero_()
            chain[-1].particle_q.grad.copy_(carry_q)
            chain[-1].particle_qd.grad.copy_(carry_qd)
            for t in reversed(range(start, stop)):
                solver.backward_step(self.records[t - start], self.dt, chain[t - start], chain[t - start + 1],
                                     materials=material)
                self.force_grad[t].copy_(chain[t - start].particle_f.grad)
            carry_q = chain[0].particle_q.grad.clone()
            carry_qd = chain[0].particle_qd.grad.clone()
        return carry_q, carry_qd, self.force_grad, self.material_grad


class _MaterialSink:
    """Adapter: the solver adds ``dL/d[mu, lambda]`` into ``grad`` (float64 here)."""

    def __init__(self, grad):
        self.grad = grad


class _RolloutFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, driver, q0, qd0, forces, mu_lambda):
        final = driver.forward(q0.detach(), qd0.detach(), None if forces is None else forces.detach())
        ctx.driver = driver
        ctx.has_forces = forces is not None
        ctx.forces_shape = None if forces is None else forces.shape
        return final.particle_q.clone(), final.particle_qd.clone()

    @staticmethod
    def backward(ctx, grad_q, grad_qd):
        driver = ctx.driver
        gq0, gqd0, gforces, gmaterials = driver.backward(grad_q.contiguous(), None if grad_qd is None else grad_qd.contiguous())
        grad_forces = None
        if ctx.has_forces:
            grad_forces = gforces.sum(dim=0) if len(ctx.forces_shape) == 2 else gforces.clone()
        return None, gq0.clone(), gqd0.clone(), grad_forces, gmaterials.clone()


def rollout(driver: Rollout, q0, qd0, forces=None, mu_lambda=None):
    """Differentiable rollout ``(q0, qd0, forces, mu_lambda) -> (q_T, qd_T)``.

    ``mu_lambda`` must equal the materials the solver was built with (it is
    the differentiation handle for the per-element Lame parameters; changing
    materials requires ``solver.notify_model_changed`` and a new build).
    """
    if mu_lambda is None:
        mu_lambda = torch.zeros((driver.solver._element_count, 2), dtype=torch.float64, device=driver.solver.device)
    return _RolloutFunction.apply(driver, q0, qd0, forces, mu_lambda)
