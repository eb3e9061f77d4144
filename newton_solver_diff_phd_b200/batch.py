"""Batched rollouts: many independent :class:`SolverDiffPhD` instances in one CUDA graph.

The reference advances one Newton model per ``SolverDiffPhD.step`` call
(``src/newton_solver_diff_phd/_src/solvers/diff_phd/solver.py:689-786``). For
many small meshes of uneven size that leaves a B200 idle, so this module runs
the steps of every instance together: per PD step, each phase of the
local/global iteration is one kernel over the work of all instances still
iterating, repeated by a device-side loop of a CUDA graph. An instance whose step has
passed its convergence gate writes it out and starts its next step at once,
so instances never wait for each other between steps. Each instance keeps its own
materials, tolerances, iteration limit, Anderson window and factor; the
result of an instance equals its single-instance ``step`` to rounding.

States are concatenated: instance ``i`` owns particles
``particle_offsets[i]:particle_offsets[i+1]`` of every ``(P, 3)`` array.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .solver import SolverDiffPhD, _stream


SCHEDULES = {"teams": _lib.BATCH_TEAMS, "phases": _lib.BATCH_PHASES}


class BatchedSolver:
    """A fixed set of solvers stepped together (``pd_batch_*`` in ``include/pd_b200.h``).

    Every solver is built for ``dt`` here (as its first ``step`` would). The
    solvers must share device, precision and state dtype, must outlive the
    batch, and must not be stepped on their own while a batched rollout runs.
    A new batch over the same solvers re-plans them: only the newest batch of
    a set of solvers may be used. Dirichlet targets and Tet4 muscle
    activations are not supported.

    ``schedule="teams"`` (default) runs each instance's whole rollout on a
    team of blocks of one persistent launch, with the single-instance step
    and adjoint bodies; ``"phases"`` runs per-phase kernels over all
    instances in a graph loop (forward only).
    """

    def __init__(self, solvers: list[SolverDiffPhD], dt: float, *, schedule: str = "teams",
                 team_nnz: int = 65536, team_samples: int = 512, svd_warm_start: bool = True,
                 task_nnz: int = 32768, run_gap: int = 2, local_cells: int = 64, measured=None):
        if not solvers:
            raise ValueError("BatchedSolver needs at least one solver")
        if not np.isfinite(dt) or dt <= 0:
            raise ValueError("dt must be finite and positive")
        if schedule not in SCHEDULES:
            raise ValueError("schedule must be 'teams' or 'phases'")
        self.schedule = schedule
        first = solvers[0]
        for solver in solvers:
            if not isinstance(solver, SolverDiffPhD):
                raise TypeError("BatchedSolver takes SolverDiffPhD instances")
            if solver.device != first.device or solver.state_dtype != first.state_dtype:
                raise ValueError("batched solvers must share device and state dtype")
        self.dt = float(dt)
        self.device = first.device
        self.state_dtype = first.state_dtype
        for solver in solvers:
            if solver._model_changed or solver._factor_key != self.dt:
                solver._build(self.dt)
            solver._sync_hex_targets()
        gravities = np.stack([s._gravity for s in solvers])
        if not np.all(gravities == gravities[0]):
            raise ValueError("batched solvers must share gravity")
        self._gravity = np.ascontiguousarray(gravities[0])
        self.solvers = list(solvers)
        self._lib = _lib.library()
        handles = (ctypes.c_void_p * len(solvers))(*[ctypes.cast(s._handle, ctypes.c_void_p).value for s in solvers])
        options = _lib.PdBatchOptions(int(svd_warm_start), int(task_nnz), int(run_gap), int(local_cells),
                                      SCHEDULES[schedule], int(team_nnz), int(team_samples))
        if measured is not None:
            # (forward durations [us], iterations, team sizes[, adjoint durations [us]]) per instance
            # of a previous rollout (measurement()).
            if len(measured) not in (3, 4):
                raise ValueError("measured is (durations, iterations, team sizes[, adjoint durations])")
            self._measured = (np.ascontiguousarray(measured[0], dtype=np.float64),
                              np.ascontiguousarray(measured[1], dtype=np.int32),
                              np.ascontiguousarray(measured[2], dtype=np.int32))
            if len(measured) == 4 and measured[3] is not None:
                self._measured += (np.ascontiguousarray(measured[3], dtype=np.float64),)
            if any(len(a) != len(solvers) for a in self._measured):
                raise ValueError("measured costs need one entry per instance")
            options.measured_us, options.measured_iterations, options.measured_team = (
                _lib.ptr(a) for a in self._measured[:3])
            if len(self._measured) == 4:
                options.measured_adjoint_us = _lib.ptr(self._measured[3])
        handle = ctypes.c_void_p()
        _lib.check(self._lib.pd_batch_create(ctypes.cast(handles, ctypes.c_void_p), len(solvers), ctypes.byref(options), ctypes.byref(handle)))
        self._handle = handle
        particles = np.zeros(len(solvers) + 1, np.int64)
        elements = np.zeros(len(solvers) + 1, np.int64)
        _lib.check(self._lib.pd_batch_layout(self._handle, _lib.ptr(particles), _lib.ptr(elements)))
        self.particle_offsets = particles
        self.element_offsets = elements
        self.particle_count = int(particles[-1])
        self._steps = 0

    @property
    def count(self) -> int:
        return len(self.solvers)

    def factor_stats(self) -> dict:
        values, runs = ctypes.c_int64(), ctypes.c_int64()
        tasks = np.zeros(4, np.int64)
        _lib.check(self._lib.pd_batch_factor_stats(self._handle, ctypes.byref(values), ctypes.byref(runs),
                                                   _lib.ptr(tasks)))
        return {"values": values.value, "runs": runs.value, "tasks": dict(zip(("local", "gather", "s", "st"),
                                                                                tasks.tolist()))}

    def team_sizes(self):
        """``(blocks per instance, blocks of the team launch)`` (teams schedule)."""
        sizes = np.zeros(self.count, np.int32)
        grid = ctypes.c_int32()
        _lib.check(self._lib.pd_batch_team_sizes(self._handle, _lib.ptr(sizes), ctypes.byref(grid)))
        return sizes, grid.value

    def backward(self, x_record: torch.Tensor, grad_q: torch.Tensor, grad_qd: torch.Tensor | None = None, *,
                 materials: bool = True):
        """Adjoint of the last rollout (teams schedule).

        ``x_record``: the rollout's float64 ``(steps, P, 3)`` record;
        ``grad_q``/``grad_qd``: loss gradients w.r.t. the final ``(P, 3)`` state.
        Returns ``(dL/dq0, dL/dqd0, dL/dforces (steps, P, 3), dL/d(mu, lambda)
        (E, 2) float64 or None, adjoint iterations (steps, count))``.
        """
        steps = int(x_record.shape[0])
        shape = (self.particle_count, 3)
        if x_record.dtype != torch.float64 or tuple(x_record.shape) != (steps,) + shape or not x_record.is_contiguous():
            raise ValueError("x_record must be the rollout's contiguous float64 (steps, P, 3) record")
        grad_q = grad_q.detach().to(self.device, self.state_dtype).contiguous()
        grad_qd = (torch.zeros_like(grad_q) if grad_qd is None
                   else grad_qd.detach().to(self.device, self.state_dtype).contiguous())
        if tuple(grad_q.shape) != shape or tuple(grad_qd.shape) != shape:
            raise ValueError("final-state gradients must have shape (P, 3)")
        key = (steps, materials)
        if getattr(self, "_adjoint_key", None) != key:
            self._adjoint_buffers = (
                torch.empty((2,) + shape, dtype=self.state_dtype, device=self.device),
                torch.empty((2,) + shape, dtype=self.state_dtype, device=self.device),
                torch.empty((steps,) + shape, dtype=self.state_dtype, device=self.device),
                torch.empty((int(self.element_offsets[-1]), 2), dtype=torch.float64, device=self.device)
                if materials else None,
                torch.empty((2,) + shape, dtype=self.state_dtype, device=self.device),
            )
            self._adjoint_key = key
        gq, gqd, gf, gm, final = self._adjoint_buffers
        final[0].copy_(grad_q)
        final[1].copy_(grad_qd)
        iterations = np.zeros((steps, self.count), np.int32)
        _lib.check(
            self._lib.pd_batch_backward(
                self._handle, steps, self.dt, _lib.ptr(x_record), _lib.ptr(final[0]), _lib.ptr(final[1]),
                _lib.ptr(gq), _lib.ptr(gqd), _lib.ptr(gf), _lib.ptr(gm), _lib.ptr(iterations), _stream(),
            )
        )
        slot = (steps - 1) & 1
        return gq[slot], gqd[slot], gf, gm, iterations

    def timeline(self):
        """Start and end (global-timer ns) of each instance's last forward and
        adjoint rollout on its lane: two ``(count, 2)`` uint64 arrays."""
        forward = np.zeros((self.count, 2), np.uint64)
        adjoint = np.zeros((self.count, 2), np.uint64)
        _lib.check(self._lib.pd_batch_timeline(self._handle, _lib.ptr(forward), _lib.ptr(adjoint), _stream()))
        return forward, adjoint

    def measurement(self):
        """``(forward durations [us], iterations, team sizes, adjoint durations [us] or None)``
        of every instance in the last forward rollout and the last adjoint (when one ran):
        the ``measured`` costs a re-planned batch of the same instances takes."""
        forward, adjoint = self.timeline()
        us = (forward[:, 1].astype(np.float64) - forward[:, 0].astype(np.float64)) / 1.0e3
        adjoint_us = None
        if np.all(adjoint[:, 1] >= adjoint[:, 0]) and np.all(adjoint[:, 1] > 0):
            adjoint_us = (adjoint[:, 1].astype(np.float64) - adjoint[:, 0].astype(np.float64)) / 1.0e3
        _, iterations = self.read()
        sizes, _ = self.team_sizes()
        return us, iterations.sum(axis=0).astype(np.int32), sizes, adjoint_us

    def concat(self, tensors) -> torch.Tensor:
        """Concatenate per-instance ``(n_i, 3)`` tensors into one ``(P, 3)`` state array."""
        out = torch.cat([t.to(self.device, self.state_dtype) for t in tensors]).contiguous()
        if out.shape != (self.particle_count, 3):
            raise ValueError("per-instance tensors must match the instance particle counts")
        return out

    def split(self, tensor: torch.Tensor) -> list[torch.Tensor]:
        """Per-instance views of the last axis-(-2) ``P`` rows of a concatenated array."""
        o = self.particle_offsets
        return [tensor[..., o[i]:o[i + 1], :] for i in range(self.count)]

    def rollout(self, q0: torch.Tensor, qd0: torch.Tensor, forces: torch.Tensor, steps: int, *,
                record: bool = True, out=None, stepwise: bool = False):
        """Run ``steps`` PD steps of every instance in one graph launch.

        ``q0``, ``qd0``: ``(P, 3)``; ``forces``: ``(P, 3)`` applied every step or
        ``(steps, P, 3)``. Returns ``(q, qd, x_record)`` with ``q``, ``qd`` of
        shape ``(steps, P, 3)`` (state dtype) and ``x_record`` float64
        ``(steps, P, 3)`` (or ``None``). ``out`` may pass those three arrays
        to reuse them (the captured graph is reused while every pointer matches).
        ``stepwise=True`` launches the same kernels one by one instead of as
        one graph (for profilers; slower, same results).
        """
        steps = int(steps)
        if steps < 1:
            raise ValueError("steps must be positive")
        shape = (self.particle_count, 3)
        for name, tensor in (("q0", q0), ("qd0", qd0)):
            if tensor.dtype != self.state_dtype or tuple(tensor.shape) != shape or not tensor.is_contiguous():
                raise ValueError(f"{name} must be a contiguous {self.state_dtype} (P, 3) tensor")
            if tensor.device != self.device:
                raise ValueError(f"{name} must be on the solver device")
        if forces.dtype != self.state_dtype or not forces.is_contiguous() or forces.device != self.device:
            raise ValueError("forces must be a contiguous tensor of the state dtype on the solver device")
        if tuple(forces.shape) == shape:
            stride = 0
        elif tuple(forces.shape) == (steps,) + shape:
            stride = 3 * self.particle_count
        else:
            raise ValueError("forces must have shape (P, 3) or (steps, P, 3)")
        if out is None:
            q = torch.empty((steps,) + shape, dtype=self.state_dtype, device=self.device)
            qd = torch.empty_like(q)
            x_record = torch.empty((steps,) + shape, dtype=torch.float64, device=self.device) if record else None
        else:
            q, qd, x_record = out
        self._steps = steps
        _lib.check(
            (self._lib.pd_batch_forward_stepwise if stepwise else self._lib.pd_batch_forward)(
                self._handle, steps, self.dt, _lib.ptr(self._gravity), _lib.ptr(q0), _lib.ptr(qd0), _lib.ptr(forces),
                stride, _lib.ptr(q), _lib.ptr(qd), _lib.ptr(x_record), _stream(),
            )
        )
        return q, qd, x_record

    def read(self):
        """``(status bits per instance since the last read, iterations (steps, count) of the last
        rollout)``; the read clears the status bits (like ``SolverDiffPhD.read_status``); synchronises."""
        status = np.zeros(self.count, np.int32)
        iterations = np.zeros((max(self._steps, 0), self.count), np.int32)
        _lib.check(self._lib.pd_batch_read(self._handle, _lib.ptr(status), _lib.ptr(iterations) if self._steps else None,
                                           _stream()))
        return status, iterations

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            try:
                self._lib.pd_batch_destroy(handle)
            except Exception:
                pass
            self._handle = None


def _time_forward(batch, q0, qd0, forces, steps):
    out = batch.rollout(q0, qd0, forces, steps)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    batch.rollout(q0, qd0, forces, steps, out=out)
    end.record()
    torch.cuda.synchronize()
    return start.elapsed_time(end)


def autotune(solvers, dt, q0, qd0, forces, *, steps: int = 2, windows=(3, 5, 8),
             teams=((65536, 512), (32768, 256), (131072, 1024)), replan_steps: int = 0,
             instance_windows: bool = False, **options):
    """Pick the Anderson window and the team sizing of a batch from short rollouts.

    Times a ``steps``-step forward rollout of the batch for every window (with
    the first team sizing), then for every other team sizing with the best
    window, and returns ``(BatchedSolver, report)`` built with the fastest
    setting (the solvers keep its window). ``q0``, ``qd0``, ``forces`` are the
    concatenated rollout inputs; the probe runs the rollout's first steps.

    With ``instance_windows`` every instance also gets its own window: the one
    of the probed windows with which it needed the fewest iterations without
    reaching its iteration limit (Anderson mixing stalls on some strongly
    nonlinear instances that plain local/global iterations solve); that
    mixed setting is timed like the others and kept when it is the fastest.
    With ``replan_steps`` > 0 a rollout of that many steps then measures every
    instance's cost; with ``instance_windows``, instances that reached their
    iteration limit there fall back to window 0 (no mixing) and the rollout is
    measured again; the batch is then re-planned from those costs (larger
    teams for the instances on the critical path) when that is faster.
    """
    report = []
    best = None
    per_window = {}

    def apply(assignment):
        for solver, window in zip(solvers, assignment):
            if solver.anderson_window != window:
                solver.set_anderson_window(window)

    def probe(assignment, label, team_nnz, team_samples):
        nonlocal best
        apply(assignment)
        batch = BatchedSolver(solvers, dt, team_nnz=team_nnz, team_samples=team_samples, **options)
        ms = _time_forward(batch, q0, qd0, forces, steps)
        status, iterations = batch.read()
        report.append({"window": label, "team_nnz": team_nnz, "team_samples": team_samples, "ms": ms,
                       "iterations": int(iterations.sum()), "instances_at_limit": int(np.count_nonzero(status & 1))})
        if best is None or ms < best[0]:
            best = (ms, list(assignment), label, team_nnz, team_samples)
        del batch
        return status, iterations

    for window in windows:
        status, iterations = probe([window] * len(solvers), window, *teams[0])
        per_window[window] = (iterations.sum(axis=0), (status & 1) != 0)
    if instance_windows and len(windows) > 1:
        order = list(windows)
        cost = np.stack([per_window[w][0] + np.where(per_window[w][1], np.iinfo(np.int32).max // 4, 0)
                         for w in order])
        mixed = [order[k] for k in np.argmin(cost, axis=0)]
        if len(set(mixed)) > 1:
            probe(mixed, "per-instance", *teams[0])
    for team_nnz, team_samples in teams[1:]:
        probe(best[1], best[2], team_nnz, team_samples)
    _, assignment, label, team_nnz, team_samples = best
    apply(assignment)
    batch = BatchedSolver(solvers, dt, team_nnz=team_nnz, team_samples=team_samples, **options)
    chosen = {"window": label, "team_nnz": team_nnz, "team_samples": team_samples}
    if replan_steps:
        # Second stage: one rollout of `replan_steps` steps with the chosen
        # setting measures every instance's duration and iterations; the batch
        # is re-planned from those costs when that rollout gets faster.
        first = _time_forward(batch, q0, qd0, forces, replan_steps)
        if instance_windows:
            status, _ = batch.read()
            stalled = [i for i in np.flatnonzero(status & 1) if assignment[i] != 0]
            if stalled:
                for i in stalled:
                    assignment[i] = 0
                apply(assignment)
                del batch
                batch = BatchedSolver(solvers, dt, team_nnz=team_nnz, team_samples=team_samples, **options)
                report.append({"stall_fallback": [int(i) for i in stalled], "ms_before": first})
                first = _time_forward(batch, q0, qd0, forces, replan_steps)
                chosen["window"] = "per-instance"
        measured = batch.measurement()
        replanned = BatchedSolver(solvers, dt, team_nnz=team_nnz, team_samples=team_samples, measured=measured,
                                  **options)
        second = _time_forward(replanned, q0, qd0, forces, replan_steps)
        report.append({"replan_steps": replan_steps, "ms": first, "replanned_ms": second})
        if second < first:
            batch = replanned
            chosen["replanned"] = True
    if chosen["window"] == "per-instance":
        counts = np.unique([s.anderson_window for s in solvers], return_counts=True)
        chosen["windows"] = {str(int(w)): int(c) for w, c in zip(*counts)}
    return batch, {"chosen": chosen, "probes": report, "probe_steps": steps}
