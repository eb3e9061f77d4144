"""Minimal Newton-style model, state and control containers on PyTorch tensors.

The reference solver consumes Newton 1.7 ``Model``/``State``/``Control``
objects (imported at ``src/newton_solver_diff_phd/_src/solvers/diff_phd/solver.py:14``).
Newton is not part of this package, so these containers carry exactly the
fields that solver reads, with Newton's names, shapes and dtypes:

* ``particle_q``, ``particle_qd``, ``particle_f``: ``(N, 3)`` float32;
* ``particle_inv_mass`` ``(N,)`` float32 (zero marks a Dirichlet particle),
  ``particle_flags`` ``(N,)`` int32 (bit 0 = ACTIVE), ``particle_world``;
* ``tet_indices`` ``(4E,)`` int32, ``tet_poses`` ``(E, 3, 3)`` float32 inverse
  rest edge matrices, ``tet_materials`` ``(E, 3)`` float32 ``[mu, lambda, damping]``,
  ``tet_activations`` ``(E,)`` float32;
* ``gravity`` ``(worlds, 3)`` float32.

``ModelBuilder.add_soft_grid`` uses this package's five-tet split
(:mod:`newton_solver_diff_phd_b200.meshes`); Newton's own split is not
reproduced.
"""

from __future__ import annotations

import numpy as np
import torch

from . import meshes

PARTICLE_FLAG_ACTIVE = 1


def _normalize(device) -> torch.device:
    """A CUDA device with an explicit index (``cuda`` means the current device)."""
    device = torch.device(device)
    if device.type == "cuda" and device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    return device


class State:
    """Particle state: positions, velocities and external forces."""

    def __init__(self, particle_q: torch.Tensor, particle_qd: torch.Tensor, particle_f: torch.Tensor):
        self.particle_q = particle_q
        self.particle_qd = particle_qd
        self.particle_f = particle_f

    def requires_grad_(self, flag: bool = True) -> "State":
        """Give every array a zeroed ``.grad`` buffer, as Warp arrays with ``requires_grad``.

        The tensors stay plain (no autograd graph); the solver's backward pass
        accumulates into their ``.grad`` directly.
        """
        for tensor in (self.particle_q, self.particle_qd, self.particle_f):
            if flag and tensor.grad is None:
                tensor.grad = torch.zeros_like(tensor)
            elif not flag:
                tensor.grad = None
        return self


class Control:
    """Per-step controls: Tet4 fibre contractions ``tet_activations`` (E,) float32 or None."""

    def __init__(self, tet_activations: torch.Tensor | None = None):
        self.tet_activations = tet_activations


class Model:
    def __init__(self, device: str | torch.device = "cuda"):
        self.device = _normalize(device)
        self.particle_q = None
        self.particle_qd = None
        self.particle_inv_mass = None
        self.particle_flags = None
        self.particle_world = None
        self.gravity = None
        self.tet_indices = None
        self.tet_poses = None
        self.tet_materials = None
        self.tet_activations = None
        self.body_count = 0
        self.shape_count = 0
        self.requires_grad = False

    @property
    def particle_count(self) -> int:
        return 0 if self.particle_q is None else int(self.particle_q.shape[0])

    @property
    def tet_count(self) -> int:
        return 0 if self.tet_indices is None else int(self.tet_indices.numel() // 4)

    def state(self, requires_grad: bool | None = None) -> State:
        requires_grad = self.requires_grad if requires_grad is None else requires_grad
        state = State(
            self.particle_q.detach().clone(),
            self.particle_qd.detach().clone(),
            torch.zeros_like(self.particle_q),
        )
        if requires_grad:
            state.requires_grad_(True)
        return state

    def control(self) -> Control:
        return Control(None if self.tet_activations is None else self.tet_activations.detach().clone())


class ModelBuilder:
    """Collects particles and tetrahedra, then finalizes a :class:`Model`."""

    def __init__(self, gravity=(0.0, 0.0, -9.81)):
        self.gravity = tuple(float(g) for g in gravity)
        self.particle_q: list = []
        self.particle_qd: list = []
        self.particle_mass: list = []
        self.tet_indices: list = []
        self.tet_materials: list = []
        self._poses: list = []

    @property
    def particle_count(self) -> int:
        return len(self.particle_q)

    def add_particles(self, pos, vel, mass, radius=None):
        self.particle_q.extend([list(map(float, p)) for p in pos])
        self.particle_qd.extend([list(map(float, v)) for v in vel])
        self.particle_mass.extend([float(m) for m in mass])

    def add_particle(self, pos, vel, mass, radius=None) -> int:
        """Add one particle; returns its index."""
        self.add_particles([pos], [vel], [mass])
        return self.particle_count - 1

    def add_tetrahedron(self, i, j, k, l, k_mu=1.0e3, k_lambda=1.0e3, k_damp=0.0) -> None:
        """Add one tetrahedron over existing particles, its rest pose from their current positions."""
        tet = np.array([[i, j, k, l]], dtype=np.int32)
        vertices = np.asarray(self.particle_q, dtype=np.float64)
        self.tet_indices.extend(tet.tolist())
        self.tet_materials.append([float(k_mu), float(k_lambda), float(k_damp)])
        self._poses.extend(meshes.tet_rest_poses(vertices, tet))

    def add_soft_grid(self, pos, rot, vel, dim_x, dim_y, dim_z, cell_x, cell_y, cell_z, density, k_mu, k_lambda,
                      k_damp, fix_left=False, fix_right=False, fix_bottom=False):
        """Add a Tet4 block of ``dim_x x dim_y x dim_z`` cubes split into five tetrahedra each.

        ``rot`` must be the identity; cells may have per-axis sizes.
        """
        if rot is not None and not np.allclose(np.asarray(rot, dtype=float), (0.0, 0.0, 0.0, 1.0)):
            raise NotImplementedError("add_soft_grid supports the identity rotation")
        vertices, tets, _ = meshes.tet_grid(dim_x, dim_y, dim_z, 1.0)
        vertices = vertices * np.array([cell_x, cell_y, cell_z]) + np.asarray(pos, dtype=np.float64)
        start = self.particle_count
        poses = meshes.tet_rest_poses(vertices, tets)
        volumes = np.abs(1.0 / np.linalg.det(poses)) / 6.0
        mass = np.zeros(len(vertices))
        np.add.at(mass, tets.ravel(), np.repeat(volumes * density / 4.0, 4))
        x = vertices[:, 0]
        if fix_left:
            mass[x == x.min()] = 0.0
        if fix_right:
            mass[x == x.max()] = 0.0
        if fix_bottom:
            z = vertices[:, 2]
            mass[z == z.min()] = 0.0
        self.add_particles(vertices, np.tile(np.asarray(vel, dtype=float), (len(vertices), 1)), mass)
        self.tet_indices.extend((tets + start).tolist())
        self.tet_materials.extend([[float(k_mu), float(k_lambda), float(k_damp)]] * len(tets))
        self._poses.extend(poses)

    def finalize(self, device="cuda", requires_grad: bool = False) -> Model:
        device = _normalize(device)
        model = Model(device)
        q = np.asarray(self.particle_q, dtype=np.float32).reshape(-1, 3)
        model.particle_q = torch.tensor(q, device=device)
        model.particle_qd = torch.tensor(np.asarray(self.particle_qd, dtype=np.float32).reshape(-1, 3), device=device)
        mass = np.asarray(self.particle_mass, dtype=np.float64)
        inverse = np.where(mass > 0.0, 1.0 / np.where(mass > 0.0, mass, 1.0), 0.0).astype(np.float32)
        model.particle_inv_mass = torch.tensor(inverse, device=device)
        model.particle_flags = torch.full((len(q),), PARTICLE_FLAG_ACTIVE, dtype=torch.int32, device=device)
        model.particle_world = torch.full((len(q),), -1, dtype=torch.int32, device=device)
        model.gravity = torch.tensor([self.gravity], dtype=torch.float32, device=device)
        if self.tet_indices:
            model.tet_indices = torch.tensor(np.asarray(self.tet_indices, dtype=np.int32).ravel(), device=device)
            model.tet_poses = torch.tensor(np.asarray(self._poses, dtype=np.float32), device=device)
            model.tet_materials = torch.tensor(np.asarray(self.tet_materials, dtype=np.float32), device=device)
            model.tet_activations = torch.zeros(len(self.tet_indices), dtype=torch.float32, device=device)
        model.requires_grad = requires_grad
        if requires_grad and model.tet_materials is not None:
            model.tet_materials.grad = torch.zeros_like(model.tet_materials)
        return model
