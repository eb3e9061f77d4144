"""Synthetic Hex8 cantilever scenes of the batched workload.

A cantilever is an ``nx x ny x nz`` grid of cubic Hex8 cells (edge ``edge``)
with the ``x = 0`` face pinned, built like the reference cantilever example
(``src/newton_solver_diff_phd/examples/_diff_phd_cantilever.py``: cells in
binary corner order, Lame parameters from Young's modulus and Poisson's
ratio, lumped mean-cell-volume mass). The batched family draws uneven sizes
``nx`` in ``[4, 40]`` with ``ny = nz = max(2, nx // 4)``, per-instance Young's
modulus log-uniform in ``[1e5, 1e7]`` Pa, Poisson's ratio uniform in
``[0.3, 0.45]`` and a random +X force in ``[0, 50]`` N on every tip vertex.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import meshes
from .model import ModelBuilder


@dataclass
class Cantilever:
    nx: int
    ny: int
    nz: int
    young: float
    poisson: float
    tip_forces: np.ndarray  # (tip vertices,) +X force magnitudes [N]


def cantilever_family(count: int, seed: int = 0, nx_range=(4, 40), edge: float = 0.01) -> list[Cantilever]:
    """The seeded batched family: uneven grids, materials and tip forces."""
    rng = np.random.default_rng(seed)
    family = []
    for _ in range(count):
        nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        ny = max(2, nx // 4)
        young = float(np.exp(rng.uniform(np.log(1.0e5), np.log(1.0e7))))
        poisson = float(rng.uniform(0.3, 0.45))
        forces = rng.uniform(0.0, 50.0, (ny + 1) * (ny + 1))
        family.append(Cantilever(nx, ny, ny, young, poisson, forces))
    return family


def cantilever_model(spec: Cantilever, edge: float = 0.01, device="cuda", gravity=(0.0, 0.0, 0.0)):
    """``(model, mesh, hex_materials, forces)`` of one cantilever.

    ``forces`` is the float32 ``(particles, 3)`` external force array: the
    spec's +X magnitudes on the tip face ``x = nx * edge``, zero elsewhere.
    """
    vertices, hexes, _ = meshes.hex_grid(spec.nx, spec.ny, spec.nz, edge)
    pinned = vertices[:, 0] <= 1.0e-12
    builder = ModelBuilder(gravity=gravity)
    builder.add_particles(pos=vertices.tolist(), vel=np.zeros_like(vertices).tolist(),
                          mass=[0.0 if p else 1.0 for p in pinned])
    model = builder.finalize(device)
    mu, lam = meshes.lame_from_young(np.full(len(hexes), spec.young), spec.poisson)
    materials = np.stack([mu, lam], axis=1)
    tip = np.flatnonzero(np.abs(vertices[:, 0] - spec.nx * edge) <= 1.0e-12)
    forces = np.zeros_like(vertices, dtype=np.float32)
    forces[tip, 0] = np.asarray(spec.tip_forces, dtype=np.float32)[: len(tip)]
    return model, meshes.Mesh(f"cantilever{spec.nx}x{spec.ny}x{spec.nz}", vertices, hexes), materials, forces
