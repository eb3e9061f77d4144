"""Shared scene builders for the tests (the reference's small fixtures)."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
DENSITY = 1000.0


def golden(name):
    return np.load(GOLDEN / name)


def tet_grid_model(contrast=1.0, device="cuda", requires_grad=False, fix_left=True, gravity=-9.81, cell=0.1):
    """The reference test grid: 3x2x2 cubes at z=1, k_mu 2e4, k_lambda 5e4 (tests/test_diff_phd_solver.py:65-92)."""
    import torch

    from newton_solver_diff_phd_b200 import ModelBuilder

    builder = ModelBuilder(gravity=(0.0, 0.0, gravity))
    builder.add_soft_grid(
        pos=(0.0, 0.0, 1.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=3, dim_y=2, dim_z=2, cell_x=cell, cell_y=cell,
        cell_z=cell, density=DENSITY, k_mu=2.0e4, k_lambda=5.0e4, k_damp=0.0, fix_left=fix_left,
    )
    model = builder.finalize(device, requires_grad=requires_grad)
    if contrast != 1.0:
        q = model.particle_q.cpu().numpy()
        tets = model.tet_indices.cpu().numpy().reshape(-1, 4)
        stiff = q[tets].mean(axis=1)[:, 0] > q[:, 0].mean()
        materials = model.tet_materials.detach().cpu().numpy()
        materials[stiff, :2] *= contrast
        with torch.no_grad():
            model.tet_materials.copy_(torch.tensor(materials))
    return model


def deformed_arrays(vertices, free, seed=3, stretch=(1.3, 0.8, 1.1), speed=0.5):
    """The reference ``_deformed_state`` (tests/test_diff_phd_solver.py:109-120) as float32-rounded arrays."""
    rng = np.random.default_rng(seed)
    q = np.asarray(vertices, dtype=np.float32).astype(np.float64)
    center = q.mean(axis=0)
    deformed = np.where(free[:, None], center + (q - center) * np.asarray(stretch), q)
    deformed[free] += 0.01 * rng.standard_normal((free.sum(), 3))
    velocity = np.where(free[:, None], speed * rng.standard_normal(q.shape), 0.0)
    return deformed.astype(np.float32), velocity.astype(np.float32)


def oracle_tet_body(model, material="pd", **kwargs):
    from oracle import pd_oracle

    materials = model.tet_materials.detach().cpu().numpy().astype(np.float64)
    return pd_oracle.Body.tet(
        model.tet_indices.cpu().numpy().reshape(-1, 4),
        model.tet_poses.cpu().numpy(),
        model.particle_inv_mass.cpu().numpy() > 0,
        materials[:, 0],
        materials[:, 1],
        DENSITY,
        material=material,
        **kwargs,
    )


def two_cube_mesh():
    """The reference Hex8 fixture: two 0.1 m cubes (tests/test_diff_phd_hex.py:25-36)."""
    from newton_solver_diff_phd_b200 import Mesh

    vertices = np.array([[x, y, z] for x in range(3) for y in range(2) for z in range(2)], dtype=float) * 0.1
    elements = np.array([np.arange(8), np.arange(4, 12)], dtype=np.int32)
    return Mesh("two-cubes", vertices, elements)


def particle_model(vertices, pinned, device="cuda", requires_grad=False, gravity=0.0):
    from newton_solver_diff_phd_b200 import ModelBuilder

    builder = ModelBuilder(gravity=(0.0, 0.0, gravity))
    builder.add_particles(
        pos=np.asarray(vertices).tolist(),
        vel=np.zeros_like(vertices).tolist(),
        mass=[0.0 if p else 1.0 for p in pinned],
    )
    return builder.finalize(device, requires_grad=requires_grad)
