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


# ---------------------------------------------------------------------------
# The Tet4 contact workload: a soft block resting on a fixed plane, poked by a
# rigid sphere probe. The block is 20 x 20 x 10 cubes of 1 mm split into five
# tetrahedra each (20,000 Tet4, 4,851 particles; E = 1e5 Pa, nu = 0.45,
# density 1100 kg/m^3); the plane is a frictional boundary z = 0 holding the
# bottom-face particles; the probe is a meshed ball of radius 3 mm (an
# icosphere of 162 surface particles around a centre, 320 tetrahedra) whose particles are
# prescribed (Dirichlet) and move down 4 mm at constant speed over the
# rollout; block and probe meet through the penalty mesh contact (radius
# 0.55 mm, normal stiffness 5e3 N/m, tangential damping 50 N s/m, friction
# 0.5).


@dataclass
class Poke:
    offset: tuple          # probe offset (dx, dy) [m] from the block's top centre
    nx: int = 20
    ny: int = 20
    nz: int = 10
    edge: float = 1.0e-3
    young: float = 1.0e5
    poisson: float = 0.45
    density: float = 1100.0
    probe_radius: float = 3.0e-3
    probe_level: int = 2      # icosphere subdivisions: 162 surface particles, 320 faces
    probe_travel: float = 4.0e-3
    start_gap: float = 0.25e-3
    steps: int = 200
    dt: float = 1.0e-3


def _icosphere(level: int):
    """Unit sphere triangulated from the icosahedron by ``level`` 4-to-1 subdivisions: ``(points, faces)``."""
    phi = (1.0 + 5.0 ** 0.5) / 2.0
    points = [np.array(p, dtype=np.float64) for p in
              ([0, 1, phi], [0, -1, phi], [0, 1, -phi], [0, -1, -phi], [1, phi, 0], [-1, phi, 0],
               [1, -phi, 0], [-1, -phi, 0], [phi, 0, 1], [-phi, 0, 1], [phi, 0, -1], [-phi, 0, -1])]
    points = [p / np.linalg.norm(p) for p in points]
    # The 20 faces: every triple of mutually adjacent vertices.
    table = np.array(points)
    distance = np.linalg.norm(table[:, None] - table[None], axis=2)
    adjacent = np.abs(distance - distance[distance > 1e-9].min()) < 1e-9
    faces = [(a, b, c) for a in range(12) for b in range(a + 1, 12) for c in range(b + 1, 12)
             if adjacent[a, b] and adjacent[b, c] and adjacent[a, c]]
    for _ in range(level):
        midpoint = {}

        def middle(i, j):
            key = (min(i, j), max(i, j))
            if key not in midpoint:
                m = points[i] + points[j]
                points.append(m / np.linalg.norm(m))
                midpoint[key] = len(points) - 1
            return midpoint[key]

        refined = []
        for a, b, c in faces:
            ab, bc, ca = middle(a, b), middle(b, c), middle(c, a)
            refined += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = refined
    return np.array(points), np.array(faces, dtype=np.int32)


def poke_scene(spec: Poke, device="cuda"):
    """``(model, options)`` of the poke workload.

    ``options`` holds the solver keywords of the contact (``frictional_boundary``,
    ``frictional_vertices``, ``mesh_contact``), the per-step prescribed probe
    positions ``dirichlet`` (float32 ``(steps, N, 3)``), the block's surface
    faces and the probe's particle range.
    """
    vertices, tets, _ = meshes.tet_grid(spec.nx, spec.ny, spec.nz, spec.edge)
    mu, lam = meshes.lame_from_young(spec.young, spec.poisson)
    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=spec.nx, dim_y=spec.ny,
                          dim_z=spec.nz, cell_x=spec.edge, cell_y=spec.edge, cell_z=spec.edge,
                          density=spec.density, k_mu=float(mu), k_lambda=float(lam), k_damp=0.0)
    block = builder.particle_count
    points, faces = _icosphere(spec.probe_level)
    top = spec.nz * spec.edge
    center = np.array([spec.nx * spec.edge / 2 + spec.offset[0], spec.ny * spec.edge / 2 + spec.offset[1],
                       top + spec.probe_radius + spec.start_gap])
    ball = np.vstack((points * spec.probe_radius + center, center[None]))
    for p in ball:
        builder.add_particle(p, (0.0, 0.0, 0.0), 0.0)
    hub = block + len(points)
    for a, b, c in faces:
        tet = [hub, block + a, block + b, block + c]
        edges = ball[[a, b, c]] - center
        if np.linalg.det(edges) < 0.0:
            tet[2], tet[3] = tet[3], tet[2]
        builder.add_tetrahedron(*tet, k_mu=float(mu), k_lambda=float(lam))
    model = builder.finalize(device)
    surface = meshes.boundary_faces_tet(tets)
    bottom = np.flatnonzero(np.abs(vertices[:, 2]) <= 1.0e-12).astype(np.int32)
    q0 = model.particle_q.detach().cpu().numpy().astype(np.float64)
    dirichlet = np.repeat(q0[None], spec.steps, axis=0)
    for t in range(spec.steps):
        dirichlet[t, block:, 2] -= spec.probe_travel * (t + 1) / spec.steps
    options = {
        "frictional_boundary": ("planar", (0.0, 0.0, 1.0, 0.0)),
        "frictional_vertices": bottom,
        "mesh_contact": (0.55e-3, 5.0e3, 5.0e3, 50.0, 0.5, surface, faces + block),
        "dirichlet": dirichlet.astype(np.float32),
        "surface": surface,
        "probe": (block, model.particle_count),
    }
    return model, options


# ---------------------------------------------------------------------------
# The large Hex8 twist-release workload: an 80 x 20 x 20 cell cantilever
# (32,000 Hex8, 35,721 particles) of 1 cm cells, the x = 0 face pinned, the
# middle third of the x slabs ten times stiffer (the rule of the reference
# cantilever, cells nx//3 < i <= 2 (nx//3)), nu = 0.45, density 1000 kg/m^3,
# no gravity. The initial state rotates every cross-section about the beam
# axis by an angle growing linearly from 0 at the root to 30 degrees at the
# tip (the reference twisted_positions) and releases it at rest.


@dataclass
class Twist:
    nx: int = 80
    ny: int = 20
    nz: int = 20
    edge: float = 0.01
    young: float = 1.0e6
    stiff_ratio: float = 10.0
    poisson: float = 0.45
    density: float = 1000.0
    angle_degrees: float = 30.0
    steps: int = 100
    dt: float = 1.0e-3


def twisted_positions(rest: np.ndarray, angle: float) -> np.ndarray:
    """Cross-sections rotated about the beam's centre line, 0 at the root to ``angle`` [rad] at the tip."""
    rest = np.asarray(rest, dtype=np.float64)
    low, high = rest.min(axis=0), rest.max(axis=0)
    theta = angle * (rest[:, 0] - low[0]) / (high[0] - low[0])
    center = 0.5 * (low[1:] + high[1:])
    offset = rest[:, 1:] - center
    q = rest.copy()
    q[:, 1] = center[0] + np.cos(theta) * offset[:, 0] - np.sin(theta) * offset[:, 1]
    q[:, 2] = center[1] + np.sin(theta) * offset[:, 0] + np.cos(theta) * offset[:, 1]
    root = rest[:, 0] == low[0]
    q[root] = rest[root]
    return q


def twist_cantilever(spec: Twist, device="cuda"):
    """``(model, mesh, hex_materials, q0, tip)``: the twisted initial positions (float64) and the tip-face particles."""
    vertices, hexes, cells = meshes.hex_grid(spec.nx, spec.ny, spec.nz, spec.edge)
    pinned = vertices[:, 0] <= 1.0e-12
    builder = ModelBuilder(gravity=(0.0, 0.0, 0.0))
    builder.add_particles(pos=vertices.tolist(), vel=np.zeros_like(vertices).tolist(),
                          mass=[0.0 if p else 1.0 for p in pinned])
    model = builder.finalize(device)
    slab = np.asarray(cells)  # x index of every cell
    third = spec.nx // 3
    stiff = (slab > third) & (slab <= 2 * third)
    young = spec.young * np.where(stiff, spec.stiff_ratio, 1.0)
    mu, lam = meshes.lame_from_young(young, spec.poisson)
    q0 = twisted_positions(vertices, np.radians(spec.angle_degrees))
    tip = np.flatnonzero(np.abs(vertices[:, 0] - spec.nx * spec.edge) <= 1.0e-12)
    mesh = meshes.Mesh(f"twist{spec.nx}x{spec.ny}x{spec.nz}", vertices, hexes)
    return model, mesh, np.stack([mu, lam], axis=1), q0, tip


# ---------------------------------------------------------------------------
# The reference's own Hex8 cantilever (src/newton_solver_diff_phd/examples/
# _diff_phd_cantilever.py:82-185, geometry of tools/bake_cantilever.py:22-49):
# 20 x 5 x 5 cubic cells in binary corner order, vertex (i, j, k) at index
# i*36 + j*6 + k, the x = 0 face pinned; x slabs 7..12 (cells 20//3 < i <=
# 2*(20//3)) at E = 1e7 Pa, the rest 1e6 Pa, nu = 0.45, density 1000 kg/m^3,
# no gravity; a +x fibre of stiffness 1e5 and target length 0 in cells i*25
# (the bottom-edge cells (i, 0, 0)); vertex-plane energies of stiffness 100 on
# vertices 720 and 750 against the half-space z + 0.1 >= 0. The axial motion
# pulls every tip vertex with +x force 80 t / 25 N at step t = 0..24 (dt 0.01,
# rel 1e-4); the twist motion releases the cross-sections rotated linearly
# along x up to 30 degrees at the tip (dt 0.001, 100 steps, rel 1e-6). The
# reference bakes 0.016 m cells; BASELINE's variant uses 0.01 m.


@dataclass
class ReferenceCantilever:
    edge: float = 0.016
    motion: str = "axial"     # "axial" or "twist"
    nx: int = 20
    ny: int = 5
    nz: int = 5
    young: float = 1.0e6
    stiff_ratio: float = 10.0
    poisson: float = 0.45
    density: float = 1000.0
    muscle_stiffness: float = 1.0e5
    plane_vertices: tuple = (720, 750)
    plane_stiffness: float = 100.0
    plane: tuple = (0.0, 0.0, 1.0, 0.1)
    twist_degrees: float = 30.0

    @property
    def dt(self) -> float:
        return 0.01 if self.motion == "axial" else 0.001

    @property
    def steps(self) -> int:
        return 25 if self.motion == "axial" else 100

    @property
    def rel_tol(self) -> float:
        return 1.0e-4 if self.motion == "axial" else 1.0e-6

    def tip_force(self, step: int) -> float:
        """+x force on every tip vertex at ``step`` [N] (zero for the twist release)."""
        return 80.0 * step / 25.0 if self.motion == "axial" else 0.0


def reference_cantilever(spec: ReferenceCantilever, device="cuda"):
    """``(model, solver_options, q0, tip)`` of the reference cantilever.

    ``solver_options`` are the ``SolverDiffPhD`` keywords of the reference
    example (hex mesh and materials, fibres, targets, planar energies and the
    convergence settings); ``q0`` is the float64 initial position (the rest
    pose, or the twisted pose); ``tip`` the tip-face particles.
    """
    if spec.motion not in ("axial", "twist"):
        raise ValueError("motion must be 'axial' or 'twist'")
    vertices, hexes, cells = meshes.hex_grid(spec.nx, spec.ny, spec.nz, spec.edge)
    pinned = vertices[:, 0] == 0.0
    builder = ModelBuilder(gravity=(0.0, 0.0, 0.0))
    builder.add_particles(pos=vertices.tolist(), vel=np.zeros_like(vertices).tolist(),
                          mass=[0.0 if p else spec.density * spec.edge**3 for p in pinned])
    model = builder.finalize(device)
    third = spec.nx // 3
    stiff = (cells > third) & (cells <= 2 * third)
    mu, lam = meshes.lame_from_young(spec.young * np.where(stiff, spec.stiff_ratio, 1.0), spec.poisson)
    muscle = np.zeros(len(hexes))
    muscle[np.arange(spec.nx) * spec.ny * spec.nz] = spec.muscle_stiffness
    options = {
        "hex_mesh": meshes.Mesh(f"cantilever{spec.nx}x{spec.ny}x{spec.nz}", vertices, hexes),
        "hex_materials": np.column_stack([mu, lam]),
        "density": spec.density,
        "material": "pd",
        "muscle_directions": np.tile([1.0, 0.0, 0.0], (len(hexes), 1)),
        "muscle_stiffness": muscle,
        "muscle_targets": np.zeros(len(hexes)),
        "planar_energies": (np.asarray(spec.plane_vertices, dtype=np.int32), spec.plane_stiffness, spec.plane),
        "max_iterations": 5000,
        "abs_tol": 1.0e-9,
        "rel_tol": spec.rel_tol,
        "anderson_window": 5,
    }
    q0 = vertices.copy() if spec.motion == "axial" else twisted_positions(vertices, np.radians(spec.twist_degrees))
    tip = np.flatnonzero(vertices[:, 0] == vertices[:, 0].max())
    return model, options, q0, tip
