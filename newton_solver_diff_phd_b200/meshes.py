"""Synthetic Hex8 and Tet4 grids used by the DiffPhD projective-dynamics path.

Vertex numbering follows the reference cantilever baker
(``tools/bake_cantilever.py:22-49``): vertex ``(i, j, k)`` of an
``nx x ny x nz`` cell grid has index ``i*(ny+1)*(nz+1) + j*(nz+1) + k`` and
every Hex8 cell lists its corners in binary ``(a, b, c)`` order
``000, 001, 010, 011, 100, 101, 110, 111``.

The Tet4 grid splits every cube into five tetrahedra. The reference obtains
its tetrahedra from Newton's ``ModelBuilder.add_soft_grid``, which is not part
of the reference tree, so the split here is this package's own definition:
cubes of even parity ``(i+j+k) % 2 == 0`` use the four even binary corners as
the central tetrahedron, odd cubes the four odd corners, so that neighbouring
cubes share face diagonals. Every tetrahedron is ordered with positive rest
volume. Both the solver and the oracle consume the same arrays.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# Binary corner index a*4 + b*2 + c of the cube corner (a, b, c).
_EVEN_SPLIT = ((0, 3, 5, 6), (1, 0, 3, 5), (2, 0, 6, 3), (4, 0, 5, 6), (7, 3, 6, 5))
_ODD_SPLIT = ((1, 2, 4, 7), (0, 1, 4, 2), (3, 1, 2, 7), (5, 1, 7, 4), (6, 2, 4, 7))


@dataclass
class Mesh:
    """Rest vertices and element connectivity, mirroring the reference ``Mesh``
    dataclass (``src/newton_solver_diff_phd/_src/geometry/usd.py:11-17``)."""

    name: str
    vertices: np.ndarray
    indices: np.ndarray


def grid_vertices(nx: int, ny: int, nz: int, edge: float, origin=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Vertices of an ``nx x ny x nz`` cell grid in x-major order, float64 [m]."""
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    points = np.stack((i.ravel(), j.ravel(), k.ravel()), axis=1).astype(np.float64) * float(edge)
    return points + np.asarray(origin, dtype=np.float64)


def _vertex(ny: int, nz: int, i, j, k):
    return i * (ny + 1) * (nz + 1) + j * (nz + 1) + k


def hex_grid(nx: int, ny: int, nz: int, edge: float, origin=(0.0, 0.0, 0.0)):
    """Hex8 grid: ``(vertices, hexes (E,8) int32, cell_x (E,) int32)``.

    Cells are numbered ``i*ny*nz + j*nz + k`` like the reference baker.
    """
    vertices = grid_vertices(nx, ny, nz, edge, origin)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    hexes = np.stack(
        [_vertex(ny, nz, i + a, j + b, k + c) for a in (0, 1) for b in (0, 1) for c in (0, 1)], axis=1
    ).astype(np.int32)
    return vertices, hexes, i.astype(np.int32)


def tet_grid(nx: int, ny: int, nz: int, edge: float, origin=(0.0, 0.0, 0.0)):
    """Five-tet split grid: ``(vertices, tets (5E,4) int32, cube (5E,) int32)``.

    Tetrahedra of cube ``c = i*ny*nz + j*nz + k`` occupy rows ``5c .. 5c+4``.
    """
    vertices, hexes, _ = hex_grid(nx, ny, nz, edge, origin)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    odd = ((i + j + k).ravel() & 1).astype(bool)
    tets = np.empty((len(hexes), 5, 4), dtype=np.int32)
    tets[~odd] = hexes[~odd][:, np.asarray(_EVEN_SPLIT)]
    tets[odd] = hexes[odd][:, np.asarray(_ODD_SPLIT)]
    tets = tets.reshape(-1, 4)
    edges = vertices[tets[:, 1:]] - vertices[tets[:, :1]]
    negative = np.linalg.det(edges) < 0.0
    tets[negative, 2], tets[negative, 3] = tets[negative, 3].copy(), tets[negative, 2].copy()
    cube = np.repeat(np.arange(len(hexes), dtype=np.int32), 5)
    return vertices, tets, cube


def tet_rest_poses(vertices: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """Inverse rest edge matrices ``Dm^{-1}`` with ``Dm = [x1-x0, x2-x0, x3-x0]`` (columns), float64."""
    x = np.asarray(vertices, dtype=np.float64)[np.asarray(tets)]
    dm = np.stack((x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]), axis=2)
    return np.linalg.inv(dm)


def boundary_faces_tet(tets: np.ndarray) -> np.ndarray:
    """Triangles that belong to exactly one tetrahedron, ``(F,3)`` int32."""
    tets = np.asarray(tets)
    faces = tets[:, [[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]]].reshape(-1, 3)
    key = np.sort(faces, axis=1)
    _, first, counts = np.unique(key, axis=0, return_index=True, return_counts=True)
    return faces[first[counts == 1]].astype(np.int32)


def lame_from_young(young, poisson):
    """Lame parameters ``(mu, lambda)`` from Young's modulus and Poisson ratio.

    Matches ``src/newton_solver_diff_phd/examples/_diff_phd_cantilever.py:95-96``.
    """
    young = np.asarray(young, dtype=np.float64)
    poisson = np.asarray(poisson, dtype=np.float64)
    mu = young / (2.0 * (1.0 + poisson))
    lam = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson))
    return mu, lam


def lame_young_derivatives(poisson):
    """``(dmu/dE, dlambda/dE, dmu/dnu * 1/E, dlambda/dnu * 1/E)`` for the chain rule to E and nu."""
    nu = np.asarray(poisson, dtype=np.float64)
    dmu_de = 1.0 / (2.0 * (1.0 + nu))
    dlam_de = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    dmu_dnu = -1.0 / (2.0 * (1.0 + nu) ** 2)
    dlam_dnu = (1.0 + 2.0 * nu * nu) / ((1.0 + nu) ** 2 * (1.0 - 2.0 * nu) ** 2)
    return dmu_de, dlam_de, dmu_dnu, dlam_dnu
