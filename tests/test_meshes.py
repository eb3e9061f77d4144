"""Index assembly: vertex numbering, cell corner order and the five-tet split."""

import numpy as np

from newton_solver_diff_phd_b200 import meshes


def test_hex_grid_matches_reference_baker_numbering():
    # tools/bake_cantilever.py:22-49: vertex i*(ny+1)*(nz+1) + j*(nz+1) + k, binary corners.
    nx, ny, nz = 20, 5, 5
    vertices, hexes, cells = meshes.hex_grid(nx, ny, nz, 0.016)
    assert vertices.shape == (756, 3) and hexes.shape == (500, 8)
    node = lambda i, j, k: i * (ny + 1) * (nz + 1) + j * (nz + 1) + k  # noqa: E731
    expected = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                expected.append([node(i + a, j + b, k + c) for a in (0, 1) for b in (0, 1) for c in (0, 1)])
    np.testing.assert_array_equal(hexes, np.asarray(expected))
    np.testing.assert_array_equal(cells, np.repeat(np.arange(nx), ny * nz))
    np.testing.assert_allclose(vertices[node(3, 2, 1)], np.array([3, 2, 1]) * 0.016)


def test_tet_split_tiles_every_cube_consistently():
    vertices, tets, cube = meshes.tet_grid(4, 3, 2, 0.5)
    poses = meshes.tet_rest_poses(vertices, tets)
    volumes = 1.0 / np.linalg.det(poses) / 6.0
    assert np.all(volumes > 0)
    np.testing.assert_allclose(np.bincount(cube, weights=volumes), 0.125)
    # Neighbouring cubes share face diagonals: every interior face triangle has two owners.
    faces = np.sort(tets[:, [[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]]].reshape(-1, 3), axis=1)
    _, counts = np.unique(faces, axis=0, return_counts=True)
    assert counts.max() == 2
    boundary = meshes.boundary_faces_tet(tets)
    assert len(boundary) == 2 * 2 * (4 * 3 + 4 * 2 + 3 * 2)


def test_lame_chain_rule_derivatives():
    young, nu = 2.0e6, 0.4
    mu, lam = meshes.lame_from_young(young, nu)
    dmu_de, dlam_de, dmu_dnu, dlam_dnu = meshes.lame_young_derivatives(nu)
    h = 1e-6
    mu2, lam2 = meshes.lame_from_young(young, nu + h)
    mu1, lam1 = meshes.lame_from_young(young, nu - h)
    np.testing.assert_allclose(mu / young, dmu_de)
    np.testing.assert_allclose(lam / young, dlam_de)
    np.testing.assert_allclose((mu2 - mu1) / (2 * h) / young, dmu_dnu, rtol=1e-6)
    np.testing.assert_allclose((lam2 - lam1) / (2 * h) / young, dlam_dnu, rtol=1e-6)
