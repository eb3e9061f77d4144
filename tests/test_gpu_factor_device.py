"""The factor build with the numeric LDL^T and the rows of L^{-1} computed on the device
(pd_inverse_build_on, SolverDiffPhD.set_factor_device) against the host build: every array
bit-identical, and the same error for a matrix that is not positive definite.

The host build is itself bit-identical to the reference's sparse.py setup
(tests/test_factor.py); the device build must therefore reproduce it exactly,
including the reference's exact-zero omission (the "cancel" matrix has entries
of L^{-1} that cancel to zero) and rows that span many 256-label chunks
(the 32x8x8 Tet4 block and a 40x10x10 Hex8 cantilever).
"""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from newton_solver_diff_phd_b200 import ModelBuilder, SolverDiffPhD, _lib, meshes
from oracle import pd_oracle
from tests.helpers import golden

pytestmark = pytest.mark.gpu

ARRAYS = ["permutation", "s_offsets", "s_columns", "s_values", "st_offsets", "st_columns", "st_values"]


def assert_same(matrix_csr):
    host = _lib.inverse_factor(matrix_csr)
    device = _lib.inverse_factor(matrix_csr, device=torch.cuda.current_device())
    for key in ARRAYS:
        np.testing.assert_array_equal(device[key], host[key], err_msg=key)
    return host


@pytest.mark.parametrize("name", ["cancel", "grid2d", "tet322", "hex632"])
def test_golden_matrices(name):
    g = golden("sparse_factors.npz")
    host = assert_same(_lib.dense_to_csr(g[name + "__matrix"]))
    np.testing.assert_array_equal(host["s_values"], g[name + "__s_values"])


def test_exact_cancellation_and_identity_rows():
    matrix = np.asarray(((2.0, 2.0, 2.0, 0.0), (2.0, 5.0, 5.0, 0.0), (2.0, 5.0, 10.0, 0.0), (0.0, 0.0, 0.0, 1.0)))
    assert_same(_lib.dense_to_csr(matrix))


def test_indefinite_matrix_fails_like_the_host():
    matrix = np.asarray(((4.0, 1.0, 0.0), (1.0, 3.0, 5.0), (0.0, 5.0, 2.0)))
    messages = []
    for device in (None, torch.cuda.current_device()):
        with pytest.raises(ValueError) as info:
            _lib.inverse_factor(_lib.dense_to_csr(matrix), device=device)
        messages.append(str(info.value))
    assert "positive definite" in messages[0] and messages[0] == messages[1]


def _csr(matrix):
    matrix = sp.csr_matrix(matrix)
    matrix.sort_indices()
    return matrix.indptr, matrix.indices, matrix.data


def test_hex_cantilever_with_multi_chunk_rows():
    vertices, hexes, _ = meshes.hex_grid(40, 10, 10, 0.01)
    free = vertices[:, 0] > 1.0e-12
    young = np.exp(np.random.default_rng(3).uniform(np.log(1.0e5), np.log(1.0e7), len(hexes)))
    mu, lam = meshes.lame_from_young(young, 0.45)
    matrix = pd_oracle.Body.hex(vertices, hexes, free, mu, lam, 1000.0).matrix(0.01)
    host = assert_same(_csr(matrix))
    assert len(vertices) > 4096 and len(host["s_values"]) > 10 * len(vertices)


def test_solver_steps_are_bitwise_equal_with_the_device_build():
    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=32, dim_y=8, dim_z=8, cell_x=0.01,
                          cell_y=0.01, cell_z=0.01, density=1000.0, k_mu=3.0e5, k_lambda=1.2e6, k_damp=0.0,
                          fix_left=True)
    model = builder.finalize("cuda")
    results = []
    for device_build in (False, True):
        solver = SolverDiffPhD(model, density=1000.0, rel_tol=1.0e-6, abs_tol=1.0e-9)
        solver.set_factor_device(device_build)
        state, out = model.state(), model.state()
        for _ in range(3):
            solver.step(state, out, None, None, 5.0e-3)
            state, out = out, state
        solver.check_status()
        results.append((state.particle_q.clone(), solver.factor_stats()))
        del solver
    assert results[0][1] == results[1][1]
    assert torch.equal(results[0][0], results[1][0])
