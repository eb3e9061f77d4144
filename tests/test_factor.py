"""C++ inverse factor against the reference sparse.py setup, run on the same rows."""

import numpy as np
import pytest

from newton_solver_diff_phd_b200 import _lib
from tests.helpers import golden

NAMES = ["cancel", "grid2d", "tet322", "hex632"]
ARRAYS = ["permutation", "s_offsets", "s_columns", "s_values", "st_offsets", "st_columns", "st_values"]


@pytest.mark.parametrize("name", NAMES)
def test_inverse_factor_is_bit_identical_to_reference(name):
    g = golden("sparse_factors.npz")
    out = _lib.inverse_factor(_lib.dense_to_csr(g[name + "__matrix"]))
    for key in ARRAYS:
        np.testing.assert_array_equal(out[key], g[f"{name}__{key}"], err_msg=key)


def test_exact_cancellation_values():
    # A = L diag(2, 3, 5) L^T with unit lower L: S has five entries (tests/test_diff_phd_sparse.py:21-35).
    matrix = np.asarray(((2.0, 2.0, 2.0), (2.0, 5.0, 5.0), (2.0, 5.0, 10.0)))
    out = _lib.inverse_factor(_lib.dense_to_csr(matrix))
    np.testing.assert_array_equal(out["s_offsets"], (0, 1, 3, 5))
    np.testing.assert_array_equal(out["s_columns"], (0, 0, 1, 1, 2))
    np.testing.assert_array_equal(
        out["s_values"], (1 / np.sqrt(2), -1 / np.sqrt(3), 1 / np.sqrt(3), -1 / np.sqrt(5), 1 / np.sqrt(5))
    )


@pytest.mark.parametrize("name", NAMES)
def test_factor_solves_the_matrix(name):
    g = golden("sparse_factors.npz")
    matrix = g[name + "__matrix"]
    out = _lib.inverse_factor(_lib.dense_to_csr(matrix))
    n = len(matrix)
    s = np.zeros((n, n))
    for r in range(n):
        lo, hi = out["s_offsets"][r], out["s_offsets"][r + 1]
        s[r, out["s_columns"][lo:hi]] = out["s_values"][lo:hi]
    np.testing.assert_allclose(s.T @ s @ matrix, np.eye(n), atol=1e-11)
    assert np.all(out["s_values"] != 0.0)
    for r in range(n):
        assert np.all(np.diff(out["s_columns"][out["s_offsets"][r]:out["s_offsets"][r + 1]]) > 0)


def test_factor_rejects_invalid_rows():
    with pytest.raises(ValueError, match="symmetric"):
        _lib.inverse_factor(_lib.dense_to_csr(np.array([[2.0, 1.0], [0.5, 2.0]])))
    with pytest.raises(ValueError, match="positive"):
        _lib.inverse_factor(_lib.dense_to_csr(np.array([[1.0, 2.0], [2.0, 1.0]])))
    with pytest.raises(ValueError, match="positive definite"):
        _lib.inverse_factor(_lib.dense_to_csr(np.array([[0.0, 0.0], [0.0, 1.0]])))
    with pytest.raises(ValueError, match="finite"):
        _lib.inverse_factor(_lib.dense_to_csr(np.array([[np.inf]])))


def test_isolated_dirichlet_rows_are_identity():
    matrix = np.eye(5)
    matrix[:3, :3] = [[4.0, -1.0, 0.0], [-1.0, 4.0, -1.0], [0.0, -1.0, 4.0]]
    out = _lib.inverse_factor(_lib.dense_to_csr(matrix))
    for r in range(5):
        lo, hi = out["s_offsets"][r], out["s_offsets"][r + 1]
        if out["permutation"][r] >= 3:
            np.testing.assert_array_equal(out["s_values"][lo:hi], [1.0])
