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


def _dense_from_runs(row_runs, run_col, run_off, values, n):
    m = np.zeros((n, n))
    for r in range(n):
        for k in range(row_runs[r], row_runs[r + 1]):
            lo, hi = run_off[k], run_off[k + 1]
            m[r, run_col[k]:run_col[k] + hi - lo] = values[lo:hi]
    return m


def _hex_cantilever_matrix(nx, ny):
    from newton_solver_diff_phd_b200 import meshes
    from oracle import pd_oracle

    vertices, hexes, _ = meshes.hex_grid(nx, ny, ny, 0.01)
    free = vertices[:, 0] > 1e-9
    mu, lam = meshes.lame_from_young(np.full(len(hexes), 1e6), 0.4)
    return pd_oracle.Body.hex(vertices, hexes, free, mu, lam, 1000.0).matrix(0.01)


@pytest.mark.parametrize("name", NAMES + ["cantilever"])
@pytest.mark.parametrize("gap", [0, 2])
def test_run_format_is_the_same_factor(name, gap):
    """The postorder run matrices hold exactly the CSR factor: S_run = S[rows, cols] relabelled."""
    matrix = _hex_cantilever_matrix(8, 2) if name == "cantilever" else golden("sparse_factors.npz")[name + "__matrix"]
    out = _lib.inverse_factor(_lib.dense_to_csr(matrix), run_gap=gap)
    runs = out["runs"]
    n = len(matrix)
    label = runs["label_of"]
    assert sorted(label.tolist()) == list(range(n))
    s = np.zeros((n, n))
    for r in range(n):
        lo, hi = out["s_offsets"][r], out["s_offsets"][r + 1]
        s[r, out["s_columns"][lo:hi]] = out["s_values"][lo:hi]
    # Row r of S (elimination order) is run-format row label[permutation[r]].
    particle_of = np.empty(n, np.int64)
    particle_of[label] = np.arange(n)
    s_run = _dense_from_runs(runs["s_row_runs"], runs["s_run_col"], runs["s_run_off"], runs["s_values"], n)
    position = np.empty(n, np.int64)
    position[out["permutation"]] = np.arange(n)
    rows = np.array([position[particle_of[u]] for u in range(n)])
    np.testing.assert_array_equal(s_run, s[rows][:, particle_of])
    st_run = _dense_from_runs(runs["st_row_runs"], runs["st_run_col"], runs["st_run_off"], runs["st_values"], n)
    np.testing.assert_array_equal(st_run, s_run.T)
    # S^T S applied through the run format equals the inverse.
    rhs = np.random.default_rng(0).standard_normal((n, 3))
    x = np.empty_like(rhs)
    x[particle_of] = st_run @ (s_run @ rhs[particle_of])
    np.testing.assert_allclose(matrix @ x, rhs, atol=1e-9 * np.abs(rhs).max())
    if gap >= 2 and name == "cantilever":
        # Postorder labels make every row of S a single contiguous run.
        assert np.all(np.diff(runs["s_row_runs"]) <= 1)


def test_threaded_inverse_rows_are_bit_identical():
    """Rows of the inverse split over host threads by column range give the same arrays."""
    import scipy.sparse as sp

    from newton_solver_diff_phd_b200 import _lib, meshes
    from oracle import pd_oracle

    vertices, hexes, _ = meshes.hex_grid(14, 5, 5, 0.01)
    free = vertices[:, 0] > 1.0e-12
    mu, lam = meshes.lame_from_young(np.full(len(hexes), 1.0e6), 0.45)
    body = pd_oracle.Body.hex(vertices, hexes, free, mu, lam, 1000.0)
    a = sp.csr_matrix(body.matrix(0.01))
    a = ((a + a.T) * 0.5).tocsr()
    a.sort_indices()
    lib = _lib.library()
    results = []
    try:
        for work in (1 << 62, 0):
            _lib.check(lib.pd_inverse_parallel_work(work))
            results.append(_lib.inverse_factor((a.indptr, a.indices, a.data)))
    finally:
        _lib.check(lib.pd_inverse_parallel_work(1 << 16))
    for key in ("permutation", "s_offsets", "s_columns", "s_values", "st_offsets", "st_columns", "st_values"):
        assert np.array_equal(results[0][key], results[1][key]), key


@pytest.mark.parametrize("name", NAMES)
def test_threaded_ldlt_is_bit_identical_to_reference(name):
    """The numeric LDL^T (left-looking columns) and the rows of L^{-1} (chunked rows) level by
    level over host threads, forced on every factor, reproduce the reference's setup exactly on
    the golden matrices."""
    g = golden("sparse_factors.npz")
    lib = _lib.library()
    try:
        _lib.check(lib.pd_inverse_parallel_levels(0))
        out = _lib.inverse_factor(_lib.dense_to_csr(g[name + "__matrix"]))
    finally:
        _lib.check(lib.pd_inverse_parallel_levels(1 << 15))
    for key in ARRAYS:
        np.testing.assert_array_equal(out[key], g[f"{name}__{key}"], err_msg=key)


def test_threaded_ldlt_matches_the_sequential_loop_and_its_errors():
    """A 2,541-row Hex8 beam (hundreds of elimination-tree levels, separator chains at the top,
    rows spanning several 256-label chunks, groups of up to 32 rows): the level-parallel LDL^T and
    the grouped inverse rows give the sequential loops' arrays bit for bit; an indefinite matrix
    fails with the same message both ways."""
    import scipy.sparse as sp

    from newton_solver_diff_phd_b200 import meshes
    from oracle import pd_oracle

    vertices, hexes, _ = meshes.hex_grid(20, 10, 10, 0.01)
    free = vertices[:, 0] > 1.0e-12
    young = np.exp(np.random.default_rng(5).uniform(np.log(1.0e5), np.log(1.0e7), len(hexes)))
    mu, lam = meshes.lame_from_young(young, 0.45)
    a = sp.csr_matrix(pd_oracle.Body.hex(vertices, hexes, free, mu, lam, 1000.0).matrix(0.01))
    a.sort_indices()
    indefinite = np.asarray(((4.0, 1.0, 0.0), (1.0, 3.0, 5.0), (0.0, 5.0, 2.0)))
    lib = _lib.library()
    results, messages = [], []
    try:
        for entries in (1 << 62, 0):
            _lib.check(lib.pd_inverse_parallel_levels(entries))
            results.append(_lib.inverse_factor((a.indptr, a.indices, a.data)))
            with pytest.raises(ValueError) as info:
                _lib.inverse_factor(_lib.dense_to_csr(indefinite))
            messages.append(str(info.value))
    finally:
        _lib.check(lib.pd_inverse_parallel_levels(1 << 15))
    for key in ARRAYS:
        assert np.array_equal(results[0][key], results[1][key]), key
    assert "positive definite" in messages[0] and messages[0] == messages[1]


def test_level_path_handles_empty_and_tiny_matrices():
    """The level path forced on 0-, 1- and 2-row matrices gives the sequential loops' arrays."""
    lib = _lib.library()
    matrices = [np.zeros((0, 0)), np.eye(1) * 2.0, np.array([[4.0, 1.0], [1.0, 3.0]])]
    sequential = [_lib.inverse_factor(_lib.dense_to_csr(m)) for m in matrices]
    try:
        _lib.check(lib.pd_inverse_parallel_levels(0))
        levels = [_lib.inverse_factor(_lib.dense_to_csr(m)) for m in matrices]
    finally:
        _lib.check(lib.pd_inverse_parallel_levels(1 << 15))
    for a, b in zip(sequential, levels):
        for key in ARRAYS:
            assert np.array_equal(a[key], b[key]), key
