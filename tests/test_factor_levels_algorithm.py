"""The level-by-level algorithms of the factor build, restated in Python on the CPU.

``csrc/pd_factor_device.cu`` computes the numeric LDL^T as left-looking columns
(as the threaded host path of ``csrc/factor.cpp`` does) and the rows of L^{-1}
in label chunks, level by level of the elimination tree; the host computes
the rows of L^{-1} as dense segments in groups of consecutive rows. These
tests restate the three schedules step for step (levels, label ranges, chunk
bounds recorded per stored row, merge order; group formation, outside
columns before the group's own rows, zero multipliers skipped, updates by
exact zeros, compaction; and the device's one-thread-per-label form of the
grouped schedule) and check that they reproduce the sequential
right-looking factorisation and row walk of ``oracle/factor_port.py`` bit for
bit, for chunk widths from one label (every row split everywhere) to wider
than the matrix. The CUDA kernels themselves are checked against the host
build on the GPU (``tests/test_gpu_factor_device.py``).
"""

import numpy as np
import pytest
import scipy.sparse as sp

from newton_solver_diff_phd_b200 import meshes
from oracle import factor_port, pd_oracle


def beam(nx, ny, nz):
    vertices, hexes, _ = meshes.hex_grid(nx, ny, nz, 0.01)
    free = vertices[:, 0] > 1.0e-12
    young = np.exp(np.random.default_rng(3).uniform(np.log(1.0e5), np.log(1.0e7), len(hexes)))
    mu, lam = meshes.lame_from_young(young, 0.45)
    matrix = sp.csr_matrix(pd_oracle.Body.hex(vertices, hexes, free, mu, lam, 1000.0).matrix(0.01))
    csr = factor_port._validate(matrix)
    permutation = factor_port.nested_dissection(factor_port._adjacency(csr))
    lower, diagonal = factor_port.ldlt(csr, permutation)
    return csr, permutation, lower, diagonal


def row_walk(lower):
    """The sequential walk: row i = e_i - sum_k L(i, k) row k, ascending k, exact zeros omitted."""
    rows = []
    for i in range(len(lower)):
        current = {i: 1.0}
        for k in sorted(lower[i]):
            coefficient = lower[i][k]
            if coefficient == 0.0:
                continue
            for c, value in zip(*rows[k]):
                current[c] = current.get(c, 0.0) - coefficient * value
        kept = sorted(c for c in current if current[c] != 0.0)
        rows.append((kept, [current[c] for c in kept]))
    return rows


def levels_of(lower):
    level, lo = [0] * len(lower), [0] * len(lower)
    for i in range(len(lower)):
        level[i] = max((level[k] + 1 for k in lower[i]), default=0)
        lo[i] = min([i] + [lo[k] for k in lower[i]])
    return level, lo


def chunked_rows(lower, width):
    """Rows in (row, chunk) items per level; each row keeps its chunk bounds for later rows."""
    level, lo = levels_of(lower)
    stored, bounds = {}, {}
    for current_level in range(max(level) + 1):
        for i in [r for r in range(len(lower)) if level[r] == current_level]:
            cols, vals, offsets = [], [], [0]
            for j in range(lo[i] // width, i // width + 1):
                c_begin, c_end = max(lo[i], j * width), min(i, (j + 1) * width - 1) + 1
                acc = [1.0 if c_begin + t == i else 0.0 for t in range(c_end - c_begin)]
                for k in sorted(lower[i]):
                    coefficient = lower[i][k]
                    j0 = lo[k] // width
                    if coefficient == 0.0 or not j0 <= j <= k // width:
                        continue
                    b, e = bounds[k][j - j0], bounds[k][j - j0 + 1]
                    for c, value in zip(stored[k][0][b:e], stored[k][1][b:e]):
                        assert c_begin <= c < c_end
                        acc[c - c_begin] = acc[c - c_begin] - coefficient * value
                for t, value in enumerate(acc):
                    if value != 0.0:
                        cols.append(c_begin + t)
                        vals.append(value)
                offsets.append(len(cols))
            stored[i], bounds[i] = (cols, vals), offsets
    return [stored[i] for i in range(len(lower))]


def grouped_rows(lower, width, group_rows, share):
    """Dense segments [lo_i, i] per row; groups of consecutive rows; per (group, chunk): the
    outside columns ascending over every row holding them, then the group's own rows."""
    n = len(lower)
    _, lo = levels_of(lower)
    starts, a, mark = [0], 0, {}
    for r in range(1, n):
        outside = [k for k in lower[r] if k < a]
        shared = sum(mark.get(k) == a for k in outside)
        if r - a >= group_rows or shared < share * len(outside):
            a = r
            starts.append(r)
        for k in lower[r]:
            if k < a:
                mark[k] = a
    starts.append(n)
    dense = {}
    for a, b in zip(starts[:-1], starts[1:]):  # consecutive groups: every outside row is done
        union = sorted({k for r in range(a, b) for k in lower[r] if k < a})
        for j in range(min(lo[a:b]) // width, (b - 1) // width + 1):
            c0, c1 = j * width, (j + 1) * width
            tile = {r: [1.0 if c0 + t == r else 0.0 for t in range(width)] for r in range(a, b)}
            for k in union + list(range(a, b - 1)):
                source = dense[k] if k < a else None
                for r in range(max(a, k + 1), b):
                    coefficient = lower[r].get(k, 0.0)
                    if coefficient == 0.0:
                        continue
                    for c in range(max(lo[k], c0), min(k + 1, c1)):
                        value = source[c - lo[k]] if k < a else tile[k][c - c0]
                        tile[r][c - c0] = tile[r][c - c0] - coefficient * value
            for r in range(a, b):
                segment = dense.setdefault(r, [0.0] * (r - lo[r] + 1))
                for c in range(max(lo[r], c0), min(r + 1, c1)):
                    segment[c - lo[r]] = tile[r][c - c0]
    rows = []
    for i in range(n):
        kept = [(lo[i] + u, value) for u, value in enumerate(dense[i]) if value != 0.0]
        rows.append(([c for c, _ in kept], [value for _, value in kept]))
    return rows


def grouped_rows_by_label(lower, width, group_rows, share):
    """``inverse_rows_group_kernel``'s view of the grouped schedule: one thread per label c of a
    (group, chunk) item holds the entries (a + r, c) of the group's rows, applies the outside
    columns k with lo_k <= c <= k in ascending order, then its own rows, and writes the entries
    inside each row's labels; groups in elimination order, levels replaced by that order."""
    n = len(lower)
    _, lo = levels_of(lower)
    starts, a, mark = [0], 0, {}
    for r in range(1, n):
        outside = [k for k in lower[r] if k < a]
        shared = sum(mark.get(k) == a for k in outside)
        if r - a >= group_rows or shared < share * len(outside):
            a = r
            starts.append(r)
        for k in lower[r]:
            if k < a:
                mark[k] = a
    starts.append(n)
    dense = [[None] * (i - lo[i] + 1) for i in range(n)]
    for a, b in zip(starts[:-1], starts[1:]):
        rows = b - a
        union = sorted({k for r in range(a, b) for k in lower[r] if k < a})
        outer = [[lower[a + r].get(k, 0.0) for r in range(rows)] for k in union]
        inner = [[lower[a + r].get(a + kk, 0.0) if kk < r else 0.0 for kk in range(rows)] for r in range(rows)]
        for j in range(min(lo[a:b]) // width, (b - 1) // width + 1):
            for t in range(width):
                c = j * width + t
                acc = [1.0 if a + r == c else 0.0 for r in range(rows)]
                for u, k in enumerate(union):
                    if c < lo[k] or c > k:
                        continue
                    x = dense[k][c - lo[k]]
                    for r in range(rows):
                        if outer[u][r] != 0.0:
                            acc[r] = acc[r] - outer[u][r] * x
                for kk in range(rows - 1):
                    k = a + kk
                    if lo[k] <= c <= k:
                        for r in range(kk + 1, rows):
                            if inner[r][kk] != 0.0:
                                acc[r] = acc[r] - inner[r][kk] * acc[kk]
                for r in range(rows):
                    if lo[a + r] <= c <= a + r:
                        dense[a + r][c - lo[a + r]] = acc[r]
    rows_out = []
    for i in range(n):
        kept = [(lo[i] + u, value) for u, value in enumerate(dense[i]) if value != 0.0]
        rows_out.append(([c for c, _ in kept], [value for _, value in kept]))
    return rows_out


def left_looking(csr, permutation, lower, dense=False):
    """Columns level by level: entry (i, j) = A(i, j) - sum m(i, k) e(j, k) over shared k, ascending.
    With ``dense`` (the host's top levels) the sum runs over every column k < j of row i, reading
    e(j, k) = 0 where row j lacks k; such a column k may not be factored yet, and row i then still
    holds A(i, k) there, a finite value times zero."""
    n = len(lower)
    permuted = sp.csr_matrix(csr[permutation][:, permutation])
    initial = {(i, int(k)): permuted[i, int(k)] for i in range(n) for k in list(lower[i]) + [i]}
    pattern = [sorted(lower[i]) for i in range(n)]
    rows_of = [[] for _ in range(n)]
    for i in range(n):
        for k in pattern[i]:
            rows_of[k].append(i)
    level, _ = levels_of(lower)
    unscaled, multiplier, pivot = {}, {}, [0.0] * n
    for current_level in range(max(level) + 1):
        columns = [j for j in range(n) if level[j] == current_level]
        for j in columns:
            acc = initial[(j, j)]
            for k in pattern[j]:
                acc = acc - multiplier[(j, k)] * unscaled[(j, k)]
            pivot[j] = acc
            for i in rows_of[j]:
                acc = initial[(i, j)]
                shared = [k for k in pattern[i] if k < j and (dense or k in lower[j])]
                for k in shared:  # ascending: the merge of two sorted patterns
                    acc = acc - multiplier.get((i, k), initial[(i, k)]) * unscaled.get((j, k), 0.0)
                unscaled[(i, j)] = acc
        for j in columns:
            for i in rows_of[j]:
                multiplier[(i, j)] = unscaled[(i, j)] / pivot[j]
    return multiplier, pivot


@pytest.mark.parametrize("width", [1, 3, 16, 64, 4096])
def test_chunked_rows_reproduce_the_row_walk(width):
    _, _, lower, _ = beam(6, 3, 3)
    walk = row_walk(lower)
    for (cols, vals), (ref_cols, ref_vals) in zip(chunked_rows(lower, width), walk):
        assert cols == ref_cols
        assert np.array_equal(np.asarray(vals), np.asarray(ref_vals))


@pytest.mark.parametrize("dense", [False, True])
def test_left_looking_columns_reproduce_the_right_looking_factor(dense):
    csr, permutation, lower, diagonal = beam(8, 3, 3)
    multiplier, pivot = left_looking(csr, permutation, lower, dense)
    assert np.array_equal(np.asarray(pivot), diagonal)
    for i, row in enumerate(lower):
        for k, value in row.items():
            assert multiplier[(i, k)] == value


@pytest.mark.parametrize("width, group_rows, share", [(1, 32, 0.5), (7, 4, 0.5), (64, 32, 0.0), (4096, 2, 1.0)])
def test_grouped_dense_rows_reproduce_the_row_walk(width, group_rows, share):
    _, _, lower, _ = beam(6, 3, 3)
    walk = row_walk(lower)
    for (cols, vals), (ref_cols, ref_vals) in zip(grouped_rows(lower, width, group_rows, share), walk):
        assert cols == ref_cols
        assert np.array_equal(np.asarray(vals), np.asarray(ref_vals))


@pytest.mark.parametrize("width, group_rows", [(16, 32), (256, 4)])
def test_grouped_rows_by_label_reproduce_the_row_walk(width, group_rows):
    _, _, lower, _ = beam(6, 3, 3)
    walk = row_walk(lower)
    for (cols, vals), (ref_cols, ref_vals) in zip(grouped_rows_by_label(lower, width, group_rows, 0.5), walk):
        assert cols == ref_cols
        assert np.array_equal(np.asarray(vals), np.asarray(ref_vals))
