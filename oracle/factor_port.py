"""CPU restatement of the reference's exact inverse factor setup.

TEST INFRASTRUCTURE ONLY (imported by tests/ and by bench.py's CPU legs; the
product builds its factor with ``csrc/factor.cpp``). It restates the host
setup of ``src/newton_solver_diff_phd/_src/solvers/diff_phd/sparse.py``:

* ordering: nested dissection by BFS level sets, each part ordered
  recursively, parts of at most 24 vertices and every separator by minimum
  degree with ties to the lowest index (``sparse.py:18-70``);
* ``P A P^T = L D L^T`` with the reference's rounding sequence
  (``sparse.py:98-156``): every multiplier is ``U_ik / d_k`` of the entry
  before division, and every entry subtracts ``multiplier * U_jk`` over
  pivots ``k`` in increasing order. Here the elimination is organised by rows
  (left-looking, a dense accumulator per row, the pattern from the
  elimination tree) instead of the reference's right-looking pivot loop; the
  operands and their order per entry are the same, so the factor is
  bit-identical;
* ``S = D^{-1/2} L^{-1} P`` row by row (``sparse.py:159-177``), exact zeros
  dropped, then CSR of ``S`` (rows in elimination order, columns in particle
  order) and of ``S^T`` (``sparse.py:180-190, 300-307``).

Pinned by ``tests/test_oracle.py`` against ``tests/golden/sparse_factors.npz``
(made by the reference's own ``sparse.py``).
"""

from __future__ import annotations

from collections import deque

import numpy as np
import scipy.sparse as sp

LEAF = 24


def _adjacency(csr: sp.csr_matrix) -> list[set[int]]:
    out = []
    for i in range(csr.shape[0]):
        row = set(csr.indices[csr.indptr[i]:csr.indptr[i + 1]].tolist())
        row.discard(i)
        out.append(row)
    return out


def minimum_degree(nodes: set[int], adjacency: list[set[int]]) -> list[int]:
    """Greedy elimination of ``nodes`` (graph restricted to them), fewest neighbours first."""
    graph = {v: adjacency[v] & nodes for v in nodes}
    order = []
    while graph:
        best = None
        for v, neighbours in graph.items():
            key = (len(neighbours), v)
            if best is None or key < best:
                best = key
        v = best[1]
        neighbours = graph.pop(v)
        order.append(v)
        for w in neighbours:
            others = graph[w]
            others.discard(v)
            others |= neighbours
            others.discard(w)
    return order


def _levels(start: int, nodes: set[int], adjacency: list[set[int]]) -> dict[int, int]:
    level = {start: 0}
    queue = deque((start,))
    while queue:
        v = queue.popleft()
        for w in adjacency[v]:
            if w in nodes and w not in level:
                level[w] = level[v] + 1
                queue.append(w)
    return level


def nested_dissection(adjacency: list[set[int]]) -> np.ndarray:
    """Elimination order (position -> original row) of the reference's ordering."""

    def order(nodes: set[int]) -> list[int]:
        if len(nodes) <= LEAF:
            return minimum_degree(nodes, adjacency)
        start = min(nodes, key=lambda v: (len(adjacency[v] & nodes), v))
        level = _levels(start, nodes, adjacency)
        if len(level) != len(nodes):
            parts = [set(level)]
            rest = nodes - parts[0]
            while rest:
                part = set(_levels(min(rest), rest, adjacency))
                parts.append(part)
                rest -= part
            return [v for part in parts for v in order(part)]
        far = max(level.values())
        peripheral = min(v for v, d in level.items() if d == far)
        level = _levels(peripheral, nodes, adjacency)
        counts = np.bincount(np.fromiter(level.values(), dtype=np.int64))
        cut = int(np.searchsorted(np.cumsum(counts), len(nodes) / 2))
        below = {v for v in nodes if level[v] < cut}
        above = {v for v in nodes if level[v] > cut}
        if not below or not above:
            return minimum_degree(nodes, adjacency)
        middle = nodes - below - above
        return order(below) + order(above) + minimum_degree(middle, adjacency)

    return np.asarray(order(set(range(len(adjacency)))), dtype=np.int32)


def _validate(csr: sp.csr_matrix) -> sp.csr_matrix:
    csr = sp.csr_matrix(csr, dtype=np.float64)
    csr.sum_duplicates()
    csr.sort_indices()
    if not np.isfinite(csr.data).all():
        raise ValueError("matrix coefficients must be finite")
    csr.eliminate_zeros()
    n = csr.shape[0]
    if np.any(csr.diagonal() <= 0.0):
        raise ValueError("matrix must be positive definite with positive diagonal entries")
    if (csr != csr.T).nnz:
        raise ValueError("matrix_rows must contain both halves of an exactly symmetric matrix")
    if n > np.iinfo(np.int32).max:
        raise ValueError("matrix size exceeds int32 sparse indexing")
    return csr


def ldlt(csr: sp.csr_matrix, permutation: np.ndarray):
    """Rows of unit-lower ``L`` (dict column -> value, structural zeros kept) and ``D``."""
    n = csr.shape[0]
    permuted = sp.csr_matrix(csr[permutation][:, permutation])
    permuted.sort_indices()
    lower_a = sp.tril(permuted, format="csr")
    # Row patterns of L: row i holds every node on the elimination-tree paths
    # from the columns of A's row i up to i (the tree grows as rows finish:
    # a path that ends at a root hangs that root under i).
    parent = np.full(n, -1, dtype=np.int64)
    patterns = []
    mark = np.full(n, -1, dtype=np.int64)
    for i in range(n):
        columns = lower_a.indices[lower_a.indptr[i]:lower_a.indptr[i + 1]]
        pattern = []
        mark[i] = i
        for j in columns:
            j = int(j)
            while j < i and mark[j] != i:
                pattern.append(j)
                mark[j] = i
                if parent[j] == -1:
                    parent[j] = i
                j = int(parent[j])
        patterns.append(np.asarray(sorted(pattern), dtype=np.int64))
    # Numeric factorisation, row by row: x holds the undivided entries U_i*.
    diagonal = np.empty(n, dtype=np.float64)
    column_rows = [[] for _ in range(n)]   # completed rows j with U_jk stored, increasing j
    column_values = [[] for _ in range(n)]
    lower = []
    x = np.zeros(n, dtype=np.float64)
    for i in range(n):
        lo, hi = lower_a.indptr[i], lower_a.indptr[i + 1]
        x[lower_a.indices[lo:hi]] = lower_a.data[lo:hi]
        pattern = patterns[i]
        row = {}
        for k in pattern:
            k = int(k)
            u_ik = x[k]
            multiplier = u_ik / diagonal[k]
            row[k] = multiplier
            rows = column_rows[k]
            if rows:
                x[rows] -= multiplier * np.asarray(column_values[k])
            x[i] -= multiplier * u_ik
        pivot = x[i]
        if not np.isfinite(pivot) or pivot <= 0.0:
            raise ValueError(f"matrix is not positive definite: LDLT pivot {i} is {pivot}")
        diagonal[i] = pivot
        for k in pattern:
            k = int(k)
            column_rows[k].append(i)
            column_values[k].append(x[k])
        x[pattern] = 0.0
        x[i] = 0.0
        lower.append(row)
    return lower, diagonal


def inverse_rows(lower, diagonal, permutation):
    """Rows of ``S = D^{-1/2} L^{-1} P``: (particle columns, values) per elimination row."""
    n = len(lower)
    present_rows, unscaled = [], []
    out = []
    work = np.zeros(n, dtype=np.float64)
    for i, row in enumerate(lower):
        work[: i + 1] = 0.0
        work[i] = 1.0
        for k in sorted(row):
            work[present_rows[k]] -= row[k] * unscaled[k]
        present = np.flatnonzero(work[: i + 1])
        values = work[present].copy()
        present_rows.append(present)
        unscaled.append(values)
        out.append((permutation[present], values * (1.0 / np.sqrt(diagonal[i]))))
    return out


def inverse_factor(matrix) -> dict:
    """The exact inverse factor of a symmetric positive definite matrix (dense or sparse).

    Returns the arrays of ``S`` and ``S^T`` in CSR (``s_offsets``,
    ``s_columns``, ``s_values``, ``st_*``) and the ``permutation``, like the
    product's host builder.
    """
    csr = _validate(sp.csr_matrix(matrix))
    n = csr.shape[0]
    permutation = nested_dissection(_adjacency(csr))
    lower, diagonal = ldlt(csr, permutation)
    rows = inverse_rows(lower, diagonal, permutation)
    s_offsets = np.zeros(n + 1, dtype=np.int64)
    columns, values = [], []
    for i, (cols, vals) in enumerate(rows):
        order = np.argsort(cols, kind="stable")
        columns.append(cols[order])
        values.append(vals[order])
        s_offsets[i + 1] = s_offsets[i] + len(cols)
    s_columns = np.concatenate(columns).astype(np.int32) if columns else np.zeros(0, np.int32)
    s_values = np.concatenate(values) if values else np.zeros(0)
    if not np.isfinite(s_values).all():
        raise ValueError("inverse factor overflowed float64")
    s = sp.csr_matrix((s_values, s_columns, s_offsets), shape=(n, n))
    st = sp.csr_matrix(s.T)
    st.sort_indices()
    return {
        "permutation": permutation,
        "s_offsets": s_offsets.astype(np.int32),
        "s_columns": s_columns,
        "s_values": s_values,
        "st_offsets": st.indptr.astype(np.int32),
        "st_columns": st.indices.astype(np.int32),
        "st_values": st.data.copy(),
        "factorization_nnz": n + sum(len(r) for r in lower),
    }
