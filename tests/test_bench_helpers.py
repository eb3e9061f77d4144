"""Host-side arithmetic of bench.py's batched leg, on stand-in solvers (no GPU).

The batched roofline's algorithmic bytes follow the per-iteration formula of
the path (factor products, vectors, elements, Anderson history, convergence,
refinement residual), with nnz(A) counted from the Hex8 grid's 27-point
stencil; the stalled-instance report states each instance's nominal strain
F / (E A).
"""

import numpy as np
import pytest

import bench
from newton_solver_diff_phd_b200.scenes import Cantilever


class FakeSolver:
    def __init__(self, nnz_s, window):
        self.nnz_s = nnz_s
        self.anderson_window = window

    def factor_stats(self):
        return 0, self.nnz_s, 0


def test_batched_roofline_counts_the_algorithmic_bytes():
    spec = Cantilever(2, 2, 2, 1.0e6, 0.4, np.zeros(9))
    family = [(spec, None, FakeSolver(nnz_s=1000, window=5), None)]
    iterations = np.array([[3], [4]])
    result = bench.batched_roofline(family, iterations, forward_ms=1.0)
    n, e, nnz_a = 27, 8, 343  # 3x3x3 vertices; (2 + 3 + 2)^3 stencil entries
    per_iteration = (2 * (1000 * 8 + 4 * (n + 1)) + 2 * (3 * n * 4) * 2 + e * 8 * 4 + 3 * e * 8 + 2 * 3 * n * 8
                     + (2 * 5 + 4) * 3 * n * 8 + 4 * 3 * n * 8 + nnz_a * 12 + 2 * 3 * n * 8)
    assert result["algorithmic_bytes_per_launch"] == pytest.approx(7 * per_iteration)
    assert result["achieved"] == pytest.approx(7 * per_iteration / 1.0e-3 / 1.0e9)
    assert result["frac"] == pytest.approx(result["achieved"] / result["peak"])
    assert result["bound"] == "hbm" and result["traffic"] is None


def test_stalled_instances_report_the_nominal_strain():
    tip = np.full(9, 10.0)  # 3 x 3 tip face of a 2 x 2 cross-section
    family = [(Cantilever(4, 2, 2, 2.0e5, 0.4, tip), None, None, None),
              (Cantilever(4, 2, 2, 1.0e7, 0.4, tip), None, None, None)]
    report = bench.stalled_instances(family, np.array([1, 0]))
    assert [r["instance"] for r in report] == [0]
    area = 2 * 2 * 0.01 * 0.01
    assert report[0]["tip_force_n"] == pytest.approx(90.0)
    assert report[0]["nominal_strain"] == pytest.approx(90.0 / (2.0e5 * area))
