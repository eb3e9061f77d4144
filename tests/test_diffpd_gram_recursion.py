"""The Gram-matrix form of the L-BFGS two-loop recursion, restated in NumPy on the CPU.

The ``gram`` recursion of ``csrc/pd_diffpd.cu`` (``SolverDiffPD(two_loop="gram")``)
never forms the two loops' intermediate vectors: it keeps the matrix
``G[i][j] = s_i . y_j`` of the stored pairs and the products ``s_i . g``,
computes the first loop's ``s_i . r_i = s_i . g - sum_{j newer} alpha_j G[i][j]``
and the second loop's ``y_i . d_i = y_i . d_0 + sum_{j older} c_j G[j][i]``
from them, ``r = g - sum alpha_j y_j`` and ``d = d_0 + sum c_j s_j`` in the
reference's elementwise order, and the slope ``d . g`` as
``d_0 . g + sum c_j (s_j . g)``. Every dot product of an iteration then falls
into two batched team sums instead of one per pair and loop. The sums are
rounded in a different order than the reference's two loops
(``diff_pd/solver.py`` two-loop, restated in ``oracle/diff_pd_oracle.py``);
this restatement, in the kernel's order of operations, keeps every golden
iteration count, halving and fallback of the reference's scenes and lands
within 1e-11 m of the golden positions (3.5e-12 m on the 160-iteration step
whose history wraps, below 1e-15 m on the others).
"""

import numpy as np
import pytest
import scipy.linalg

from oracle.diff_pd_oracle import DiffPdStep
from tests.helpers import golden
from tests.test_oracle import DIFF_PD_FORCES, DIFF_PD_SCENES


class GramStep(DiffPdStep):
    def two_loop(self, grad, pairs):
        m = len(pairs)
        S = [s for s, _ in pairs]
        Y = [y for _, y in pairs]
        gram = [[np.sum(S[i] * Y[j]) for j in range(m)] for i in range(m)]
        sg = [np.sum(s * grad) for s in S]
        rho = [1.0 / gram[i][i] for i in range(m)]
        alpha = [0.0] * m
        for i in reversed(range(m)):
            sr = sg[i]
            for j in reversed(range(i + 1, m)):
                sr = sr - alpha[j] * gram[i][j]
            alpha[i] = rho[i] * sr
        r = grad.copy()
        for j in reversed(range(m)):
            r = r - alpha[j] * Y[j]
        d0 = scipy.linalg.cho_solve(self.factor, r)
        coef = [0.0] * m
        for i in range(m):
            yd = np.sum(Y[i] * d0)
            for j in range(i):
                yd = yd + coef[j] * gram[j][i]
            coef[i] = alpha[i] - rho[i] * yd
        slope = np.sum(d0 * grad)
        direction = d0
        for j in range(m):
            slope = slope + coef[j] * sg[j]
            direction = direction + coef[j] * S[j]
        return direction, slope


@pytest.mark.parametrize("scene", DIFF_PD_SCENES)
def test_gram_recursion_keeps_the_golden_iterations(scene):
    g = golden("diff_pd.npz")
    key = scene + "__"
    step = GramStep(g[key + "rest"], g[key + "tets"], 1000.0, 4.0e4, 5.0e4, g[key + "free"], (0.0, 0.0, -9.81),
                    DIFF_PD_FORCES.get(scene, []))
    dt = float(g[key + "dt"])
    for t in range(len(g[key + "iterations"])):
        x, v, iterations = step.step(g[key + "q_in"][t], g[key + "v_in"][t], g[key + "f"][t], dt)
        assert iterations == int(g[key + "iterations"][t])
        assert step.halvings == int(g[key + "halvings"][t])
        assert step.fallbacks == int(g[key + "fallbacks"][t])
        np.testing.assert_allclose(x, g[key + "q_out"][t], rtol=0.0, atol=1.0e-11)
