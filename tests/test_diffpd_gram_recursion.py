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


class KernelScheduleStep(DiffPdStep):
    """``diffpd_gram_body``'s bookkeeping step for step: pairs in a ring of ``history`` slots
    (``slot_of(age)``, age 0 the newest), the history push and the second batched sum after the
    line search, the batched sums as the kernel's product lists indexed as the kernel indexes
    them, and the Gram matrix, ``rho`` and ``s_j . g`` kept per slot between iterations."""

    def step(self, q, v, f_ext, dt):
        q = np.asarray(q, dtype=np.float64)
        v = np.asarray(v, dtype=np.float64)
        if self.dt != dt:
            self._matrix(dt)
        inertia = self.mass / dt**2
        h2m = dt * dt / self.mass
        from oracle.diff_pd_oracle import EPS, state_force
        rhs = q + dt * v + h2m * np.asarray(f_ext, dtype=np.float64) + h2m * state_force(q, v, self.mass, self.gravity,
                                                                                            self.forces)
        mask = self.free[:, None].astype(np.float64)
        self.status = self.halvings = self.fallbacks = 0
        threshold = self.rel_tol * np.linalg.norm(mask * (inertia * rhs)) + self.abs_tol
        objective = lambda x, e: 0.5 * np.sum((x - rhs) * (inertia * (x - rhs))) + e
        x = q.copy()
        energy, force, singular = self.energy_force(x)
        if singular:
            self.status |= 2
            return x, (x - q) / dt, 0
        value = objective(x, energy)
        grad = (inertia * (x - rhs) - force) * mask
        m = self.history
        s_hist, y_hist = [None] * m, [None] * m
        gram, rho, alpha, coef, sg = np.zeros((m, m)), [0.0] * m, [0.0] * m, [0.0] * m, [0.0] * m
        pairs, newest = 0, m - 1
        x_last, g_last = x, grad
        iterations = 0
        while True:
            slot_of = lambda age: (newest - age + m) % m
            for age in range(pairs):
                i = slot_of(age)
                sr = sg[i]
                for newer in range(age):
                    sr = sr - alpha[slot_of(newer)] * gram[i, slot_of(newer)]
                alpha[i] = rho[i] * sr
            r = grad.copy()
            for age in range(pairs):
                r = r - alpha[slot_of(age)] * y_hist[slot_of(age)]
            d0 = scipy.linalg.cho_solve(self.factor, r)
            products = [np.sum(y_hist[slot_of(k)] * d0) for k in range(pairs)] + [np.sum(d0 * grad), np.sum(grad * grad)]
            for age in range(pairs - 1, -1, -1):
                i = slot_of(age)
                yd = products[age]
                for older in range(pairs - 1, age, -1):
                    yd = yd + coef[slot_of(older)] * gram[slot_of(older), i]
                coef[i] = alpha[i] - rho[i] * yd
            slope = products[pairs]
            for age in range(pairs - 1, -1, -1):
                slope = slope + coef[slot_of(age)] * sg[slot_of(age)]
            if slope > 0.0:
                direction = d0
                for age in range(pairs - 1, -1, -1):
                    direction = direction + coef[slot_of(age)] * s_hist[slot_of(age)]
            else:
                slope, direction = products[pairs + 1], grad * mask
                self.fallbacks += 1
            step, evaluations = 1.0, 0
            while True:
                trial = x - step * direction
                trial_energy, trial_force, singular = self.energy_force(trial)
                trial_value = objective(trial, trial_energy)
                evaluations += 1
                if singular:
                    break
                if evaluations > self.max_ls_iter:
                    self.status |= 4
                    break
                if not np.isnan(trial_value) and trial_value < value - 1.0e-4 * step * slope + EPS:
                    break
                step /= 2.0
                self.halvings += 1
            x, value = trial, trial_value
            grad = (inertia * (x - rhs) - trial_force) * mask
            newest = (newest + 1) % m
            pairs = min(pairs + 1, m)
            slot_of = lambda age: (newest - age + m) % m
            s_hist[newest], y_hist[newest] = x - x_last, grad - g_last
            x_last, g_last = x, grad
            older = pairs - 1
            s_new, y_new = s_hist[newest], y_hist[newest]
            products = ([np.sum(grad * grad)] + [np.sum(s_hist[slot_of(age)] * grad) for age in range(pairs)]
                        + [np.sum(s_new * y_hist[slot_of(age)]) for age in range(1, older + 1)]
                        + [np.sum(s_hist[slot_of(age)] * y_new) for age in range(1, older + 1)]
                        + [np.sum(y_new * s_new)])
            assert len(products) == 3 * pairs
            for age in range(pairs):
                sg[slot_of(age)] = products[1 + age]
            for age in range(1, older + 1):
                gram[newest, slot_of(age)] = products[pairs + age]
                gram[slot_of(age), newest] = products[pairs + older + age]
            gram[newest, newest] = products[3 * pairs - 1]
            rho[newest] = 1.0 / products[3 * pairs - 1]
            iterations += 1
            if singular:
                self.status |= 2
                break
            if np.sqrt(products[0]) <= threshold:
                break
            if iterations >= self.max_pd_iter:
                self.status |= 1
                break
        return x, (x - q) / dt, iterations


@pytest.mark.parametrize("scene", DIFF_PD_SCENES)
def test_kernel_bookkeeping_matches_the_gram_recursion(scene):
    g = golden("diff_pd.npz")
    key = scene + "__"
    args = (g[key + "rest"], g[key + "tets"], 1000.0, 4.0e4, 5.0e4, g[key + "free"], (0.0, 0.0, -9.81),
            DIFF_PD_FORCES.get(scene, []))
    kernel, restated = KernelScheduleStep(*args), GramStep(*args)
    dt = float(g[key + "dt"])
    for t in range(len(g[key + "iterations"])):
        inputs = (g[key + "q_in"][t], g[key + "v_in"][t], g[key + "f"][t], dt)
        x, _, iterations = kernel.step(*inputs)
        x_ref, _, iterations_ref = restated.step(*inputs)
        assert iterations == iterations_ref == int(g[key + "iterations"][t])
        assert (kernel.halvings, kernel.fallbacks) == (restated.halvings, restated.fallbacks)
        np.testing.assert_array_equal(x, x_ref)


def test_kernel_bookkeeping_wraps_a_short_history():
    """History 2 on the long step: the ring evicts a pair every iteration, so every Gram row and
    column is rewritten in place; the step still matches the restatement bit for bit."""
    g = golden("diff_pd.npz")
    key = "history__"
    args = (g[key + "rest"], g[key + "tets"], 1000.0, 4.0e4, 5.0e4, g[key + "free"], (0.0, 0.0, -9.81), [])
    kernel, restated = KernelScheduleStep(*args, history=2), GramStep(*args, history=2)
    inputs = (g[key + "q_in"][0], g[key + "v_in"][0], g[key + "f"][0], float(g[key + "dt"]))
    x, _, iterations = kernel.step(*inputs)
    x_ref, _, iterations_ref = restated.step(*inputs)
    assert iterations == iterations_ref > 2
    np.testing.assert_array_equal(x, x_ref)
