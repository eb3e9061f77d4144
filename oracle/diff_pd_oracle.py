"""Dense NumPy restatement of the reference's DiffPD ``pd_eigen`` forward step.

TEST INFRASTRUCTURE ONLY (imported by tests/, by __graft_entry__.smoke() and by
bench.py's DiffPD leg, as the checker and the timed CPU baseline). It restates
``src/newton_solver_diff_phd/_src/solvers/diff_pd/solver.py:65-591`` and
``kernels.py``: the explicit state forces (gravity first, then planar and arc
penalty contacts with velocity friction, ``kernels.py:118-152``) give
``rhs = q + h v + h^2/m (f_ext + f_state(q, v))``; L-BFGS minimises
``Phi(x) = 1/2 m/h^2 |x - rhs|^2 + E_pd(x)`` from ``x = q`` with the
projective-dynamics matrix ``A`` as initial Hessian (two-loop recursion over
at most ``history`` pairs, ``rho = 1 / y.s`` without a curvature check), the
masked gradient as fallback when the direction does not descend, and a
backtracking Armijo search (``c = 1e-4``, at most ``max_ls_iter`` halvings,
the last trial accepted untested), until ``|g| <= rel |m/h^2 rhs_free| + abs``.
The element energies are the corotated ``w_c/2 |F - R|^2`` and volume
``w_v/2 |F - P_v|^2`` terms with the mean volume per element.

Vectorised over elements with NumPy's SVD and a dense factorisation of ``A``.
Pinned by ``tests/test_oracle.py`` against ``tests/golden/diff_pd.npz``, which
``tests/golden/make_diff_pd_golden.py`` made with the reference's own
``tests/reference_oracle_diff_pd.py``.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg

from .pd_oracle import volume_offsets

EPS = np.finfo(np.float64).eps


def state_force(q, v, mass, gravity, forces):
    """Gravity ``m g`` then each (kind, raw parameters) contact in order, for every particle."""
    total = np.broadcast_to(mass * np.asarray(gravity, np.float64), q.shape).copy()
    for kind, parameters in forces:
        p = np.asarray(parameters, dtype=np.float64)
        if kind == "planar_contact":
            normal = p[:3] / np.linalg.norm(p[:3])
            offset = p[3] / np.linalg.norm(p[:3])
            power, kn, kf, mu = int(p[4]), p[5], p[6], p[7]
            distance = q @ normal + offset
            fn = kn * (-np.minimum(0.0, distance)) ** (power - 1)
            normals = np.broadcast_to(normal, q.shape)
            active = np.ones(len(q), dtype=bool)
        else:
            center, axis, start = p[:3], p[3:6] / np.linalg.norm(p[3:6]), p[6:9] / np.linalg.norm(p[6:9])
            aux = np.cross(axis, start)
            radius, angle, power, kn, kf, mu = p[9], p[10], int(p[11]), p[12], p[13], p[14]
            local = q - center
            projected = local - (local @ axis)[:, None] * axis
            theta = np.arctan2(projected @ aux, projected @ start)
            active = (theta > 0.0) & (theta < angle)
            length = np.linalg.norm(projected, axis=1)
            fn = kn * (-np.minimum(0.0, radius - length)) ** (power - 1)
            normals = -projected / (length + EPS)[:, None]
        tangential = v - np.sum(v * normals, axis=1)[:, None] * normals
        friction = np.minimum(kf, mu * fn / (np.linalg.norm(tangential, axis=1) + EPS))
        force = fn[:, None] * normals - friction[:, None] * tangential
        total += np.where(active[:, None], force, 0.0)
    return total


class DiffPdStep:
    """The reference step on a Tet4 mesh; ``step`` returns ``(x, v, iterations)`` and records
    ``halvings``, ``fallbacks`` and the status bits (1 not converged, 2 singular, 4 line search)."""

    def __init__(self, rest, tets, density, corotated, volume, free, gravity, forces=(), *, max_pd_iter=4000,
                 max_ls_iter=10, abs_tol=1.0e-9, rel_tol=1.0e-4, history=10):
        rest = np.asarray(rest, dtype=np.float64)
        self.tets = np.asarray(tets, dtype=np.int64)
        self.free = np.asarray(free, dtype=bool)
        self.gravity = np.asarray(gravity, dtype=np.float64)
        self.forces = list(forces)
        self.weights = [(name, w) for name, w in (("corotated", corotated), ("volume", volume)) if w is not None]
        self.max_pd_iter, self.max_ls_iter = max_pd_iter, max_ls_iter
        self.abs_tol, self.rel_tol, self.history = abs_tol, rel_tol, history
        corners = rest[self.tets]
        edges = np.transpose(corners[:, 1:] - corners[:, :1], (0, 2, 1))
        inverse = np.linalg.inv(edges)
        self.gradients = np.concatenate((-inverse.sum(axis=1)[:, None], inverse), axis=1)   # (E, 4, 3)
        a, b, c = edges[:, :, 0], edges[:, :, 1], edges[:, :, 2]
        volumes = np.abs(np.einsum("ei,ei->e", a, np.cross(b, c)) / 6.0)
        self.volume = float(sum(volumes.tolist()) / len(volumes))
        self.mass = density * self.volume
        self.dt = None

    def _matrix(self, dt):
        n = len(self.free)
        inertia = self.mass / dt**2
        a = np.diag(np.where(self.free, inertia, 1.0))
        weight = sum(w for _, w in self.weights)
        blocks = np.einsum("eic,ejc->eij", self.gradients, self.gradients) * weight * self.volume
        rows = np.repeat(self.tets, 4, axis=1).ravel()
        cols = np.tile(self.tets, (1, 4)).ravel()
        mask = self.free[rows] & self.free[cols]
        np.add.at(a, (rows[mask], cols[mask]), blocks.reshape(-1)[mask])
        self.factor = scipy.linalg.cho_factor(a)
        self.dt = dt

    def energy_force(self, x):
        """Total energy, per-particle forces and whether a volume projection met a singular F."""
        f = np.einsum("eki,ekj->eij", x[self.tets], self.gradients)
        u, sigma, vh = np.linalg.svd(f)
        energy = 0.0
        stress = np.zeros_like(f)
        singular = False
        for name, w in self.weights:
            if name == "corotated":
                projected = u @ vh
            else:
                singular |= bool(np.any(sigma.min(axis=1) < EPS))
                offsets = volume_offsets(sigma)
                projected = u @ ((sigma + offsets)[..., :, None] * vh)
            difference = f - projected
            energy += float(np.sum(w * 0.5 * np.einsum("eij,eij->e", difference, difference) * self.volume))
            stress += w * difference
        contributions = -np.einsum("eij,ekj->eki", stress, self.gradients) * self.volume
        force = np.zeros_like(x)
        np.add.at(force, self.tets.ravel(), contributions.reshape(-1, 3))
        return energy, force, singular

    def step(self, q, v, f_ext, dt):
        q = np.asarray(q, dtype=np.float64)
        v = np.asarray(v, dtype=np.float64)
        if self.dt != dt:
            self._matrix(dt)
        inertia = self.mass / dt**2
        h2m = dt * dt / self.mass
        rhs = q + dt * v + h2m * np.asarray(f_ext, dtype=np.float64) + h2m * state_force(q, v, self.mass, self.gravity,
                                                                                            self.forces)
        mask = self.free[:, None].astype(np.float64)
        self.status = 0
        self.halvings = self.fallbacks = 0

        def objective(x, energy):
            return 0.5 * np.sum((x - rhs) * (inertia * (x - rhs))) + energy

        x = q.copy()
        energy, force, singular = self.energy_force(x)
        if singular:
            self.status |= 2
            return x, (x - q) / dt, 0
        value = objective(x, energy)
        grad = (inertia * (x - rhs) - force) * mask
        threshold = self.rel_tol * np.linalg.norm(mask * (inertia * rhs)) + self.abs_tol
        pairs = []   # (s, y) oldest first
        x_last = g_last = None
        for iteration in range(self.max_pd_iter):
            if x_last is not None:
                pairs.append((x - x_last, grad - g_last))
                if len(pairs) > self.history:
                    pairs.pop(0)
            x_last, g_last = x, grad
            direction, slope = self.two_loop(grad, pairs)
            if slope <= 0:
                direction = grad * mask
                slope = np.sum(grad * grad)
                self.fallbacks += 1
            step = 1.0
            evaluations = 0
            while True:
                trial = x - step * direction
                trial_energy, trial_force, singular = self.energy_force(trial)
                trial_value = objective(trial, trial_energy)
                evaluations += 1
                if singular:
                    self.status |= 2
                    return trial, (trial - q) / dt, iteration + 1
                if evaluations > self.max_ls_iter:
                    self.status |= 4
                    break
                if not np.isnan(trial_value) and trial_value < value - 1.0e-4 * step * slope + EPS:
                    break
                step /= 2.0
                self.halvings += 1
            x, value = trial, trial_value
            grad = (inertia * (x - rhs) - trial_force) * mask
            if np.linalg.norm(grad) <= threshold:
                return x, (x - q) / dt, iteration + 1
        self.status |= 1
        return x, (x - q) / dt, self.max_pd_iter

    def two_loop(self, grad, pairs):
        """The L-BFGS direction ``H grad`` with ``A^{-1}`` as initial inverse Hessian over ``pairs``
        (oldest first) and its slope ``direction . grad``."""
        r = grad.copy()
        rhos = [1.0 / np.sum(y * s) for s, y in pairs]
        alphas = [0.0] * len(pairs)
        for k in reversed(range(len(pairs))):
            s, y = pairs[k]
            alphas[k] = rhos[k] * np.sum(s * r)
            r = r - alphas[k] * y
        direction = scipy.linalg.cho_solve(self.factor, r)
        for k in range(len(pairs)):
            s, y = pairs[k]
            beta = rhos[k] * np.sum(y * direction)
            direction = direction + s * (alphas[k] - beta)
        return direction, np.sum(direction * grad)
