"""CPU port of the reference's sparse DiffPhD path, used as the timed CPU baseline.

TEST INFRASTRUCTURE ONLY (imported by tests/ and by bench.py's CPU-baseline
leg). It follows the reference's CPU code path step for step: the local step
over all elements, the fixed-order gather, ``x = S^T (S b)`` with the exact
inverse factor (``sparse.py:322-352``), Dirichlet values, type-II Anderson
with a ring history (``anderson.py``), the dual stopping gate
(``kernels.py:294-347``), and the backward fixed point ``mu <- A^{-1}(g + K mu)``
with Anderson and the dual-norm stop (``adjoint.py:927-964, 1054-1086``).

The reference's own CPU path (Warp CPU kernels) needs warp-lang and newton,
which are not installed; this port runs the same algorithm with NumPy/SciPy
(SpMV in SciPy's compiled CSR kernels, projections vectorised over elements).
The factor arrays come from the caller (they are bit-identical to the
reference's ``sparse.py`` output).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import pd_oracle


class SparsePort:
    """The reference's sparse step and adjoint on the host cores.

    ``threads > 1`` spreads the element projections (NumPy's batched SVD
    releases the GIL) and the row blocks of the two factor products over a
    thread pool; the arithmetic of every element and every row is unchanged.
    """

    def __init__(self, body: pd_oracle.Body, factor: dict, dt: float, window: int = 5, threads: int = 1):
        n = body.n
        self.body = body
        self.dt = dt
        self.window = window
        self.inertia = body.mass / dt**2
        self.s = sp.csr_matrix((factor["s_values"], factor["s_columns"], factor["s_offsets"]), shape=(n, n))
        self.st = sp.csr_matrix((factor["st_values"], factor["st_columns"], factor["st_offsets"]), shape=(n, n))
        self.threads = max(1, int(threads))
        self.pool = None
        if self.threads > 1:
            from concurrent.futures import ThreadPoolExecutor

            self.pool = ThreadPoolExecutor(self.threads)
            rows = np.linspace(0, n, self.threads + 1).astype(int)
            self.s_blocks = [self.s[a:b] for a, b in zip(rows[:-1], rows[1:])]
            self.st_blocks = [self.st[a:b] for a, b in zip(rows[:-1], rows[1:])]
            cuts = np.linspace(0, len(body.elements), self.threads + 1).astype(int)
            self.element_blocks = list(zip(cuts[:-1], cuts[1:]))
        # The corotated + volume pair shares one SVD per sample (Tet4 or Hex8
        # without fibres or planes, the path's plain workloads).
        self.fast_projection = (self.pool is not None and body.material == "pd" and body.muscle_directions is None
                                and body.planes is None)

    def _product(self, blocks, vector):
        return np.vstack(list(self.pool.map(lambda block: block @ vector, blocks)))

    def solve(self, rhs):
        if self.pool is None:
            return self.st @ (self.s @ rhs)
        return self._product(self.st_blocks, self._product(self.s_blocks, rhs))

    def _contributions(self, bounds, x, boundary):
        body = self.body
        lo, hi = bounds
        elements, gradients = body.elements[lo:hi], body.gradients[lo:hi]
        f = np.einsum("eki,eskj->esij", x[elements], gradients)
        fd = np.einsum("eki,eskj->esij", boundary[elements], gradients)
        u, sigma, vh = np.linalg.svd(f)
        offsets = pd_oracle.volume_offsets(sigma.reshape(-1, 3)).reshape(sigma.shape)
        volume = body.sample_volume[lo:hi]
        stress = np.zeros_like(f)
        stress += (2.0 * body.mu[lo:hi, None] * volume)[..., None, None] * (u @ vh - fd)
        stress += (body.lame[lo:hi, None] * volume)[..., None, None] * (u @ ((sigma + offsets)[..., :, None] * vh) - fd)
        return np.einsum("esij,eskj->eki", stress, gradients)

    def projection_rhs(self, x, boundary, targets=None):
        body = self.body
        if not self.fast_projection:
            return body.projection_rhs(x, boundary, targets)
        parts = list(self.pool.map(lambda bounds: self._contributions(bounds, x, boundary), self.element_blocks))
        p = np.zeros((body.n, 3))
        np.add.at(p, body.elements.ravel(), np.concatenate(parts).reshape(-1, 3))
        return p

    def _anderson(self):
        return {"x": [], "g": []}

    @staticmethod
    def _mix(history, x, previous, window):
        g = x - previous
        history["x"].append(previous)
        history["g"].append(g)
        m = len(history["g"]) - 1
        if m >= 1:
            dg = np.stack([(history["g"][i + 1] - history["g"][i]).ravel() for i in range(m)], axis=1)
            dx = np.stack([(history["x"][i + 1] - history["x"][i]).ravel() for i in range(m)], axis=1)
            gram = dg.T @ dg
            gram += max(1.0e-6 * np.trace(gram) / m, 1.0e-12) * np.eye(m)
            gamma = np.linalg.solve(gram, dg.T @ g.ravel())
            if np.linalg.norm(gamma) >= 10.0:
                history["x"].clear()
                history["g"].clear()
            else:
                x = ((previous + g).ravel() - (dx + dg) @ gamma).reshape(-1, 3)
        del history["x"][:-window]
        del history["g"][:-window]
        return x

    def step(self, q, v, f_ext, gravity, *, max_iterations, abs_tol, rel_tol, boundary=None, targets=None):
        body, dt = self.body, self.dt
        q = np.asarray(q, dtype=np.float64)
        v = np.asarray(v, dtype=np.float64)
        free = body.free
        if boundary is None:
            boundary = np.where(free[:, None], 0.0, q)
        q_tilde = q + dt * v + dt**2 * (np.asarray(f_ext, np.float64) / body.mass + np.asarray(gravity, np.float64))
        x = q.copy()
        previous_p = np.zeros_like(x)
        history = self._anderson()
        for iteration in range(max_iterations):
            previous = x
            p = self.projection_rhs(x, boundary, targets)
            x = self.solve(self.inertia * q_tilde + p)
            x[~free] = boundary[~free]
            if self.window:
                x = self._mix(history, x, previous, self.window)
            x[~free] = boundary[~free]
            step_norm = np.linalg.norm(x - previous)
            change = np.linalg.norm(p - previous_p)
            done = (iteration > 0 and step_norm <= rel_tol * np.linalg.norm(previous) + abs_tol
                    and change <= rel_tol * np.linalg.norm(previous_p) + abs_tol)
            previous_p = p
            if done:
                return x, iteration + 1, True
        return x, max_iterations, False

    def backward(self, x_next, dl_dq, dl_dv, *, max_iterations, abs_tol, rel_tol, targets=None, mode="reference"):
        """Adjoint fixed point of one step; returns ``mu`` and the material gradient."""
        body, dt = self.body, self.dt
        free = body.free
        k_matrix = sp.csr_matrix(pd_oracle.stiffness_matrix_blocks(body, x_next, targets, mode))
        rhs = np.asarray(dl_dq, np.float64) + np.asarray(dl_dv, np.float64) / dt
        solution = np.zeros_like(rhs)
        history = self._anderson()
        for iteration in range(max_iterations):
            previous = solution
            work = rhs + (k_matrix @ solution.ravel()).reshape(-1, 3)
            raw = self.solve(work)
            raw[~free] = 0.0
            step_norm = np.linalg.norm(raw - previous)
            if self.window:
                raw = self._mix(history, raw, previous, self.window)
            raw[~free] = 0.0
            solution = raw
            if iteration > 0 and step_norm < rel_tol * np.linalg.norm(raw) + abs_tol:
                break
        f = body.deformation(x_next)
        material = np.zeros((len(body.elements), 2))
        for name, _weight in body.energies():
            if name == "corotated":
                stress = f - pd_oracle.corotated(f)
            elif name == "volume":
                stress = f - pd_oracle.volume_projection(f)
            else:
                continue
            value = -np.einsum("eki,esij,eskj,es->e", solution[body.elements], stress, body.gradients, body.sample_volume)
            material[:, 1 if name == "volume" else 0] += value if name == "volume" else 2.0 * value
        return solution, material, iteration + 1


    def backward_cg(self, x_next, dl_dq, dl_dv, *, max_iterations, abs_tol, rel_tol, targets=None, mode="exact"):
        """The same adjoint solve by conjugate gradients on ``(A - K) mu = g`` over the free rows,
        preconditioned by ``A^{-1} = S^T S`` (the preconditioned residual is the fixed-point step, so
        the stop rule ``|z| < rel |mu| + abs`` is the fixed point's). Returns ``mu``, the material
        gradient and the iteration count."""
        body, dt = self.body, self.dt
        free = body.free
        if not hasattr(self, "a_matrix"):
            self.a_matrix = sp.csr_matrix(body.matrix(dt))
        k_matrix = sp.csr_matrix(pd_oracle.stiffness_matrix_blocks(body, x_next, targets, mode))
        r = np.asarray(dl_dq, np.float64) + np.asarray(dl_dv, np.float64) / dt
        r[~free] = 0.0
        mu = np.zeros_like(r)
        p = np.zeros_like(r)
        previous_rho = 0.0
        iterations = 0
        for k in range(max_iterations):
            z = self.solve(r)
            z[~free] = 0.0
            rho = float(np.sum(r * z))
            iterations = k + 1
            if k > 0 and np.linalg.norm(z) < rel_tol * np.linalg.norm(mu) + abs_tol:
                break
            if not rho > 0.0:
                break
            beta = 0.0 if k == 0 or not previous_rho > 0.0 else rho / previous_rho
            previous_rho = rho
            p = z + beta * p
            p[~free] = 0.0
            q = self.a_matrix @ p - (k_matrix @ p.ravel()).reshape(-1, 3)
            q[~free] = 0.0
            curvature = float(np.sum(p * q))
            if not curvature > 0.0:
                break
            alpha = rho / curvature
            mu = mu + alpha * p
            r = r - alpha * q
        f = body.deformation(x_next)
        material = np.zeros((len(body.elements), 2))
        for name, _weight in body.energies():
            if name == "corotated":
                stress = f - pd_oracle.corotated(f)
            elif name == "volume":
                stress = f - pd_oracle.volume_projection(f)
            else:
                continue
            value = -np.einsum("eki,esij,eskj,es->e", mu[body.elements], stress, body.gradients, body.sample_volume)
            material[:, 1 if name == "volume" else 0] += value if name == "volume" else 2.0 * value
        return mu, material, iterations


def time_hex_iterations(job):
    """Cost of one forward local/global iteration and of one adjoint CG iteration of one Hex8
    instance with this port, from a given state: ``(particles, forward s/iteration, adjoint
    s/iteration)``. ``job`` is ``(vertices, hexes, free, mu, lame, forces, factor, q, v, dt,
    iterations)`` with ``factor`` the inverse factor of ``body.matrix(dt)`` (picklable: a process
    pool measures instances side by side)."""
    import time

    vertices, hexes, free, mu, lame, forces, factor, q, v, dt, iterations = job
    body = pd_oracle.Body.hex(vertices, hexes, free, mu, lame, 1000.0)
    port = SparsePort(body, factor, dt)
    q = np.asarray(q, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    start = time.perf_counter()
    x, _, _ = port.step(q, v, forces, np.zeros(3), max_iterations=iterations, abs_tol=0.0, rel_tol=0.0)
    forward = (time.perf_counter() - start) / iterations
    seed = np.ones_like(q)
    start = time.perf_counter()
    _, _, count = port.backward_cg(x, seed, np.zeros_like(seed), max_iterations=iterations, abs_tol=0.0, rel_tol=0.0)
    adjoint = (time.perf_counter() - start) / max(count, 1)
    return len(vertices), forward, adjoint
