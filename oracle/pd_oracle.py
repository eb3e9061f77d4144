"""Dense NumPy oracle of the DiffPhD projective-dynamics step and its adjoint.

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the product path never
does. It restates the reference algorithm independently of the CUDA kernels:

* projections with NumPy's SVD (``projections.py:88-316`` conventions),
  vectorised over all element samples;
* the constant matrix assembled densely and solved with a Cholesky factor
  (the reference applies it as ``S^T S``, ``sparse.py``);
* type-II Anderson mixing with list history and the dual stopping gate
  (``anderson.py:276-317``, ``kernels.py:294-401``, ``solver.py:582-659``);
* Hex8 with isoparametric trilinear quadrature at the eight Gauss points, the
  quadrature of ``HexOracle`` (``tests/test_diff_phd_hex.py:39-109``);
* the backward pass with finite-difference projection Jacobians and a dense
  solve of ``(A - K)_FF mu = g_F`` (``reference_backward``,
  ``tests/reference_oracle.py:477-615``), with K from the mean weight per energy
  (``mode="reference"``, ``adjoint.py:17-18``) or from per-element weights
  (``mode="exact"``).

Pinning: tests/test_oracle.py checks this module against the vectors in
tests/golden, which tests/golden/make_golden.py generated by running the
reference's own ``tests/reference_oracle.py``, ``HexOracle`` and ``sparse.py``.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg

EPS = np.finfo(np.float64).eps


# --------------------------------------------------------------------------- projections
def svd(f):
    """Batched unsigned SVD: ``F = U diag(sigma) V^T`` with sigma >= 0 descending."""
    u, sigma, vh = np.linalg.svd(f)
    return u, sigma, np.swapaxes(vh, -1, -2)


def corotated(f):
    u, _, v = svd(f)
    return u @ np.swapaxes(v, -1, -2)


def volume_offsets(sigma):
    """Offsets D with prod(sigma + D) = 1 by the reference fixed point (50 iterations, eps stop)."""
    sigma = np.atleast_2d(sigma)
    product = np.prod(sigma, axis=1)
    d = sigma / (product ** (1.0 / 3.0))[:, None] - sigma
    done = np.zeros(len(sigma), dtype=bool)
    for _ in range(50):
        s = sigma + d
        constraint = np.prod(s, axis=1) - 1.0
        gradient = np.stack((s[:, 1] * s[:, 2], s[:, 0] * s[:, 2], s[:, 0] * s[:, 1]), axis=1)
        following = ((np.sum(gradient * d, axis=1) - constraint) / np.sum(gradient * gradient, axis=1))[:, None] * gradient
        converged = np.max(np.abs(following - d), axis=1) <= EPS
        update = ~done & ~converged
        d = np.where(update[:, None], following, d)
        done |= converged
        if done.all():
            break
    return d


def volume_projection(f):
    u, sigma, v = svd(f)
    d = volume_offsets(sigma.reshape(-1, 3)).reshape(sigma.shape)
    return u @ ((sigma + d)[..., :, None] * np.swapaxes(v, -1, -2))


def nh_stretches(target, mu, lame, penalty):
    """Proximal Neo-Hookean singular values by damped Newton (32 iterations, floor 1e-4)."""
    target = np.atleast_2d(target)
    sigma = np.maximum(target, 1.0e-4)
    done = np.zeros(len(target), dtype=bool)
    for _ in range(32):
        log_j = np.log(np.maximum(np.prod(sigma, axis=1), 1.0e-12))
        gradient = mu * sigma - mu / sigma + (lame * log_j)[:, None] / sigma + penalty * (sigma - target)
        small = np.linalg.norm(gradient, axis=1) < 1.0e-10
        done |= small
        if done.all():
            break
        hessian = lame / (sigma[:, :, None] * sigma[:, None, :])
        idx = np.arange(3)
        hessian[:, idx, idx] = mu + (mu + lame - lame * log_j)[:, None] / sigma**2 + penalty
        hessian += 1.0e-9 * np.eye(3)
        delta = np.linalg.solve(hessian, gradient[..., None])[..., 0]
        alpha = np.ones(len(sigma))
        trial = sigma - delta
        for _ in range(20):
            bad = trial.min(axis=1) <= 0.5e-4
            if not bad.any():
                break
            alpha = np.where(bad, 0.5 * alpha, alpha)
            trial = sigma - alpha[:, None] * delta
        step = np.max(np.abs(trial - sigma), axis=1)
        new = np.maximum(trial, 1.0e-4)
        sigma = np.where(done[:, None], sigma, new)
        done |= step < 1.0e-10
        if done.all():
            break
    return sigma


def nh_projection(f, mu, lame, penalty):
    u, sigma, v = svd(f)
    s = nh_stretches(sigma.reshape(-1, 3), mu, lame, penalty).reshape(sigma.shape)
    return u @ (s[..., :, None] * np.swapaxes(v, -1, -2))


def muscle_projection(f, direction, target):
    fibre = np.einsum("...ij,...j->...i", f, direction)
    length = np.linalg.norm(fibre, axis=-1)
    scale = np.where(length > EPS, target / np.where(length > EPS, length, 1.0), 0.0)
    return scale[..., None] * fibre


# --------------------------------------------------------------------------- meshes
def tet_gradients(rest_poses):
    """Rest gradients G = [-sum rows of Dm^{-1}; Dm^{-1}] per tetrahedron, (E, 4, 3)."""
    rest_poses = np.asarray(rest_poses, dtype=np.float64)
    return np.concatenate((-rest_poses.sum(axis=1)[:, None], rest_poses), axis=1)


def hex_quadrature(vertices, hexes):
    """Isoparametric trilinear gradients and weights at the 2x2x2 Gauss points.

    Returns ``gradients (E, 8 samples, 8 corners, 3)`` and ``weights (E, 8)`` (det J).
    """
    gauss = np.array([-1.0, 1.0]) / np.sqrt(3.0)
    signs = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], dtype=np.float64)
    points = np.array([[x, y, z] for x in gauss for y in gauss for z in gauss])
    grads = np.empty((len(hexes), 8, 8, 3))
    weights = np.empty((len(hexes), 8))
    for s, p in enumerate(points):
        dn = np.empty((8, 3))
        for a in range(3):
            b, c = [k for k in range(3) if k != a]
            dn[:, a] = signs[:, a] * (1 + signs[:, b] * p[b]) * (1 + signs[:, c] * p[c]) / 8.0
        jac = np.einsum("eki,kj->eij", vertices[hexes], dn)
        inv = np.linalg.inv(jac)
        grads[:, s] = np.einsum("kj,eji->eki", dn, inv)
        weights[:, s] = np.linalg.det(jac)
    return grads, weights


class Body:
    """A soft body for the oracle: elements, per-sample gradients and volume weights.

    Tet4: ``gradients (E, 1, 4, 3)``, ``sample_volume (E, 1)`` = Vbar for every element
    (the reference gives every element the mean volume, ``solver.py:60-64``).
    Hex8: isoparametric quadrature with ``sample_volume`` = det J of each Gauss point.
    """

    def __init__(self, elements, gradients, sample_volume, mean_volume, free, mu, lame, density, material="pd",
                 muscle_directions=None, muscle_stiffness=None, planes=None, sample_weight_volume=None):
        self.elements = np.asarray(elements)
        self.gradients = np.asarray(gradients, dtype=np.float64)
        self.sample_volume = np.asarray(sample_volume, dtype=np.float64)
        self.vbar = float(mean_volume)
        self.free = np.asarray(free, dtype=bool)
        self.n = len(self.free)
        self.mu = np.asarray(mu, dtype=np.float64)
        self.lame = np.asarray(lame, dtype=np.float64)
        self.mass = density * self.vbar
        self.material = material
        self.nh = (self.mu.mean(), self.lame.mean(), 2.0 * self.mu.mean())
        self.muscle_directions = None
        if muscle_directions is not None:
            d = np.asarray(muscle_directions, dtype=np.float64)
            k = np.broadcast_to(np.asarray(muscle_stiffness, dtype=np.float64), (len(self.elements),)).copy()
            lengths = np.linalg.norm(d, axis=1)
            d = np.where(k[:, None] > 0, d / np.where(lengths > 0, lengths, 1.0)[:, None], 0.0)
            self.muscle_directions = d
            self.muscle_stiffness = k
        self.planes = None
        if planes is not None:
            nodes, stiffness, plane = planes
            plane = np.asarray(plane, dtype=np.float64)
            self.planes = (np.asarray(nodes), np.broadcast_to(np.asarray(stiffness, float), (len(nodes),)),
                           plane / np.linalg.norm(plane[:3]))

    @classmethod
    def tet(cls, tets, rest_poses, free, mu, lame, density, **kwargs):
        g = tet_gradients(rest_poses)[:, None]
        volumes = np.abs(1.0 / np.linalg.det(np.asarray(rest_poses, dtype=np.float64))) / 6.0
        vbar = volumes.mean()
        return cls(tets, g, np.full((len(tets), 1), vbar), vbar, free, mu, lame, density, **kwargs)

    @classmethod
    def hex(cls, vertices, hexes, free, mu, lame, density, **kwargs):
        g, w = hex_quadrature(np.asarray(vertices, dtype=np.float64), np.asarray(hexes))
        vbar = w.sum(axis=1).mean()
        return cls(hexes, g, w, vbar, free, mu, lame, density, **kwargs)

    # energies: list of (name, weight per element-sample (E, S))
    def energies(self):
        if self.material == "pd":
            return [("corotated", 2.0 * self.mu[:, None] * self.sample_volume),
                    ("volume", self.lame[:, None] * self.sample_volume)]
        return [("neo_hookean", 2.0 * self.mu[:, None] * self.sample_volume)]

    def matrix(self, dt):
        """Dense constant matrix with Dirichlet rows eliminated (identity)."""
        a = np.diag(np.where(self.free, self.mass / dt**2, 1.0))
        total = sum(weight for _name, weight in self.energies())
        g = self.gradients
        gg = np.einsum("eskc,eslc->eskl", g, g)
        block = (total[..., None, None] * gg).sum(axis=1)
        if self.muscle_directions is not None:
            fibre = np.einsum("eskc,ec->esk", g, self.muscle_directions)
            mw = self.muscle_stiffness[:, None] * self.sample_volume
            block = block + (mw[..., None, None] * fibre[..., :, None] * fibre[..., None, :]).sum(axis=1)
        k = self.elements.shape[1]
        rows = np.repeat(self.elements, k, axis=1).ravel()
        cols = np.tile(self.elements, (1, k)).ravel()
        values = block.reshape(len(self.elements), -1).ravel()
        mask = self.free[rows] & self.free[cols]
        np.add.at(a, (rows[mask], cols[mask]), values[mask])
        if self.planes is not None:
            nodes, stiffness, _plane = self.planes
            for i, k_i in zip(nodes, stiffness):
                if self.free[i]:
                    a[i, i] += k_i
        return a

    def deformation(self, x):
        return np.einsum("eki,eskj->esij", x[self.elements], self.gradients)

    def projection_rhs(self, x, boundary, targets=None):
        f = self.deformation(x)
        fd = self.deformation(boundary)
        stress = np.zeros_like(f)
        for name, weight in self.energies():
            if name == "corotated":
                projected = corotated(f)
            elif name == "volume":
                projected = volume_projection(f)
            else:
                projected = nh_projection(f, *self.nh)
            stress += weight[..., None, None] * (projected - fd)
        if self.muscle_directions is not None:
            m = self.muscle_directions[:, None, :]
            t = np.asarray(targets, dtype=np.float64)[:, None]
            fibre = muscle_projection(f, np.broadcast_to(m, f.shape[:-1]), np.broadcast_to(t, f.shape[:2]))
            fdm = np.einsum("esij,ej->esi", fd, self.muscle_directions)
            mw = self.muscle_stiffness[:, None] * self.sample_volume
            stress += mw[..., None, None] * (fibre - fdm)[..., :, None] * self.muscle_directions[:, None, None, :]
        contributions = np.einsum("esij,eskj->eki", stress, self.gradients)
        p = np.zeros((self.n, 3))
        np.add.at(p, self.elements.ravel(), contributions.reshape(-1, 3))
        if self.planes is not None:
            nodes, stiffness, plane = self.planes
            gap = x[nodes] @ plane[:3] + plane[3]
            projected = x[nodes] - np.minimum(0.0, gap)[:, None] * plane[:3]
            p[nodes] += stiffness[:, None] * (projected - boundary[nodes])
        return p


# --------------------------------------------------------------------------- forward
def step(body, q, v, f_ext, gravity, dt, *, max_iterations, abs_tol, rel_tol, window=5, boundary=None,
         targets=None, integrate_pinned=False, contact=None):
    """One reference step. Returns ``(x, iterations, converged)``.

    ``contact`` is a :class:`FrictionalBoundary`; its multipliers carry over
    from call to call like the solver's warm start.
    """
    q = np.asarray(q, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    if boundary is None:
        boundary = np.where(body.free[:, None], 0.0, q + (dt * v if integrate_pinned else 0.0))
    q_tilde = q + dt * v + dt**2 * (np.asarray(f_ext, dtype=np.float64) / body.mass + np.asarray(gravity, float))
    matrix = body.matrix(dt)
    factor = scipy.linalg.cho_factor(matrix)
    inertia = body.mass / dt**2
    if contact is not None:
        contact.begin_step(q, np.linalg.inv(matrix), dt)
    x = q.copy()
    previous_rhs = np.zeros_like(x)
    history_x, history_g = [], []
    step_small = rhs_small = False
    for iteration in range(max_iterations):
        p = body.projection_rhs(x, boundary, targets)
        x_previous = x
        x = scipy.linalg.cho_solve(factor, inertia * q_tilde + p)
        if contact is not None and len(contact.nodes):
            x = contact.iterate(x_previous, x, q)
        x[~body.free] = boundary[~body.free]
        if window > 0:
            g = x - x_previous
            history_x.append(x_previous)
            history_g.append(g)
            m = len(history_g) - 1
            if m >= 1:
                dg = np.stack([(history_g[i + 1] - history_g[i]).ravel() for i in range(m)], axis=1)
                dx = np.stack([(history_x[i + 1] - history_x[i]).ravel() for i in range(m)], axis=1)
                gram = dg.T @ dg
                gram += max(1.0e-6 * np.trace(gram) / m, 1.0e-12) * np.eye(m)
                gamma = np.linalg.solve(gram, dg.T @ g.ravel())
                if np.linalg.norm(gamma) >= 10.0:
                    history_x.clear()
                    history_g.clear()
                else:
                    x = ((x_previous + g).ravel() - (dx + dg) @ gamma).reshape(-1, 3)
                    x[~body.free] = boundary[~body.free]
            del history_x[:-window]
            del history_g[:-window]
        step_small = np.linalg.norm(x - x_previous) <= rel_tol * np.linalg.norm(x_previous) + abs_tol
        rhs_small = np.linalg.norm(p - previous_rhs) <= rel_tol * np.linalg.norm(previous_rhs) + abs_tol
        previous_rhs = p
        if iteration > 0 and step_small and rhs_small:
            if contact is not None:
                x = contact.restitution(x, q, v, dt)
            return x, iteration + 1, True
    if contact is not None:
        x = contact.restitution(x, q, v, dt)
    return x, max_iterations, False


# --------------------------------------------------------------------------- backward
def _projection_jacobian(project, f, eps=1.0e-6):
    """Central-difference (9 x 9) Jacobians of a batched projection, column-major flattening."""
    jac = np.zeros(f.shape[:-2] + (9, 9))
    for c in range(9):
        df = np.zeros((3, 3))
        df[c % 3, c // 3] = 1.0
        derivative = (project(f + eps * df) - project(f - eps * df)) / (2.0 * eps)
        jac[..., :, c] = np.swapaxes(derivative, -1, -2).reshape(derivative.shape[:-2] + (9,))
    return jac


def sample_jacobians(body, x, targets=None, mode="reference"):
    """Weighted projection Jacobians ``w dP/dF`` per element sample, (E, S, 9, 9), column-major flattening."""
    f = body.deformation(x)
    e_count, s_count = f.shape[:2]
    jac = np.zeros((e_count, s_count, 9, 9))
    for name, weight in body.energies():
        if name == "corotated":
            project = corotated
        elif name == "volume":
            project = volume_projection
        else:
            project = lambda m: nh_projection(m, *body.nh)  # noqa: E731
        if mode == "reference":
            # The reference's K uses the mean weight of each energy (adjoint.py:827-832).
            w = np.full_like(weight, weight.mean())
        else:
            w = weight
        jac += w[..., None, None] * _projection_jacobian(project, f)
    if body.muscle_directions is not None:
        m = body.muscle_directions
        t = np.asarray(targets, dtype=np.float64)
        mw = body.muscle_stiffness[:, None] * body.sample_volume

        def fibre(mat):
            return muscle_projection(mat, np.broadcast_to(m[:, None], mat.shape[:-1]),
                                     np.broadcast_to(t[:, None], mat.shape[:2]))[..., :, None] * m[:, None, None, :]

        jac += mw[..., None, None] * _projection_jacobian(fibre, f)
    return jac


def stiffness_blocks(body, x, targets=None, mode="reference"):
    """Element blocks of K = sum_s G^T (w dP/dF) G as ``(E, K, 3, K, 3)`` plus their global dof indices."""
    jac = sample_jacobians(body, x, targets, mode)
    e_count, s_count = jac.shape[:2]
    # jac[..., b + 3c, b2 + 3c2] -> J4[..., c, b, c2, b2]
    j4 = jac.reshape(e_count, s_count, 3, 3, 3, 3)
    local = np.einsum("eskc,escbCB,eslC->ekblB", body.gradients, j4, body.gradients)
    corners = body.elements.shape[1]
    dofs = (3 * body.elements[:, :, None] + np.arange(3)[None, None, :]).reshape(e_count, 3 * corners)
    return local.reshape(e_count, 3 * corners, 3 * corners), dofs


def stiffness_matrix_blocks(body, x, targets=None, mode="reference"):
    """K as a SciPy CSR matrix (3N x 3N, xyz-interleaved dofs)."""
    import scipy.sparse as sp

    local, dofs = stiffness_blocks(body, x, targets, mode)
    size = dofs.shape[1]
    rows = np.repeat(dofs, size, axis=1).ravel()
    cols = np.tile(dofs, (1, size)).ravel()
    return sp.coo_matrix((local.ravel(), (rows, cols)), shape=(3 * body.n, 3 * body.n)).tocsr()


def stiffness_matrix(body, x, targets=None, mode="reference"):
    """K = sum_e sum_s G^T (w dP/dF) G, dense (3N x 3N) with xyz-interleaved dofs."""
    return stiffness_matrix_blocks(body, x, targets, mode).toarray()


def _backward_tangents(normal):
    """``_backward_tangents`` (adjoint.py:322-344): Gram-Schmidt from the axis least parallel to n."""
    axis = 0
    for d in (1, 2):
        if abs(normal[d]) < abs(normal[axis]):
            axis = d
    unit = np.eye(3)[axis]
    t1 = unit - (normal @ unit) * normal
    length = np.sqrt(t1 @ t1)
    t1 = t1 / length if length > 1.0e-12 else np.array([1.0, 0.0, 0.0])
    t2 = np.cross(normal, t1)
    length = np.sqrt(t2 @ t2)
    t2 = t2 / length if length > 1.0e-12 else np.array([0.0, 1.0, 0.0])
    return t1, t2


def woodbury_projection(operator, free, mu, contact):
    """``z = mu - W_T G^{-1} (J mu)`` of the contact rows (adjoint.py:347-471, :1272-1354).

    ``contact`` is ``(nodes, multipliers, omega, normals, friction)`` of the
    forward step. Rows: ``omega n`` of every contact with ``lambda > 0`` and
    ``omega >= 0.5``, then, with friction, the two tangents of those with
    ``lambda > 1e-8``; rows with ``|J mu| < max(1e-12, 1e-3 max|J mu|)`` are
    dropped; the columns ``(A - K)^{-1} J^T`` are solved directly here.
    """
    nodes, multiplier, omega, normal, friction = contact
    n3 = len(mu)
    rows = []
    for c, node in enumerate(nodes):
        if multiplier[c] > 0 and omega[c] >= 0.5:
            rows.append((node, omega[c] * normal[c]))
    if friction > 0:
        for c, node in enumerate(nodes):
            if multiplier[c] > 0 and omega[c] >= 0.5 and multiplier[c] > 1.0e-8:
                rows.extend((node, t) for t in _backward_tangents(normal[c]))
    if not rows:
        return mu.copy()
    values = np.array([vector @ mu[3 * node:3 * node + 3] for node, vector in rows])
    gate = max(1.0e-12, 1.0e-3 * np.abs(values).max())
    keep = np.abs(values) >= gate
    rows = [row for row, selected in zip(rows, keep) if selected]
    values = values[keep]
    columns = []
    for node, vector in rows:
        j = np.zeros(n3)
        j[3 * node:3 * node + 3] = vector
        column = np.zeros(n3)
        column[free] = np.linalg.solve(operator, j[free])
        columns.append(column)
    gram = np.array([[vector @ columns[k][3 * node:3 * node + 3] for k in range(len(rows))] for node, vector in rows])
    gram = np.tril(gram) + np.tril(gram, -1).T
    alpha = np.linalg.solve(gram, values)
    return mu - sum(a * column for a, column in zip(alpha, columns))


def backward(body, x_next, dt, dl_dq_next, dl_dv_next, targets=None, mode="reference", contact=None):
    """Dense adjoint of one step: ``mu``, ``z`` and the gradients of the step inputs, materials and
    (with fibres) the contractions; ``contact`` projects the parameter gradients (:func:`woodbury_projection`)."""
    n = body.n
    free = np.repeat(body.free, 3)
    k_matrix = stiffness_matrix(body, x_next, targets, mode)
    a_matrix = np.kron(body.matrix(dt), np.eye(3))
    operator = (a_matrix - k_matrix)[np.ix_(free, free)]
    rhs = (np.asarray(dl_dq_next) + np.asarray(dl_dv_next) / dt).ravel()
    mu = np.zeros(3 * n)
    mu[free] = np.linalg.solve(operator, rhs[free])
    inertia = body.mass / dt**2
    out = {
        "mu": mu.reshape(-1, 3),
        "q": (-(np.asarray(dl_dv_next).ravel() / dt) + inertia * mu).reshape(-1, 3),
        "qd": (dt * inertia * mu).reshape(-1, 3),
        "f": mu.reshape(-1, 3).copy(),
    }
    # Dirichlet values: g_D - (A - K)_DF mu_F without the mass term.
    pinned = ~free
    if pinned.any():
        coupling = np.zeros(3 * n)
        unassembled = element_matrix(body, dt) - k_matrix
        coupling[pinned] = (unassembled[np.ix_(pinned, free)] @ mu[free])
        out["dirichlet"] = np.where(pinned, rhs - coupling, 0.0).reshape(-1, 3)
    z = (mu if contact is None else woodbury_projection(operator, free, mu, contact)).reshape(-1, 3)
    out["z"] = z
    f = body.deformation(x_next)
    material = np.zeros((len(body.elements), 2))
    for name, weight in body.energies():
        if name == "corotated":
            stress = f - corotated(f)
        elif name == "volume":
            stress = f - volume_projection(f)
        else:
            mu_bar, lame_bar, _penalty = body.nh
            inverse_t = np.swapaxes(np.linalg.inv(f), -1, -2)
            pk1 = mu_bar * (f - inverse_t) + (lame_bar * np.log(np.maximum(np.linalg.det(f), 1.0e-12)))[..., None, None] * inverse_t
            stress = pk1 / (2.0 * mu_bar)
        # -z^T Vs G^T (F - P): contributions per sample, summed.
        value = -np.einsum("eki,esij,eskj,es->e", z[body.elements], stress, body.gradients, body.sample_volume)
        if name == "volume":
            material[:, 1] += value
        else:
            material[:, 0] += 2.0 * value
    out["materials"] = material
    if body.muscle_directions is not None:
        # dL/du = sum_k z_k . (w_m / |F m| (m . g_k)) F m (adjoint.py:647-659).
        m = body.muscle_directions
        fibre = np.einsum("esij,ej->esi", f, m)
        length = np.linalg.norm(fibre, axis=-1)
        mw = body.muscle_stiffness[:, None] * body.sample_volume
        scale = np.where(length > EPS, mw / np.where(length > EPS, length, 1.0), 0.0)
        mg = np.einsum("ej,eskj->esk", m, body.gradients)
        out["activations"] = -np.einsum("eki,esk,es,esi->e", z[body.elements], mg, scale, fibre)
    return out


def element_matrix(body, dt):
    """Unassembled element operator sum_e w G^T G (+ fibres), 3N x 3N, without mass or elimination."""
    total = sum(weight for _name, weight in body.energies())
    g = body.gradients
    gg = np.einsum("eskc,eslc->eskl", g, g)
    block = (total[..., None, None] * gg).sum(axis=1)
    k = body.elements.shape[1]
    scalar = np.zeros((body.n, body.n))
    rows = np.repeat(body.elements, k, axis=1).ravel()
    cols = np.tile(body.elements, (1, k)).ravel()
    np.add.at(scalar, (rows, cols), block.reshape(len(body.elements), -1).ravel())
    result = np.kron(scalar, np.eye(3))
    if body.muscle_directions is not None:
        m = body.muscle_directions
        mw = body.muscle_stiffness[:, None] * body.sample_volume
        for e in range(len(body.elements)):
            for s in range(g.shape[1]):
                fibre = g[e, s] @ m[e]
                local = mw[e, s] * np.kron(np.outer(fibre, fibre), np.outer(m[e], m[e]))
                dofs = np.array([3 * i + d for i in body.elements[e] for d in range(3)])
                result[np.ix_(dofs, dofs)] += local
    return result


def rollout(body, q0, v0, forces, gravity, dt, steps, **options):
    """Forward rollout; returns the list of positions after every step and iteration counts."""
    q, v = np.asarray(q0, float), np.asarray(v0, float)
    positions, iterations = [], []
    for t in range(steps):
        f = forces(t) if callable(forces) else forces
        x, it, _ = step(body, q, v, f, gravity, dt, **options)
        v = (x - q) / dt
        q = x
        positions.append(x)
        iterations.append(it)
    return positions, iterations


# ---------------------------------------------------------------------------
# The reference's mesh_contact state force (mesh_contact.py:34-210): penalty
# plus velocity friction between the surface vertices of one body and the
# faces of the other, evaluated once per step on the start-of-step state.


def closest_point_on_triangle(p, a, b, c):
    """Closest point of triangle abc to p and its barycentric weights (Voronoi regions, mesh_contact.py:34-76)."""
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = ab @ ap, ac @ ap
    if d1 <= 0.0 and d2 <= 0.0:
        return a, np.array((1.0, 0.0, 0.0))
    bp = p - b
    d3, d4 = ab @ bp, ac @ bp
    if d3 >= 0.0 and d4 <= d3:
        return b, np.array((0.0, 1.0, 0.0))
    vc = d1 * d4 - d3 * d2
    if vc <= 0.0 and d1 >= 0.0 and d3 <= 0.0:
        t = d1 / (d1 - d3)
        return a + t * ab, np.array((1.0 - t, t, 0.0))
    cp = p - c
    d5, d6 = ab @ cp, ac @ cp
    if d6 >= 0.0 and d5 <= d6:
        return c, np.array((0.0, 0.0, 1.0))
    vb = d5 * d2 - d1 * d6
    if vb <= 0.0 and d2 >= 0.0 and d6 <= 0.0:
        t = d2 / (d2 - d6)
        return a + t * ac, np.array((1.0 - t, 0.0, t))
    va = d3 * d6 - d5 * d4
    if va <= 0.0 and (d4 - d3) >= 0.0 and (d5 - d6) >= 0.0:
        t = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        return b + t * (c - b), np.array((0.0, 1.0 - t, t))
    scale = 1.0 / (va + vb + vc)
    v, w = vb * scale, vc * scale
    return a + ab * v + ac * w, np.array((1.0 - v - w, v, w))


def _pair_force(p, face_points, vp, face_velocities, radius, kn, kf, mu):
    """Force on the vertex from one face (zero outside the radius) and the closest point's weights."""
    a, b, c = face_points
    closest, weights = closest_point_on_triangle(p, a, b, c)
    gap2 = (p - closest) @ (p - closest)
    if gap2 >= radius * radius:
        return None
    gap = np.sqrt(gap2)
    if gap > EPS:
        normal = (p - closest) / gap
    else:
        normal = np.cross(b - a, c - a)
        length = np.linalg.norm(normal)
        if length <= EPS:
            return None
        normal = normal / length
    if normal @ (p - closest) < 0.0:
        normal = -normal
    magnitude = kn * (radius - gap)
    relative = vp - weights @ face_velocities
    tangential = relative - normal * (relative @ normal)
    speed = np.linalg.norm(tangential)
    friction = np.zeros(3)
    if speed > EPS:
        friction = -min(kf, mu * magnitude / (speed + EPS)) * tangential
    return magnitude * normal + friction, weights


def mesh_contact_force(q, v, faces_a, faces_b, radius, kn_left, kn_right, kf, mu):
    """Per-particle force [N]: A's surface vertices against B's faces with kn_left, B's against A's with kn_right."""
    q, v = np.asarray(q, dtype=np.float64), np.asarray(v, dtype=np.float64)
    faces_a, faces_b = np.asarray(faces_a), np.asarray(faces_b)
    force = np.zeros_like(q)
    for vertices, faces, kn in ((np.unique(faces_a), faces_b, kn_left), (np.unique(faces_b), faces_a, kn_right)):
        for vid in vertices:
            for face in faces:
                hit = _pair_force(q[vid], q[face], v[vid], v[face], radius, kn, kf, mu)
                if hit is None:
                    continue
                total, weights = hit
                force[vid] += total
                force[face] -= np.outer(weights, total)
    return force


# ---------------------------------------------------------------------------
# The reference's frictional boundary (contact.py:77-1015): per local/global
# iteration one semismooth Newton step on the Fischer-Burmeister function of
# every registered vertex against a planar, spherical or mesh boundary, an
# isotropic Coulomb stick/slip update, and the position correction through
# the columns A^{-1} e_j of the registered vertices.


def _boundary_gap(point, kind, parameters):
    """``boundary_gap`` (contact.py:77-89): signed distance to the plane or sphere."""
    if kind == "planar":
        axis = parameters[:3]
        norm = np.sqrt(axis @ axis)
        unit = axis / norm
        return point[0] * unit[0] + point[1] * unit[1] + point[2] * unit[2] + parameters[3] / norm
    offset = point - parameters[:3]
    return np.sqrt(offset @ offset) - parameters[3]


def _boundary_normal(point, kind, parameters):
    """``boundary_normal`` (contact.py:92-98)."""
    if kind == "planar":
        axis = parameters[:3]
        return axis / np.sqrt(axis @ axis)
    offset = point - parameters[:3]
    return offset / np.sqrt(offset @ offset)


def _plane_frame(normal):
    """``GetLocalFrame`` (contact.py:182-193): t1 = normalize(n x e_i) of the axis maximising |n x e_i|."""
    best = np.zeros(3)
    for i in range(3):
        candidate = np.cross(normal, np.eye(3)[i])
        if candidate @ candidate > best @ best:
            best = candidate
    t1 = best / np.sqrt(best @ best)
    t2 = np.cross(normal, t1)
    return t1, t2 / np.sqrt(t2 @ t2)


def _gram_schmidt_frame(normal):
    """Tangents of a mesh contact (contact.py:225-236): from the axis least parallel to n, first on ties."""
    axis = 0
    for d in (1, 2):
        if abs(normal[d]) < abs(normal[axis]):
            axis = d
    unit = np.eye(3)[axis]
    t1 = unit - (normal @ unit) * normal
    t1 = t1 / np.sqrt(t1 @ t1)
    t2 = np.cross(normal, t1)
    return t1, t2 / np.sqrt(t2 @ t2)


class FrictionalBoundary:
    """Frictional boundary of the reference step with the device's arithmetic layout.

    ``kind`` is ``"planar"`` with ``parameters = (nx, ny, nz, offset)``,
    ``"spherical"`` with ``(cx, cy, cz, radius)``, or ``"mesh"`` with
    ``(contact_radius, split_index, faces_left, faces_right)``. The Delassus
    matrix is ``W_ij = (n_i . n_j) B_ij`` with ``B = A^{-1}`` restricted to the
    registered vertices (contact.py:242-256); only candidates with ``omega != 0``
    enter the coupled Newton block (contact.py:450-528), the others take
    ``d lambda = rhs / E`` (contact.py:531-546).
    """

    def __init__(self, kind, parameters, nodes, friction=0.0, restitution=0.0):
        self.kind = kind
        self.nodes = np.asarray(nodes, dtype=np.int64)
        self.friction = float(friction)
        self.restitution_coefficient = float(restitution)
        k = len(self.nodes)
        self.multiplier = np.zeros(k)
        self.lambda_t = np.zeros((k, 2))
        if kind == "mesh":
            radius, split, left, right = parameters
            self.radius, self.split = float(radius), int(split)
            self.faces_left = np.asarray(left, dtype=np.int64).reshape(-1, 3)
            self.faces_right = np.asarray(right, dtype=np.int64).reshape(-1, 3)
            self.parameters = np.array([self.radius, 0.0, 0.0, 0.0])
        else:
            self.parameters = np.asarray(parameters, dtype=np.float64)
        self.candidate = np.ones(k, dtype=bool)
        self.omega = np.zeros(k)

    # -- mesh geometry (contact.py:101-148)
    def closest(self, p, node, x):
        """Closest point, unit face normal and squared distance on the surface opposite ``node``."""
        faces = self.faces_right if node < self.split else self.faces_left
        best, closest, normal = np.inf, np.zeros(3), np.array([0.0, 0.0, 1.0])
        for a, b, c in faces:
            point, _ = closest_point_on_triangle(p, x[a], x[b], x[c])
            dist2 = (p - point) @ (p - point)
            if dist2 < best:
                best, closest = dist2, point
                n = np.cross(x[b] - x[a], x[c] - x[a])
                length = np.sqrt(n @ n)
                normal = n / length if length > EPS else np.array([0.0, 0.0, 1.0])
        return closest, normal, best

    @staticmethod
    def direction(p, closest, face_normal):
        offset = p - closest
        length = np.sqrt(offset @ offset)
        return offset / length if length > 1.0e-12 else face_normal

    def begin_step(self, q, inverse, dt):
        """Panel, frames, candidates, Delassus matrix and regularisation of the step (contact.py:775-836)."""
        q = np.asarray(q, dtype=np.float64)
        k = len(self.nodes)
        self.panel = inverse[:, self.nodes]
        self.block = self.panel[self.nodes]
        self.normal = np.zeros((k, 3))
        self.t1 = np.zeros((k, 3))
        self.t2 = np.zeros((k, 3))
        for c, node in enumerate(self.nodes):
            if self.kind == "mesh":
                closest, face_normal, dist2 = self.closest(q[node], node, q)
                self.candidate[c] = np.sqrt(dist2) - self.radius <= 5.0 * self.radius
                n = self.direction(q[node], closest, face_normal)
                t1, t2 = _gram_schmidt_frame(n)
                if not self.candidate[c]:
                    self.multiplier[c] = 0.0
            else:
                n = _boundary_normal(q[node], self.kind, self.parameters)
                t1, t2 = _plane_frame(n)
            self.normal[c], self.t1[c], self.t2[c] = n, t1, t2
        self.lambda_t[:] = 0.0
        cosines = self.normal @ self.normal.T
        self.delassus = cosines * np.tril(self.block) + (cosines * np.tril(self.block, -1)).T
        self.regularization = np.maximum(dt * dt * np.diag(self.delassus), 1.0e-10)

    def _scalars(self, x):
        k = len(self.nodes)
        delta = np.zeros(k)
        omega = np.zeros(k)
        diagonal = np.ones(k)
        residual = np.zeros(k)
        if self.kind == "mesh":
            self.surface = x.copy()
        for c, node in enumerate(self.nodes):
            if not self.candidate[c]:
                continue
            if self.kind == "mesh":
                closest, _, _ = self.closest(x[node], node, x)
                delta[c] = (x[node] - closest) @ self.normal[c] - self.radius
            else:
                delta[c] = _boundary_gap(x[node], self.kind, self.parameters)
            lam, r = self.multiplier[c], self.regularization[c]
            s = max(np.sqrt(delta[c] * delta[c] + r * r * lam * lam), 1.0e-14)
            omega[c] = 1.0 - delta[c] / s
            diagonal[c] = (1.0 - r * lam / s) * r
            residual[c] = delta[c] + r * lam - s
        return delta, omega, diagonal, residual

    def _forces(self, omega, tangential):
        force = (omega * self.multiplier)[:, None] * self.normal
        if tangential:
            force = force + self.lambda_t[:, :1] * self.t1 + self.lambda_t[:, 1:] * self.t2
        return force

    def iterate(self, x, solved, q):
        """One Newton step and friction update; returns ``A^{-1} (b + J^T lambda)`` (contact.py:909-984)."""
        nodes = self.nodes
        delta, omega, diagonal, residual = self._scalars(x)
        self.omega = omega
        active = np.flatnonzero(omega != 0.0)
        force = self._forces(omega, True)
        response = self.block[:, active] @ force[active]
        rhs = -residual + omega * np.einsum("ij,ij->i", self.normal, x[nodes])
        rhs -= omega * np.einsum("ij,ij->i", self.normal, solved[nodes] + response)
        step = np.divide(rhs, diagonal, out=np.zeros_like(rhs), where=omega == 0.0)
        if len(active):
            system = omega[active, None] * self.delassus[np.ix_(active, active)] * omega[None, active]
            system[np.diag_indices(len(active))] += diagonal[active]
            step[active] = np.linalg.solve(system, rhs[active])
        self.multiplier = np.clip(self.multiplier + step, 0.0, 1.0e8)
        if self.friction > 0:
            normal_response = self.block[:, active] @ self._forces(omega, False)[active]
            for c, node in enumerate(nodes):
                if self.multiplier[c] <= 0.0:
                    self.lambda_t[c] = 0.0
                    continue
                move = solved[node] + normal_response[c] - q[node]
                n = self.normal[c]
                tangential = move - (move @ n) * n
                u1, u2 = tangential @ self.t1[c], tangential @ self.t2[c]
                diagonal_c = self.block[c, c]
                w11 = (self.t1[c] @ self.t1[c]) * diagonal_c
                w12 = (self.t1[c] @ self.t2[c]) * diagonal_c
                w22 = (self.t2[c] @ self.t2[c]) * diagonal_c
                determinant = w11 * w22 - w12 * w12
                stick = np.zeros(2)
                if abs(determinant) > 1.0e-20:
                    stick = np.array((-(w22 * u1 - w12 * u2), -(-w12 * u1 + w11 * u2))) / determinant
                radius = self.friction * self.multiplier[c]
                if np.sqrt(stick @ stick) <= radius + 1.0e-14:
                    self.lambda_t[c] = stick
                else:
                    magnitude = np.sqrt(u1 * u1 + u2 * u2)
                    self.lambda_t[c] = (-radius * u1 / magnitude, -radius * u2 / magnitude) if magnitude > 1.0e-14 \
                        else (0.0, 0.0)
        force = self._forces(omega, True)
        return solved + self.panel[:, active] @ force[active]

    def restitution(self, x, q, v, dt):
        """Post-solve restitution (contact.py:595-667)."""
        if self.restitution_coefficient <= 0 or not len(self.nodes):
            return x
        x = x.copy()
        for c, node in enumerate(self.nodes):
            if self.multiplier[c] <= 0.0:
                continue
            point = x[node].copy()
            if self.kind == "mesh":
                reference = self.normal[c]
                closest, face_normal, _ = self.closest(point, node, self.surface)
                distance = (point - closest) @ reference - self.radius
                n = self.direction(point, closest, face_normal)
                if n @ reference < 0.0:
                    n = -n
                slop = 0.1 * self.radius
            else:
                distance = _boundary_gap(point, self.kind, self.parameters)
                n = _boundary_normal(point, self.kind, self.parameters)
                slop = 1.0e-8
            norm = np.sqrt(n @ n)
            if norm <= 1.0e-12:
                continue
            n = n / norm
            if distance > slop:
                continue
            incoming = v[node] @ n
            if incoming < 0.0:
                change = -self.restitution_coefficient * incoming - ((point - q[node]) / dt) @ n
                if change > 0.0:
                    x[node] = point + dt * change * n
        return x
