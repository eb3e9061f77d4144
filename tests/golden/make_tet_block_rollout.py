"""Generate ``tests/golden/tet_block_rollout.npz``: the Tet4 block rollout by the CPU oracle.

The workload is the bench's: a 32 x 8 x 8 block of 0.01 m cubes split into
five tetrahedra each (10,240 Tet4, 2,673 particles), per-tet Young's modulus
log-uniform in [1e5, 1e7] Pa from ``default_rng(0)``, nu 0.4, density 1000,
gravity -9.81, the x = 0 face pinned, 50 steps of dt 5e-3 at rel 1e-6, abs
1e-9, Anderson window 5; the loss is ``|q_50 - target|^2`` with the target the
rest pose plus a seeded 1 mm Gaussian displacement.

Everything runs on the CPU through ``oracle/``: the exact inverse factor of
``oracle/factor_port.py`` (bit-identical to the reference's ``sparse.py``),
the forward step and the exact-mode adjoint (conjugate gradients
preconditioned by the factor) of ``oracle/sparse_port.py``, with float32
states between steps like Newton's (and the solver's) state arrays. Stored
every ``STRIDE`` steps: the step's input state and the loss gradient with
respect to its output state; plus the iteration counts of every step, the
final positions, the loss and dL/dE.

    python tests/golden/make_tet_block_rollout.py      # about ten minutes on 8 cores
"""

from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

STRIDE = 2


def workload():
    """Oracle body, factor and the rollout inputs, from the same model arrays the solver gets."""
    from newton_solver_diff_phd_b200 import ModelBuilder, meshes
    from oracle import factor_port, pd_oracle

    nx, ny, nz, edge = 32, 8, 8, 0.01
    vertices, tets, _ = meshes.tet_grid(nx, ny, nz, edge)
    rng = np.random.default_rng(0)
    young = np.exp(rng.uniform(np.log(1.0e5), np.log(1.0e7), len(tets)))
    target = vertices + rng.normal(0.0, 1.0e-3, vertices.shape)
    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=nx, dim_y=ny, dim_z=nz,
                          cell_x=edge, cell_y=edge, cell_z=edge, density=1000.0, k_mu=1.0, k_lambda=1.0, k_damp=0.0,
                          fix_left=True)
    model = builder.finalize("cpu")
    mu, lam = meshes.lame_from_young(young, 0.4)
    # The solver reads Newton's float32 material array.
    mu32 = mu.astype(np.float32).astype(np.float64)
    lam32 = lam.astype(np.float32).astype(np.float64)
    free = model.particle_inv_mass.numpy() > 0
    body = pd_oracle.Body.tet(model.tet_indices.numpy().reshape(-1, 4), model.tet_poses.numpy(), free, mu32, lam32,
                              1000.0)
    factor = factor_port.inverse_factor(sp.csr_matrix(body.matrix(5.0e-3)))
    q0 = model.particle_q.numpy().astype(np.float64)
    gravity = model.gravity.numpy()[0].astype(np.float64)
    return body, factor, q0, gravity, target.astype(np.float32), young


def main():
    from oracle.sparse_port import SparsePort

    dt, steps, rel, tol = 5.0e-3, 50, 1.0e-6, 1.0e-9
    start = time.time()
    body, factor, q0, gravity, target, young = workload()
    port = SparsePort(body, factor, dt, threads=8)
    print(f"setup {time.time() - start:.1f} s, nnz(S) {len(factor['s_values'])}", flush=True)
    q, v = q0.astype(np.float32).astype(np.float64), np.zeros_like(q0)
    inputs_q, inputs_qd, records, iterations = [], [], [], []
    for t in range(steps):
        inputs_q.append(q.astype(np.float32))
        inputs_qd.append(v.astype(np.float32))
        x, count, converged = port.step(q, v, np.zeros_like(q), gravity, max_iterations=10000, abs_tol=tol,
                                        rel_tol=rel)
        assert converged, t
        records.append(x)
        iterations.append(count)
        v = ((x - q) / dt).astype(np.float32).astype(np.float64)
        q = x.astype(np.float32).astype(np.float64)
        print(f"step {t} iterations {count} ({time.time() - start:.0f} s)", flush=True)
    final = q.astype(np.float32)
    diff = final.astype(np.float64) - target.astype(np.float64)
    loss = float((diff**2).sum())
    # Adjoint: the seed of the last step is dL/dq_50 = 2 (q_50 - target) in
    # float32, as the solver's float32 gradient arrays hold it.
    gq = (2.0 * (final - target)).astype(np.float64)
    gqd = np.zeros_like(gq)
    inertia = body.mass / dt**2
    grad_materials = np.zeros((len(body.elements), 2))
    seeds_q, seeds_qd = [None] * steps, [None] * steps
    backward_iterations = [0] * steps
    for t in reversed(range(steps)):
        seeds_q[t] = gq.astype(np.float32)
        seeds_qd[t] = gqd.astype(np.float32)
        mu_adj, material, count = port.backward_cg(records[t], gq, gqd, max_iterations=10000, abs_tol=tol,
                                                   rel_tol=rel, mode="exact")
        backward_iterations[t] = count
        grad_materials += material
        gq, gqd = inertia * mu_adj - gqd / dt, dt * inertia * mu_adj
        gq[~body.free] = 0.0
        gqd[~body.free] = 0.0
        print(f"backward {t} iterations {count} ({time.time() - start:.0f} s)", flush=True)
    dmu, dlam = 1.0 / (2.0 * 1.4), 0.4 / (1.4 * 0.2)
    grad_young = grad_materials[:, 0] * dmu + grad_materials[:, 1] * dlam
    keep = np.arange(0, steps, STRIDE)
    np.savez_compressed(
        HERE / "tet_block_rollout.npz",
        stride=STRIDE,
        steps=np.array(keep, dtype=np.int32),
        q_in=np.stack([inputs_q[t] for t in keep]),
        qd_in=np.stack([inputs_qd[t] for t in keep]),
        grad_q_out=np.stack([seeds_q[t] for t in keep]),
        grad_qd_out=np.stack([seeds_qd[t] for t in keep]),
        iterations=np.array(iterations, dtype=np.int32),
        backward_iterations=np.array(backward_iterations, dtype=np.int32),
        q_final=final,
        loss=loss,
        grad_young=grad_young,
        young=young,
    )
    print(f"done in {time.time() - start:.0f} s; loss {loss:.6e}")


if __name__ == "__main__":
    main()
