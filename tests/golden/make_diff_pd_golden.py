"""Generate ``tests/golden/diff_pd.npz`` from the reference's own DiffPD oracle.

Runs ``tests/reference_oracle_diff_pd.py`` of the reference checkout (NumPy
only; default ``/root/reference``, override with ``--reference``) on the
scenes of the reference's ``tests/test_diff_pd_solver.py``: a 3 x 2 x 2 block
of 0.1 m cubes in five tetrahedra each (this package's grid; the reference
takes its tetrahedra from Newton), corotated weight 4e4, volume weight 5e4,
density 1000, gravity -9.81, dt 0.01. For every step the fixture holds the
float32 input state, the external force, the oracle's float64 output
positions and velocities, its iteration count, line-search halvings and
gradient fallbacks.

    python tests/golden/make_diff_pd_golden.py
"""

from __future__ import annotations

import argparse
import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

DENSITY, COROTATED, VOLUME, DT = 1000.0, 4.0e4, 5.0e4, 1.0e-2
GRAVITY = (0.0, 0.0, -9.81)
ARC_START = (np.sin(np.radians(30.0)), 0.0, -np.cos(np.radians(30.0)))
SCENES = {
    # name: (grid origin, fix_left, state_forces, perturbation, steps, dt, external force seed)
    "free_fall": ((0.0, 0.0, 1.0), False, [], dict(stretch=(1.3, 0.8, 1.1), speed=0.5), 4, DT, None),
    "pinned": ((0.0, 0.0, 1.0), True, [], None, 6, DT, None),
    "planar": ((-0.15, -0.1, -0.005), False, [("planar_contact", [0.0, 0.0, 2.0, 0.0, 3, 1.0e6, 1.0, 0.1])],
               dict(velocity=(1.0, 0.0, -0.5)), 5, DT, None),
    "arc": ((-0.15, -0.1, -0.005), False,
            [("arc_contact", [0.0, 0.0, 1.0, 0.0, 2.0, 0.0, *ARC_START, 1.0, np.radians(32.0), 3, 1.0e6, 1.0, 0.1])],
            dict(velocity=(1.0, 0.0, -0.5)), 5, DT, None),
    "history": ((0.0, 0.0, 1.0), False, [], dict(noise=0.03, speed=5.0, seed=3), 1, 0.2, None),
    "external": ((0.0, 0.0, 1.0), False, [], dict(), 1, DT, 5),
}


def grid(origin, fix_left):
    from newton_solver_diff_phd_b200 import ModelBuilder

    builder = ModelBuilder(gravity=GRAVITY)
    builder.add_soft_grid(pos=origin, rot=None, vel=(0.0, 0.0, 0.0), dim_x=3, dim_y=2, dim_z=2, cell_x=0.1,
                          cell_y=0.1, cell_z=0.1, density=DENSITY, k_mu=2.0e4, k_lambda=5.0e4, k_damp=0.0,
                          fix_left=fix_left)
    return builder.finalize("cpu")


def perturb(q, free, velocity=(0.0, 0.0, 0.0), noise=0.003, speed=0.1, stretch=(1.0, 1.0, 1.0), seed=0):
    """The reference tests' ``_perturb``: float32 states."""
    rng = np.random.default_rng(seed)
    center = q.mean(axis=0)
    deformed = center + (q - center) * np.asarray(stretch) + noise * rng.standard_normal(q.shape)
    v = np.asarray(velocity) + speed * rng.standard_normal(q.shape)
    return (np.where(free[:, None], deformed, q).astype(np.float32),
            np.where(free[:, None], v, 0.0).astype(np.float32))


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", type=Path, default=Path("/root/reference"))
    args = parser.parse_args()
    spec = importlib.util.spec_from_file_location("reference_oracle_diff_pd",
                                                  args.reference / "tests" / "reference_oracle_diff_pd.py")
    oracle_module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(oracle_module)
    out = {}
    for name, (origin, fix_left, forces, perturbation, steps, dt, force_seed) in SCENES.items():
        model = grid(origin, fix_left)
        rest = model.particle_q.numpy()
        tets = model.tet_indices.numpy().reshape(-1, 4)
        free = model.particle_inv_mass.numpy() > 0
        oracle = oracle_module.ReferenceStep(rest, tets, DENSITY, COROTATED, VOLUME, free, GRAVITY, forces)
        if perturbation is None:
            q, v = rest.astype(np.float32), np.zeros_like(rest, dtype=np.float32)
        else:
            q, v = perturb(rest.astype(np.float64), free, **perturbation)
        f = np.zeros_like(q)
        if force_seed is not None:
            f = np.random.default_rng(force_seed).standard_normal(q.shape).astype(np.float32)
        record = {k: [] for k in ("q_in", "v_in", "f", "q_out", "v_out", "iterations", "halvings", "fallbacks")}
        for _ in range(steps):
            x, velocity, iterations = oracle.step(q.astype(np.float64), v.astype(np.float64), f.astype(np.float64),
                                                  dt)
            for key, value in (("q_in", q), ("v_in", v), ("f", f), ("q_out", x), ("v_out", velocity),
                               ("iterations", iterations), ("halvings", oracle.halvings),
                               ("fallbacks", oracle.fallbacks)):
                record[key].append(value)
            q, v = x.astype(np.float32), velocity.astype(np.float32)
            f = np.zeros_like(f)
        for key, values in record.items():
            out[f"{name}__{key}"] = np.asarray(values)
        out[f"{name}__dt"] = np.float64(dt)
        out[f"{name}__rest"] = rest
        out[f"{name}__tets"] = tets
        out[f"{name}__free"] = free
        print(name, "iterations", record["iterations"], "halvings", record["halvings"])
    np.savez_compressed(HERE / "diff_pd.npz", **out)


if __name__ == "__main__":
    main()
