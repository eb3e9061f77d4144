"""Parity fixtures in the ``newton.diff_phd_parity.v1`` NPZ exchange format.

The reference's parity harness (``docs/validation.md``, "Parity fixture
schema") exchanges one NPZ per case: a Tet4 scene, its rollout inputs and a
linear objective on the final state, and the outputs of a run. ``run`` reads
such a fixture, rolls it out on this solver with the step adjoint, and
returns the outputs under the schema's names; ``save`` writes inputs and
outputs together so another implementation can compare.

Inputs (SI units, float64 unless noted): ``rest_vertices (N,3)``, ``tets
(E,4)`` int, ``density``, ``mu (E)``, ``lambda (E)``, ``material`` ("pd" or
"neo_hookean"), ``dirichlet (N)`` bool (pinned particles), ``q (N,3)``,
``v (N,3)``, ``f_ext (steps,N,3)``, ``gravity (3)``, ``dt``, ``max_iterations``,
``abs_tol``, ``rel_tol``; optional ``anderson_window``, ``muscle_directions
(E,3)``, ``muscle_stiffness (E)``, ``activations (steps,E)`` (contraction
``u = 1 - a``), ``contact_kind`` ("planar" / "spherical" / "mesh"),
``contact_parameters`` (planar ``(nx, ny, nz, offset)``, spherical ``(cx, cy,
cz, r)``, mesh ``(contact_radius, split_index)`` with ``contact_faces_left``
and ``contact_faces_right (F,3)``), ``contact_vertices``, ``friction``, ``restitution``,
``mesh_contact_parameters (5)`` (radius, kn_left, kn_right, kf, mu),
``mesh_contact_faces_a/_b (F,3)``; ``objective_q``, ``objective_v (N,3)``: the
loss is ``sum(objective_q * q_T + objective_v * v_T)``.

Outputs: ``q_next``, ``v_next (steps,N,3)``, ``iterations (steps)``,
``converged (steps)``, ``contact_multipliers (steps,K)``, ``planar_gaps
(steps,K)`` (planar boundaries), ``mesh_contact_pairs (steps)``, ``dL_dq``,
``dL_dv (N,3)`` (w.r.t. the initial state), ``dL_df_ext (steps,N,3)``,
``dL_dmu``, ``dL_dlambda (E)``, ``dL_dactivations (steps,E)`` when actuated.
Values pass through float32, as Newton's public states and materials do.
"""

from __future__ import annotations

import numpy as np
import torch

from .model import ModelBuilder
from .solver import SolverDiffPhD, Tape

SCHEMA = "newton.diff_phd_parity.v1"


def _f32(array):
    return np.asarray(array, dtype=np.float32).astype(np.float64)


def _scalar(fixture, key, default=None):
    if key not in fixture:
        return default
    value = np.asarray(fixture[key])
    return value.item() if value.ndim == 0 else value


def run(fixture, device="cuda") -> dict:
    """Roll out one parity fixture (a mapping of the schema's input arrays); returns the outputs."""
    if "schema" in fixture and str(_scalar(fixture, "schema")) != SCHEMA:
        raise ValueError(f"fixture schema must be {SCHEMA}")
    rest = _f32(fixture["rest_vertices"])
    tets = np.asarray(fixture["tets"], dtype=np.int32)
    pinned = np.asarray(fixture["dirichlet"], dtype=bool)
    f_ext = _f32(fixture["f_ext"])
    steps = f_ext.shape[0]
    builder = ModelBuilder(gravity=tuple(float(g) for g in _f32(fixture["gravity"])))
    for point, fixed in zip(rest, pinned):
        builder.add_particle(point, (0.0, 0.0, 0.0), 0.0 if fixed else 1.0)
    mu, lam = _f32(fixture["mu"]), _f32(fixture["lambda"])
    for tet, m, l in zip(tets, mu, lam):
        builder.add_tetrahedron(*map(int, tet), k_mu=float(m), k_lambda=float(l))
    model = builder.finalize(device, requires_grad=True)
    options = {
        "density": float(_scalar(fixture, "density")),
        "material": str(_scalar(fixture, "material", "pd")),
        "max_iterations": int(_scalar(fixture, "max_iterations")),
        "abs_tol": float(_scalar(fixture, "abs_tol")),
        "rel_tol": float(_scalar(fixture, "rel_tol")),
        "anderson_window": int(_scalar(fixture, "anderson_window", 5)),
    }
    if "muscle_directions" in fixture:
        options["muscle_directions"] = np.asarray(fixture["muscle_directions"], dtype=np.float64)
        options["muscle_stiffness"] = np.asarray(fixture["muscle_stiffness"], dtype=np.float64)
    kind = _scalar(fixture, "contact_kind")
    if kind is not None:
        kind = str(kind)
        if kind == "mesh":
            radius, split = np.asarray(fixture["contact_parameters"], dtype=np.float64)[:2]
            parameters = (float(radius), int(split), np.asarray(fixture["contact_faces_left"]),
                          np.asarray(fixture["contact_faces_right"]))
        else:
            parameters = tuple(np.asarray(fixture["contact_parameters"], dtype=np.float64))
        options["frictional_boundary"] = (kind, parameters)
        options["frictional_vertices"] = np.asarray(fixture["contact_vertices"], dtype=np.int32)
        options["friction"] = float(_scalar(fixture, "friction", 0.0))
        options["restitution"] = float(_scalar(fixture, "restitution", 0.0))
    if "mesh_contact_parameters" in fixture:
        options["mesh_contact"] = tuple(np.asarray(fixture["mesh_contact_parameters"], dtype=np.float64)) + (
            np.asarray(fixture["mesh_contact_faces_a"]), np.asarray(fixture["mesh_contact_faces_b"]))
    solver = SolverDiffPhD(model, **options)
    activations = None
    control = model.control()
    if "activations" in fixture:
        activations = [torch.tensor(np.asarray(a, dtype=np.float32), device=model.device) for a in
                       fixture["activations"]]
        for a in activations:
            a.grad = torch.zeros_like(a)
    states = [model.state(requires_grad=True) for _ in range(steps + 1)]
    with torch.no_grad():
        states[0].particle_q.copy_(torch.as_tensor(_f32(fixture["q"]), dtype=torch.float32))
        states[0].particle_qd.copy_(torch.as_tensor(_f32(fixture["v"]), dtype=torch.float32))
    model.tet_materials.grad = torch.zeros_like(model.tet_materials)
    out = {"schema": SCHEMA, "iterations": np.zeros(steps, np.int32), "converged": np.zeros(steps, bool)}
    multipliers, gaps, pairs = [], [], []
    with Tape() as tape:
        for t in range(steps):
            with torch.no_grad():
                states[t].particle_f.copy_(torch.as_tensor(f_ext[t], dtype=torch.float32))
            if activations is not None:
                control.tet_activations = activations[t]
            solver.step(states[t], states[t + 1], control if activations is not None else None, None,
                        float(_scalar(fixture, "dt")))
            out["iterations"][t] = int(solver.iterations[0])
            out["converged"][t] = (solver.read_status() & 1) == 0
            if solver.contact_multipliers is not None:
                multipliers.append(solver.contact_multipliers.cpu().numpy().copy())
                if kind == "planar":
                    normal = np.asarray(options["frictional_boundary"][1][:3])
                    x = solver._x.cpu().numpy()[options["frictional_vertices"]]
                    gaps.append(x @ (normal / np.linalg.norm(normal)) + options["frictional_boundary"][1][3]
                                / np.linalg.norm(normal))
            if solver.mesh_contact_pairs is not None:
                pairs.append(solver.mesh_contact_pairs)
    out["q_next"] = np.stack([s.particle_q.detach().double().cpu().numpy() for s in states[1:]])
    out["v_next"] = np.stack([s.particle_qd.detach().double().cpu().numpy() for s in states[1:]])
    if multipliers:
        out["contact_multipliers"] = np.stack(multipliers)
    if gaps:
        out["planar_gaps"] = np.stack(gaps)
    if pairs:
        out["mesh_contact_pairs"] = np.asarray(pairs, dtype=np.int32)
    objective_q = torch.as_tensor(np.asarray(fixture["objective_q"], dtype=np.float64), dtype=torch.float32,
                                  device=model.device)
    objective_v = torch.as_tensor(np.asarray(fixture["objective_v"], dtype=np.float64), dtype=torch.float32,
                                  device=model.device)
    tape.backward(grads={states[-1].particle_q: objective_q, states[-1].particle_qd: objective_v})
    out["dL_dq"] = states[0].particle_q.grad.double().cpu().numpy()
    out["dL_dv"] = states[0].particle_qd.grad.double().cpu().numpy()
    out["dL_df_ext"] = np.stack([s.particle_f.grad.double().cpu().numpy() for s in states[:-1]])
    out["dL_dmu"] = model.tet_materials.grad[:, 0].double().cpu().numpy()
    out["dL_dlambda"] = model.tet_materials.grad[:, 1].double().cpu().numpy()
    if activations is not None:
        out["dL_dactivations"] = np.stack([a.grad.double().cpu().numpy() for a in activations])
    out["status"] = np.int32(solver.read_status())
    return out


def save(path, fixture, outputs) -> None:
    """Write a fixture's inputs and a run's outputs to one ``.npz`` (inputs keep their names,
    outputs get the ``out__`` prefix)."""
    arrays = {k: np.asarray(v) for k, v in fixture.items()}
    arrays["schema"] = np.asarray(SCHEMA)
    arrays.update({f"out__{k}": np.asarray(v) for k, v in outputs.items()})
    np.savez_compressed(path, **arrays)


def load(path) -> tuple[dict, dict]:
    """``(inputs, outputs)`` of a file written by :func:`save`."""
    data = np.load(path, allow_pickle=False)
    inputs = {k: data[k] for k in data.files if not k.startswith("out__")}
    outputs = {k[5:]: data[k] for k in data.files if k.startswith("out__")}
    return inputs, outputs
