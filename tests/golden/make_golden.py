"""Generate the golden fixtures under tests/golden from the reference itself.

Run in a container that has the reference checkout (default
``/root/reference``; override with ``--reference``)::

    python tests/golden/make_golden.py

What runs, all from the reference tree, unmodified:

* ``tests/reference_oracle.py`` (NumPy only): ``ReferenceStep.step`` for Tet4
  forward iterates, ``reference_backward`` for the mean-weight adjoint.
* ``HexOracle`` from ``tests/test_diff_phd_hex.py:39-109``: that module imports
  Newton and Warp at the top, so only the class definition is extracted with
  ``ast`` and executed against ``ReferenceStep``.
* ``src/.../diff_phd/sparse.py`` host setup (``_validate_rows``,
  ``_nested_dissection``, ``_factor_ldlt``, ``_inverse_rows``, ``_csr``): the
  module imports Warp for its device kernels, which never run here, so a
  minimal import stub stands in for ``warp``.

The meshes are this package's own grids (``newton_solver_diff_phd_b200.meshes``);
the reference's Tet4 grids come from Newton, which is not part of the
reference tree.
"""

from __future__ import annotations

import argparse
import ast
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from newton_solver_diff_phd_b200 import meshes  # noqa: E402


class _Anything:
    """Subscriptable, callable, attribute-rich placeholder for Warp types."""

    def __getattr__(self, name):
        return _Anything()

    def __getitem__(self, item):
        return _Anything()

    def __call__(self, *args, **kwargs):
        if len(args) == 1 and callable(args[0]) and not kwargs:
            return args[0]
        return _Anything()

    def __or__(self, other):
        return self

    __ror__ = __or__


def _warp_stub():
    module = types.ModuleType("warp")

    def kernel(*args, **kwargs):
        if args and callable(args[0]):
            return args[0]
        return lambda function: function

    module.kernel = kernel
    module.func = lambda function: function
    module.constant = lambda value: value
    module.__getattr__ = lambda name: _Anything()
    return module


def load_reference(root: Path):
    sys.modules.setdefault("warp", _warp_stub())
    sys.path.insert(0, str(root / "src"))
    sys.path.insert(0, str(root))
    import importlib.util

    def load(name, path):
        spec = importlib.util.spec_from_file_location(name, path)
        module = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(module)
        return module

    oracle = load("ref_oracle", root / "tests" / "reference_oracle.py")
    sparse = load("ref_sparse", root / "src/newton_solver_diff_phd/_src/solvers/diff_phd/sparse.py")
    source = (root / "tests" / "test_diff_phd_hex.py").read_text()
    tree = ast.parse(source)
    node = next(n for n in tree.body if isinstance(n, ast.ClassDef) and n.name == "HexOracle")
    namespace = {"np": np, "ReferenceStep": oracle.ReferenceStep}
    namespace.update({k: getattr(oracle, k) for k in dir(oracle) if not k.startswith("__")})
    exec(compile(ast.Module(body=[node], type_ignores=[]), "HexOracle", "exec"), namespace)
    return oracle, sparse, namespace["HexOracle"]


def sparse_factor(sparse, rows):
    """Run the reference setup and return its arrays (CSR of S and S^T, permutation)."""
    rows = sparse._validate_rows(rows)
    adjacency = [set(row) - {i} for i, row in enumerate(rows)]
    permutation = sparse._nested_dissection(adjacency)
    lower, diagonal = sparse._factor_ldlt(rows, permutation)
    inverse_rows = sparse._inverse_rows(lower, diagonal, permutation)
    transpose = [{} for _ in rows]
    for row, entries in enumerate(inverse_rows):
        for column, value in entries.items():
            transpose[column][row] = value
    s = sparse._csr(inverse_rows)
    st = sparse._csr(transpose)
    return {
        "permutation": permutation.astype(np.int32),
        "diagonal": diagonal,
        "s_offsets": s[0],
        "s_columns": s[1],
        "s_values": s[2],
        "st_offsets": st[0],
        "st_columns": st[1],
        "st_values": st[2],
    }


def dense_to_rows(matrix):
    return [{int(j): float(row[j]) for j in np.flatnonzero(row)} for row in matrix]


def tet_fixture_model(contrast=1.0):
    """3x2x2 Tet4 block of 0.1 m cubes at z=1, x=0 face pinned (the reference ``_grid``)."""
    vertices, tets, _ = meshes.tet_grid(3, 2, 2, 0.1, origin=(0.0, 0.0, 1.0))
    poses = meshes.tet_rest_poses(vertices, tets)
    mu = np.full(len(tets), 2.0e4)
    lame = np.full(len(tets), 5.0e4)
    if contrast != 1.0:
        stiff = vertices[tets].mean(axis=1)[:, 0] > vertices[:, 0].mean()
        mu[stiff] *= contrast
        lame[stiff] *= contrast
    # Newton stores materials as float32; the reference widens them to float64.
    mu = mu.astype(np.float32).astype(np.float64)
    lame = lame.astype(np.float32).astype(np.float64)
    free = vertices[:, 0] > 0.0
    return vertices, tets, poses, mu, lame, free


def deformed_state(vertices, free, seed=3, stretch=(1.3, 0.8, 1.1), speed=0.5):
    """The reference ``_deformed_state`` (``tests/test_diff_phd_solver.py:109-120``), float32-rounded."""
    rng = np.random.default_rng(seed)
    q = vertices.astype(np.float32).astype(np.float64)
    center = q.mean(axis=0)
    deformed = np.where(free[:, None], center + (q - center) * np.asarray(stretch), q)
    deformed[free] += 0.01 * rng.standard_normal((free.sum(), 3))
    velocity = np.where(free[:, None], speed * rng.standard_normal(q.shape), 0.0)
    return deformed.astype(np.float32).astype(np.float64), velocity.astype(np.float32).astype(np.float64)


def tet_matrix(oracle, vertices, tets, poses, mu, lame, free, material, dt, muscles=None):
    step = oracle.ReferenceStep(tets, poses, mu, lame, 1000.0, free, material, **(muscles or {}))
    return step, step.matrix(dt)


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default="/root/reference")
    parser.add_argument("--only", choices=("frictional_contact", "woodbury"), default=None,
                        help="regenerate one fixture file and leave the others untouched")
    args = parser.parse_args()
    oracle, sparse, hex_oracle = load_reference(Path(args.reference))
    if args.only == "frictional_contact":
        np.savez_compressed(HERE / "frictional_contact.npz", **frictional_contact_fixture(oracle))
        return
    if args.only == "woodbury":
        np.savez_compressed(HERE / "woodbury.npz", **woodbury_fixture(oracle))
        return

    # --- Sparse inverse factors (sparse.py host setup) ------------------------
    factors = {}
    cancel = np.asarray(((2.0, 2.0, 2.0), (2.0, 5.0, 5.0), (2.0, 5.0, 10.0)))
    factors["cancel"] = (cancel, sparse_factor(sparse, dense_to_rows(cancel)))
    nx, ny = 8, 7
    size = nx * ny + 3
    rng = np.random.default_rng(519)
    grid = np.eye(size)
    for y in range(ny):
        for x in range(nx):
            i = y * nx + x
            for j in ([i + 1] if x + 1 < nx else []) + ([i + nx] if y + 1 < ny else []):
                weight = rng.uniform(0.1, 5.0)
                grid[i, i] += weight
                grid[j, j] += weight
                grid[i, j] = grid[j, i] = -weight
    factors["grid2d"] = (grid, sparse_factor(sparse, dense_to_rows(grid)))
    vertices, tets, poses, mu, lame, free = tet_fixture_model()
    _, a_tet = tet_matrix(oracle, vertices, tets, poses, mu, lame, free, "pd", 0.004)
    factors["tet322"] = (a_tet, sparse_factor(sparse, dense_to_rows(a_tet)))
    # A Hex8 grid large enough for nested-dissection separators (> 24 vertices per part).
    hv, hh, _ = meshes.hex_grid(6, 3, 2, 0.1)
    hmat = np.column_stack((np.full(len(hh), 2.0e4), np.full(len(hh), 5.0e4)))
    hfree = hv[:, 0] > 0.0
    hoo = hex_oracle(meshes.Mesh("grid", hv, hh), hmat, hfree, "pd")
    a_hex = hoo.matrix(0.01)
    # HexOracle integrates with its own Jacobians; round-trip through the rows
    # representation, which needs exact symmetry.
    a_hex = 0.5 * (a_hex + a_hex.T)
    factors["hex632"] = (a_hex, sparse_factor(sparse, dense_to_rows(a_hex)))
    out = {}
    for name, (matrix, arrays) in factors.items():
        out[f"{name}__matrix"] = matrix
        for key, value in arrays.items():
            out[f"{name}__{key}"] = value
    np.savez_compressed(HERE / "sparse_factors.npz", **out)

    # --- Tet4 forward iterates (ReferenceStep) ---------------------------------
    forward = {}
    dt = 0.004
    for contrast in (1.0, 10.0, 100.0):
        vertices, tets, poses, mu, lame, free = tet_fixture_model(contrast)
        q, v = deformed_state(vertices, free)
        gravity = np.array([0.0, 0.0, -9.81], dtype=np.float32).astype(np.float64)
        for material in ("pd", "neo_hookean"):
            runs = [("fixed", {"max_iterations": 12, "abs_tol": 0.0, "rel_tol": 0.0})] if contrast == 1.0 else []
            runs.append(("converged", {"max_iterations": 500, "abs_tol": 1.0e-11, "rel_tol": 1.0e-10}))
            for label, options in runs:
                step = oracle.ReferenceStep(tets, poses, mu, lame, 1000.0, free, material)
                x, iterations, converged = step.step(q, v, np.zeros_like(q), gravity, dt, **options)
                key = f"c{int(contrast)}_{material}_{label}"
                forward[f"{key}__x"] = x
                forward[f"{key}__iterations"] = np.int32(iterations)
                forward[f"{key}__converged"] = np.int32(converged)
                forward[f"{key}__options"] = np.array(
                    [options["max_iterations"], options["abs_tol"], options["rel_tol"]]
                )
        forward[f"c{int(contrast)}__q"] = q
        forward[f"c{int(contrast)}__v"] = v
        forward[f"c{int(contrast)}__mu"] = mu
        forward[f"c{int(contrast)}__lame"] = lame
    # Muscle fibres (tests/test_diff_phd_solver.py:281-307).
    vertices, tets, poses, mu, lame, free = tet_fixture_model()
    rng = np.random.default_rng(5)
    directions = rng.standard_normal((len(tets), 3))
    stiffness = np.where(np.arange(len(tets)) % 2 == 0, 4.0e4, 0.0)
    contraction = np.where(stiffness > 0, 0.25, 0.0).astype(np.float32)
    q, v = deformed_state(vertices, free, speed=0.0)
    step = oracle.ReferenceStep(
        tets, poses, mu, lame, 1000.0, free, "pd", muscle_directions=directions, muscle_stiffness=stiffness
    )
    options = {"max_iterations": 500, "abs_tol": 1.0e-11, "rel_tol": 1.0e-10}
    x, iterations, converged = step.step(
        q,
        v,
        np.zeros_like(q),
        np.array([0.0, 0.0, -9.81]),
        dt,
        targets=1.0 - contraction.astype(np.float64),
        **options,
    )
    forward.update(
        {
            "muscle__q": q,
            "muscle__v": v,
            "muscle__directions": directions,
            "muscle__stiffness": stiffness,
            "muscle__contraction": contraction,
            "muscle__x": x,
            "muscle__iterations": np.int32(iterations),
            "muscle__converged": np.int32(converged),
        }
    )
    np.savez_compressed(HERE / "tet_forward.npz", **forward)

    # --- Hex8 forward (HexOracle, tests/test_diff_phd_hex.py:133-198) ----------
    hexes = {}
    vertices = np.array([[x, y, z] for x in range(3) for y in range(2) for z in range(2)], dtype=float) * 0.1
    elements = np.array([np.arange(8), np.arange(4, 12)], dtype=np.int32)
    mesh = meshes.Mesh("two-cubes", vertices, elements)
    free = np.arange(12) >= 4
    materials = np.array([[2000.0, 4000.0], [20000.0, 40000.0]])
    directions = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    stiffness = np.array([1000.0, 300.0])
    targets = np.array([0.0, 0.8])
    planes = (np.array([0, 8, 9]), 120.0, (0.0, 0.0, 2.0, -0.08))
    q = vertices.copy()
    q[4:, 0] *= 1.04
    q[4:, 2] += 0.01 * q[4:, 0]
    q = q.astype(np.float32).astype(np.float64)
    velocity = np.random.default_rng(4).normal(0, 0.03, q.shape)
    velocity[:4] = 0
    velocity = velocity.astype(np.float32).astype(np.float64)
    force = np.random.default_rng(5).normal(0, 0.2, q.shape).astype(np.float32).astype(np.float64)
    for material in ("pd", "neo_hookean"):
        hoo = hex_oracle(mesh, materials, free, material, (directions, stiffness), planes)
        x, iterations, converged = hoo.step(
            q, velocity, force, np.zeros(3), 0.003, max_iterations=1000, abs_tol=1e-12, rel_tol=1e-10, window=0,
            targets=targets,
        )
        hexes[f"{material}__x"] = x
        hexes[f"{material}__iterations"] = np.int32(iterations)
        hexes[f"{material}__converged"] = np.int32(converged)
        hexes[f"{material}__inverse"] = np.linalg.inv(hoo.matrix(0.003))
    hexes.update({"q": q, "v": velocity, "f": force, "materials": materials, "vertices": vertices})
    np.savez_compressed(HERE / "hex_forward.npz", **hexes)

    # --- Tet4 adjoint (reference_backward, mean-weight K) ----------------------
    backward = {}
    for contrast, material in ((2.0, "pd"), (1.0, "pd"), (1.0, "neo_hookean")):
        vertices, tets, poses, mu, lame, free = tet_fixture_model(contrast)
        q, v = deformed_state(vertices, free, stretch=(1.2, 0.85, 1.05), speed=0.3)
        step = oracle.ReferenceStep(tets, poses, mu, lame, 1000.0, free, material)
        options = {"max_iterations": 3000, "abs_tol": 1.0e-12, "rel_tol": 1.0e-12}
        x, iterations, converged = step.step(q, v, np.zeros_like(q), np.array([0.0, 0.0, -9.81]), dt, **options)
        rng = np.random.default_rng(49)
        gq = rng.standard_normal(q.shape).astype(np.float32).astype(np.float64)
        gv = (0.01 * rng.standard_normal(q.shape)).astype(np.float32).astype(np.float64)
        result = oracle.reference_backward(step, x, dt, gq, gv)
        key = f"c{int(contrast)}_{material}"
        backward[f"{key}__q"] = q
        backward[f"{key}__v"] = v
        backward[f"{key}__mu_lame"] = np.column_stack((mu, lame))
        backward[f"{key}__x"] = x
        backward[f"{key}__gq"] = gq
        backward[f"{key}__gv"] = gv
        for name, value in result.items():
            backward[f"{key}__out_{name}"] = value
    np.savez_compressed(HERE / "tet_backward.npz", **backward)
    np.savez_compressed(HERE / "mesh_contact.npz", **mesh_contact_fixture(oracle))
    np.savez_compressed(HERE / "frictional_contact.npz", **frictional_contact_fixture(oracle))
    np.savez_compressed(HERE / "woodbury.npz", **woodbury_fixture(oracle))
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


_TET_FACES = np.array(((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)))


def two_bodies(gap):
    """A 3x2x2 grid of 0.1 m cubes (bottom pinned) and one tetrahedron whose apex
    reaches ``gap`` above the grid top (the reference test's two-body scene)."""
    vertices, tets, _ = meshes.tet_grid(3, 2, 2, 0.1)
    grid = len(vertices)
    extra = np.array(((0.13, 0.11, 0.2 + gap), (0.33, 0.07, 0.5), (0.05, 0.18, 0.5), (0.17, 0.02, 0.55)))
    vertices = np.vstack((vertices, extra))
    tets = np.vstack((tets, np.arange(grid, grid + 4)[None]))
    faces = tets[:, _TET_FACES].reshape(-1, 3)
    _, first, counts = np.unique(np.sort(faces, axis=1), axis=0, return_index=True, return_counts=True)
    faces = faces[first[counts == 1]]
    faces_a = faces[np.all(faces < grid, axis=1)]
    faces_b = faces[np.all(faces >= grid, axis=1)]
    return vertices, tets, faces_a, faces_b


def mesh_contact_fixture(oracle):
    """``mesh_contact_force`` of the reference transcription on perturbed two-body states."""
    out = {}
    rng = np.random.default_rng(7)
    vertices, tets, faces_a, faces_b = two_bodies(-0.004)
    options = (0.02, 5.0e3, 5.0e4, 50.0, 0.5)
    out["vertices"], out["tets"], out["faces_a"], out["faces_b"] = vertices, tets, faces_a, faces_b
    out["options"] = np.array(options)
    for trial in range(4):
        q = vertices + 0.012 * rng.standard_normal(vertices.shape) * (trial > 0)
        v = rng.standard_normal(vertices.shape)
        out[f"t{trial}__q"], out[f"t{trial}__v"] = q, v
        out[f"t{trial}__force"] = oracle.mesh_contact_force(q, v, faces_a, faces_b, *options)
    return out


# Options of the reference contact tests (tests/test_diff_phd_contact.py:16-18).
CONTACT_TIGHT = {"max_iterations": 2000, "abs_tol": 1.0e-12, "rel_tol": 1.0e-11}
CONTACT_REFERENCE = {"max_iterations": 2000, "abs_tol": 1.0e-9, "rel_tol": 1.0e-6}


def surface_faces(tets):
    """Faces of exactly one tetrahedron, in first-occurrence orientation (tests/test_diff_phd_mesh_boundary.py:22-25)."""
    faces = np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]], tets[:, [1, 2, 3]]])
    _unique, index, counts = np.unique(np.sort(faces, axis=1), axis=0, return_index=True, return_counts=True)
    return faces[np.sort(index[counts == 1])]


def contact_rollout(oracle, step, contact, q, v, gravity, dt, steps, options, registered=None):
    """Step the reference oracle with its contact and chain the float32 states as the solver writes them."""
    out = {}
    for t in range(steps):
        x, iterations, converged = step.step(q, v, np.zeros_like(q), gravity, dt, contact=contact, **options)
        out[f"s{t}__q"], out[f"s{t}__v"], out[f"s{t}__x"] = q, v, x
        out[f"s{t}__iterations"] = np.int32(iterations)
        out[f"s{t}__converged"] = np.int32(converged)
        if registered is None:
            out[f"s{t}__multiplier"] = contact.multiplier.copy()
        else:
            out[f"s{t}__multiplier"] = contact.registered_multiplier()
            out[f"s{t}__candidate"] = np.isin(registered, contact.nodes).astype(np.int32)
        # write_state: q+ = x, v+ = (x - q) / h, stored as float32.
        q, v = x.astype(np.float32).astype(np.float64), ((x - q) / dt).astype(np.float32).astype(np.float64)
    return out


def frictional_contact_fixture(oracle):
    """``ReferenceContact`` / ``ReferenceMeshContact`` rollouts of the reference contact tests
    (tests/test_diff_phd_contact.py:40-142, tests/test_diff_phd_mesh_boundary.py:28-135)."""
    out = {}
    dt = 0.004
    gravity = np.array([0.0, 0.0, -9.81], dtype=np.float32).astype(np.float64)
    vertices, tets, _ = meshes.tet_grid(3, 2, 2, 0.1, origin=(0.0, 0.0, 1.0))
    # Newton keeps rest poses in float32.
    poses = meshes.tet_rest_poses(vertices, tets).astype(np.float32).astype(np.float64)
    mu = np.full(len(tets), 2.0e4, dtype=np.float32).astype(np.float64)
    lame = np.full(len(tets), 5.0e4, dtype=np.float32).astype(np.float64)
    free = np.ones(len(vertices), dtype=bool)
    nodes = np.unique(surface_faces(tets))
    center = vertices.astype(np.float32).astype(np.float64).mean(axis=0)
    sphere = ("spherical", (center[0], center[1], -0.25, 0.25))
    plane = ("planar", (0.0, 0.0, 1.0, 0.0))
    cases = {
        "plane": (plane, 0.0, 0.0, 0.001, (0.0, 0.0, -1.0), 3, CONTACT_TIGHT),
        "stick": (plane, 2.0, 0.0, 0.001, (0.05, 0.0, -1.0), 3, CONTACT_TIGHT),
        "slide": (plane, 0.1, 0.0, 0.001, (2.0, 0.0, -1.0), 3, CONTACT_TIGHT),
        "sphere": (sphere, 0.4, 0.0, 0.0005, (0.0, 0.0, -1.0), 3, CONTACT_REFERENCE),
        "chatter": (sphere, 0.4, 0.0, 0.0005, (0.0, 0.0, -1.0), 2, CONTACT_TIGHT),
        "restitution": (plane, 0.0, 0.5, 0.001, (0.0, 0.0, -1.0), 2, CONTACT_TIGHT),
    }
    out["grid__nodes"] = nodes
    for name, (boundary, friction, restitution, height, velocity, steps, options) in cases.items():
        q = vertices.astype(np.float32).astype(np.float64)
        q[:, 2] += height - q[:, 2].min()
        q = q.astype(np.float32).astype(np.float64)
        v = np.tile(np.asarray(velocity, dtype=np.float32), (len(q), 1)).astype(np.float64)
        step = oracle.ReferenceStep(tets, poses, mu, lame, 1000.0, free, "pd")
        contact = oracle.ReferenceContact(*boundary, nodes, friction=friction, restitution=restitution)
        out[f"{name}__parameters"] = np.asarray(boundary[1], dtype=np.float64)
        out[f"{name}__options"] = np.array([options["max_iterations"], options["abs_tol"], options["rel_tol"],
                                            friction, restitution])
        for key, value in contact_rollout(oracle, step, contact, q, v, gravity, dt, steps, options).items():
            out[f"{name}__{key}"] = value
    # Two soft blocks (tests/test_diff_phd_mesh_boundary.py:28-40): a free 2x1x1 block
    # above a 3x2x2 block with a pinned bottom, offset half a cell in x.
    radius = 0.01
    upper, upper_tets, _ = meshes.tet_grid(2, 1, 1, 0.1, origin=(0.05, 0.0, 0.2 + radius + 0.002))
    lower, lower_tets, _ = meshes.tet_grid(3, 2, 2, 0.1)
    split = len(upper)
    vertices = np.vstack((upper, lower))
    tets = np.vstack((upper_tets, lower_tets + split))
    poses = meshes.tet_rest_poses(vertices, tets).astype(np.float32).astype(np.float64)
    mu = np.full(len(tets), 2.0e4, dtype=np.float32).astype(np.float64)
    lame = np.full(len(tets), 5.0e4, dtype=np.float32).astype(np.float64)
    free = np.ones(len(vertices), dtype=bool)
    free[split:] = lower[:, 2] > 0.0
    faces_left, faces_right = surface_faces(upper_tets), surface_faces(lower_tets) + split
    out.update({"blocks__vertices": vertices, "blocks__tets": tets, "blocks__split": np.int32(split),
                "blocks__faces_left": faces_left, "blocks__faces_right": faces_right, "blocks__free": free})
    registered = np.unique(np.concatenate([faces_left, faces_right]))
    registered = registered[free[registered]]
    mesh_cases = {
        "mesh": (registered[registered < split], 0.0, 0.0, (0.0, 0.0, -1.0), 4, CONTACT_TIGHT),
        "mesh_stick": (registered[registered < split], 2.0, 0.0, (0.5, 0.0, -1.0), 4, CONTACT_REFERENCE),
        "mesh_restitution": (registered[registered < split], 0.0, 0.5, (0.0, 0.0, -1.0), 4, CONTACT_TIGHT),
        "mesh_two_sided": (registered, 0.0, 0.0, (0.0, 0.0, -1.0), 3, CONTACT_REFERENCE),
    }
    for name, (nodes, friction, restitution, velocity, steps, options) in mesh_cases.items():
        q = vertices.astype(np.float32).astype(np.float64)
        v = np.zeros_like(q)
        v[:split] = np.asarray(velocity, dtype=np.float32)
        step = oracle.ReferenceStep(tets, poses, mu, lame, 1000.0, free, "pd")
        contact = oracle.ReferenceMeshContact(radius, split, faces_left, faces_right, nodes, friction, restitution)
        out[f"{name}__nodes"] = nodes
        out[f"{name}__options"] = np.array([options["max_iterations"], options["abs_tol"], options["rel_tol"],
                                            friction, restitution, radius])
        for key, value in contact_rollout(oracle, step, contact, q, v, gravity, dt, steps, options, nodes).items():
            out[f"{name}__{key}"] = value
    return out


def woodbury_fixture(oracle):
    """``reference_backward`` with the contact projection after a frictional rollout with fibres
    (tests/test_diff_phd_adjoint.py:339-416): the grid on a plane, lifted 1 mm, moving at
    (0.3, 0, -1) m/s; two steps, then the recorded third step and its backward pass."""

    class RecordingContact(oracle.ReferenceContact):
        """ReferenceContact that also keeps the last iteration's omega (the StepRecord snapshot)."""

        def iterate(self, x, b_full, q):
            delta = self.gaps(x)
            s = np.maximum(np.sqrt(delta**2 + self.r**2 * self.multiplier**2), 1.0e-14)
            self.omega = 1.0 - delta / s
            return super().iterate(x, b_full, q)

    out = {}
    dt = 0.004
    gravity = np.array([0.0, 0.0, -9.81], dtype=np.float32).astype(np.float64)
    vertices, tets, _ = meshes.tet_grid(3, 2, 2, 0.1, origin=(0.0, 0.0, 1.0))
    poses = meshes.tet_rest_poses(vertices, tets).astype(np.float32).astype(np.float64)
    mu = np.full(len(tets), 2.0e4, dtype=np.float32).astype(np.float64)
    lame = np.full(len(tets), 5.0e4, dtype=np.float32).astype(np.float64)
    free = np.ones(len(vertices), dtype=bool)
    nodes = np.unique(surface_faces(tets))
    for friction in (0.0, 0.5):
        key = f"f{int(10 * friction)}"
        rng = np.random.default_rng(31)
        directions = rng.standard_normal((len(tets), 3))
        stiffness = np.full(len(tets), 4.0e4)
        contraction = rng.uniform(0.0, 0.3, len(tets)).astype(np.float32)
        targets = 1.0 - contraction.astype(np.float64)
        step = oracle.ReferenceStep(tets, poses, mu, lame, 1000.0, free, "pd", muscle_directions=directions,
                                    muscle_stiffness=stiffness)
        contact = RecordingContact("planar", (0.0, 0.0, 1.0, 0.0), nodes, friction=friction)
        q = vertices.astype(np.float32).astype(np.float64)
        q[:, 2] += 0.001 - q[:, 2].min()
        q = q.astype(np.float32).astype(np.float64)
        v = np.tile(np.array([0.3, 0.0, -1.0], dtype=np.float32), (len(q), 1)).astype(np.float64)
        for t in range(3):
            x, _iterations, converged = step.step(q, v, np.zeros_like(q), gravity, dt, contact=contact,
                                                   targets=targets, **CONTACT_TIGHT)
            assert converged
            if t < 2:
                q, v = x.astype(np.float32).astype(np.float64), ((x - q) / dt).astype(np.float32).astype(np.float64)
        q_weight = rng.standard_normal((len(q), 3)).astype(np.float32).astype(np.float64)
        qd_weight = (0.01 * rng.standard_normal((len(q), 3))).astype(np.float32).astype(np.float64)
        snapshot = (nodes, contact.multiplier.copy(), contact.omega.copy(), contact.normals.copy(), friction)
        result = oracle.reference_backward(step, x, dt, q_weight, qd_weight, contact=snapshot, targets=targets)
        out.update({f"{key}__q": q, f"{key}__v": v, f"{key}__x": x, f"{key}__gq": q_weight, f"{key}__gv": qd_weight,
                    f"{key}__directions": directions, f"{key}__contraction": contraction,
                    f"{key}__multiplier": snapshot[1], f"{key}__omega": snapshot[2], f"{key}__normal": snapshot[3]})
        for name, value in result.items():
            out[f"{key}__out_{name}"] = value
    out["nodes"] = nodes
    return out


if __name__ == "__main__":
    main()
