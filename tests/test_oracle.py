"""The oracle restatement against the reference's own outputs (tests/golden)."""

import numpy as np
import pytest

from newton_solver_diff_phd_b200 import meshes
from oracle import pd_oracle
from tests.helpers import golden


def _tet_fixture():
    vertices, tets, _ = meshes.tet_grid(3, 2, 2, 0.1, origin=(0.0, 0.0, 1.0))
    return vertices, tets, meshes.tet_rest_poses(vertices, tets), vertices[:, 0] > 0


GRAVITY = np.array([0.0, 0.0, -9.81], dtype=np.float32).astype(np.float64)


@pytest.mark.parametrize("contrast,material,label", [
    (1.0, "pd", "fixed"), (1.0, "pd", "converged"), (1.0, "neo_hookean", "fixed"), (1.0, "neo_hookean", "converged"),
    (10.0, "pd", "converged"), (10.0, "neo_hookean", "converged"), (100.0, "pd", "converged"),
    (100.0, "neo_hookean", "converged"),
])
def test_tet_forward_matches_reference_oracle(contrast, material, label):
    g = golden("tet_forward.npz")
    vertices, tets, poses, free = _tet_fixture()
    c = f"c{int(contrast)}"
    key = f"{c}_{material}_{label}"
    options = g[key + "__options"]
    body = pd_oracle.Body.tet(tets, poses, free, g[c + "__mu"], g[c + "__lame"], 1000.0, material=material)
    x, iterations, converged = pd_oracle.step(
        body, g[c + "__q"], g[c + "__v"], np.zeros((len(vertices), 3)), GRAVITY, 0.004,
        max_iterations=int(options[0]), abs_tol=float(options[1]), rel_tol=float(options[2]),
    )
    reference = g[key + "__x"]
    np.testing.assert_allclose(x, reference, rtol=0.0, atol=1.0e-10 * np.abs(reference).max())
    assert iterations == int(g[key + "__iterations"])
    assert converged == bool(g[key + "__converged"])


def test_tet_muscle_forward_matches_reference_oracle():
    g = golden("tet_forward.npz")
    vertices, tets, poses, free = _tet_fixture()
    body = pd_oracle.Body.tet(
        tets, poses, free, g["c1__mu"], g["c1__lame"], 1000.0,
        muscle_directions=g["muscle__directions"], muscle_stiffness=g["muscle__stiffness"],
    )
    x, _, converged = pd_oracle.step(
        body, g["muscle__q"], g["muscle__v"], np.zeros((len(vertices), 3)), [0.0, 0.0, -9.81], 0.004,
        max_iterations=500, abs_tol=1e-11, rel_tol=1e-10, targets=1.0 - g["muscle__contraction"].astype(np.float64),
    )
    assert converged
    np.testing.assert_allclose(x, g["muscle__x"], rtol=0.0, atol=1e-10 * np.abs(g["muscle__x"]).max())


@pytest.mark.parametrize("material", ["pd", "neo_hookean"])
def test_hex_forward_matches_reference_hex_oracle(material):
    h = golden("hex_forward.npz")
    elements = np.array([np.arange(8), np.arange(4, 12)])
    body = pd_oracle.Body.hex(
        h["vertices"], elements, np.arange(12) >= 4, h["materials"][:, 0], h["materials"][:, 1], 1000.0,
        material=material, muscle_directions=[[1.0, 0, 0], [0, 1.0, 0]], muscle_stiffness=[1000.0, 300.0],
        planes=(np.array([0, 8, 9]), 120.0, (0.0, 0.0, 2.0, -0.08)),
    )
    x, iterations, _ = pd_oracle.step(
        body, h["q"], h["v"], h["f"], np.zeros(3), 0.003, max_iterations=1000, abs_tol=1e-12, rel_tol=1e-10,
        window=0, targets=np.array([0.0, 0.8]),
    )
    np.testing.assert_allclose(x, h[material + "__x"], rtol=0, atol=1e-12)
    assert iterations == int(h[material + "__iterations"])
    np.testing.assert_allclose(np.linalg.inv(body.matrix(0.003)), h[material + "__inverse"], rtol=1e-12, atol=1e-16)


@pytest.mark.parametrize("key", ["c2_pd", "c1_pd", "c1_neo_hookean"])
def test_backward_matches_reference_backward(key):
    b = golden("tet_backward.npz")
    vertices, tets, poses, free = _tet_fixture()
    material = key.split("_", 1)[1]
    ml = b[key + "__mu_lame"]
    body = pd_oracle.Body.tet(tets, poses, free, ml[:, 0], ml[:, 1], 1000.0, material=material)
    out = pd_oracle.backward(body, b[key + "__x"], 0.004, b[key + "__gq"], b[key + "__gv"], mode="reference")
    for name in ("mu", "q", "qd", "f", "materials"):
        reference = b[key + "__out_" + name]
        np.testing.assert_allclose(out[name], reference, rtol=0, atol=1e-8 * np.abs(reference).max())


def test_projections_follow_unsigned_svd_conventions():
    # diag(1, 0, 1): Eigen keeps U = V, so the polar factor is the identity (reference test :181-204).
    f = np.diag([1.0, 0.0, 1.0])
    np.testing.assert_allclose(pd_oracle.corotated(f[None])[0] @ pd_oracle.corotated(f[None])[0].T, np.eye(3), atol=1e-14)
    # Reflections: U V^T has determinant -1 when det F < 0.
    r = pd_oracle.corotated(np.diag([1.0, 1.0, -0.5])[None])[0]
    assert abs(np.linalg.det(r) + 1.0) < 1e-12
    # The volume projection lands on det = 1.
    rng = np.random.default_rng(7)
    mats = np.eye(3) + 0.3 * rng.standard_normal((16, 3, 3))
    mats = mats[np.linalg.det(mats) > 0.1]
    np.testing.assert_allclose(np.linalg.det(pd_oracle.volume_projection(mats)), 1.0, atol=1e-9)


def test_mesh_contact_force_matches_reference_transcription():
    g = golden("mesh_contact.npz")
    for trial in range(4):
        expected = g[f"t{trial}__force"]
        got = pd_oracle.mesh_contact_force(g[f"t{trial}__q"], g[f"t{trial}__v"], g["faces_a"], g["faces_b"],
                                           *g["options"])
        np.testing.assert_allclose(got, expected, rtol=0.0, atol=1e-12 * max(np.abs(expected).max(), 1.0))


CONTACT_CASES = ["plane", "stick", "slide", "sphere", "chatter", "restitution", "mesh", "mesh_stick",
                 "mesh_restitution", "mesh_two_sided"]


def contact_scene(g, name):
    """Oracle body, boundary and per-step fixture inputs of one reference contact rollout."""
    if name.startswith("mesh"):
        vertices, tets = g["blocks__vertices"], g["blocks__tets"]
        free = g["blocks__free"]
        options = g[f"{name}__options"]
        parameters = (float(options[5]), int(g["blocks__split"]), g["blocks__faces_left"], g["blocks__faces_right"])
        boundary = pd_oracle.FrictionalBoundary("mesh", parameters, g[f"{name}__nodes"], friction=float(options[3]),
                                                restitution=float(options[4]))
    else:
        vertices, tets, _ = meshes.tet_grid(3, 2, 2, 0.1, origin=(0.0, 0.0, 1.0))
        free = np.ones(len(vertices), dtype=bool)
        options = g[f"{name}__options"]
        kind = "spherical" if name in ("sphere", "chatter") else "planar"
        boundary = pd_oracle.FrictionalBoundary(kind, g[f"{name}__parameters"], g["grid__nodes"],
                                                friction=float(options[3]), restitution=float(options[4]))
    poses = meshes.tet_rest_poses(vertices, tets).astype(np.float32).astype(np.float64)
    mu = np.full(len(tets), 2.0e4, dtype=np.float32).astype(np.float64)
    lame = np.full(len(tets), 5.0e4, dtype=np.float32).astype(np.float64)
    body = pd_oracle.Body.tet(tets, poses, free, mu, lame, 1000.0)
    solve = {"max_iterations": int(options[0]), "abs_tol": float(options[1]), "rel_tol": float(options[2])}
    steps = sum(1 for key in g.files if key.startswith(f"{name}__s") and key.endswith("__x"))
    return body, boundary, solve, steps


@pytest.mark.parametrize("name", CONTACT_CASES)
def test_frictional_boundary_matches_reference_transcription(name):
    """The restated frictional boundary against ``ReferenceContact`` / ``ReferenceMeshContact``
    rollouts (tests/test_diff_phd_contact.py:40-142, tests/test_diff_phd_mesh_boundary.py:42-110)."""
    g = golden("frictional_contact.npz")
    body, boundary, solve, steps = contact_scene(g, name)
    for t in range(steps):
        key = f"{name}__s{t}"
        q, v = g[key + "__q"], g[key + "__v"]
        x, iterations, converged = pd_oracle.step(body, q, v, np.zeros_like(q), GRAVITY, 0.004, contact=boundary,
                                                  **solve)
        assert iterations == int(g[key + "__iterations"])
        assert converged == bool(g[key + "__converged"])
        if not converged:
            # The stick/slip projection chatters to the iteration cap; the reference
            # compares only the iteration count and the status there.
            continue
        np.testing.assert_allclose(x, g[key + "__x"], rtol=0.0, atol=1.0e-9)
        if name.startswith("mesh"):
            np.testing.assert_array_equal(boundary.candidate.astype(np.int32), g[key + "__candidate"])
        if name != "mesh_two_sided":
            tolerance = {"rtol": 1.0e-5, "atol": 1.0e-6} if name.startswith("mesh") else {"rtol": 1.0e-6, "atol": 1.0e-9}
            np.testing.assert_allclose(boundary.multiplier, g[key + "__multiplier"], **tolerance)


@pytest.mark.parametrize("key", ["f0", "f5"])
def test_woodbury_projection_matches_reference_backward(key):
    """The restated contact projection of the parameter gradients against ``reference_backward``
    with contact (tests/reference_oracle.py:497-615) after a frictional rollout with fibres."""
    g = golden("woodbury.npz")
    vertices, tets, _ = meshes.tet_grid(3, 2, 2, 0.1, origin=(0.0, 0.0, 1.0))
    poses = meshes.tet_rest_poses(vertices, tets).astype(np.float32).astype(np.float64)
    mu = np.full(len(tets), 2.0e4, dtype=np.float32).astype(np.float64)
    lame = np.full(len(tets), 5.0e4, dtype=np.float32).astype(np.float64)
    body = pd_oracle.Body.tet(tets, poses, np.ones(len(vertices), dtype=bool), mu, lame, 1000.0,
                              muscle_directions=g[key + "__directions"], muscle_stiffness=np.full(len(tets), 4.0e4))
    friction = 0.5 if key == "f5" else 0.0
    contact = (g["nodes"], g[key + "__multiplier"], g[key + "__omega"], g[key + "__normal"], friction)
    targets = 1.0 - g[key + "__contraction"].astype(np.float64)
    out = pd_oracle.backward(body, g[key + "__x"], 0.004, g[key + "__gq"], g[key + "__gv"], targets=targets,
                             contact=contact)
    for name in ("mu", "z", "q", "qd", "f", "materials", "activations"):
        reference = g[f"{key}__out_{name}"]
        np.testing.assert_allclose(out[name], reference, rtol=0.0, atol=1.0e-6 * np.abs(reference).max(), err_msg=name)


@pytest.mark.parametrize("name", ["cancel", "grid2d", "tet322", "hex632"])
def test_factor_port_is_bit_identical_to_the_reference_setup(name):
    from oracle import factor_port

    g = golden("sparse_factors.npz")
    out = factor_port.inverse_factor(g[name + "__matrix"])
    for key in ("permutation", "s_offsets", "s_columns", "s_values", "st_offsets", "st_columns", "st_values"):
        np.testing.assert_array_equal(out[key], g[f"{name}__{key}"], err_msg=key)


def test_factor_port_rejects_what_the_reference_rejects():
    from oracle import factor_port

    with pytest.raises(ValueError, match="symmetric"):
        factor_port.inverse_factor(np.array([[2.0, 1.0], [0.5, 2.0]]))
    with pytest.raises(ValueError, match="positive"):
        factor_port.inverse_factor(np.array([[1.0, 2.0], [2.0, 1.0]]))


# The reference publishes its port's results on its own Hex8 cantilever
# (docs/validation/cantilever-reference-2026-11-02.json:264-265): min Gauss
# det(F) 0.9661699048673299 over the 25 axial steps, at most 16 iterations,
# and 192 iterations over steps 3..24 (cantilever-performance-2026-11-02.json:142).
def test_oracle_reproduces_the_published_axial_cantilever():
    from newton_solver_diff_phd_b200.scenes import ReferenceCantilever, reference_cantilever

    spec = ReferenceCantilever(edge=0.016, motion="axial")
    _, options, q0, tip = reference_cantilever(spec, device="cpu")
    mesh = options["hex_mesh"]
    mu, lam = options["hex_materials"].T
    body = pd_oracle.Body.hex(mesh.vertices, mesh.indices, mesh.vertices[:, 0] != 0.0, mu, lam, spec.density,
                              muscle_directions=options["muscle_directions"],
                              muscle_stiffness=options["muscle_stiffness"], planes=options["planar_energies"])
    q = q0.astype(np.float32).astype(np.float64)
    v = np.zeros_like(q)
    iterations, determinants = [], []
    for t in range(spec.steps):
        f = np.zeros_like(q)
        f[tip, 0] = np.float32(spec.tip_force(t))
        x, count, converged = pd_oracle.step(body, q, v, f, np.zeros(3), spec.dt, max_iterations=5000, abs_tol=1e-9,
                                             rel_tol=spec.rel_tol, window=5, targets=options["muscle_targets"])
        assert converged
        v = ((x - q) / spec.dt).astype(np.float32).astype(np.float64)
        q = x.astype(np.float32).astype(np.float64)
        iterations.append(count)
        determinants.append(np.linalg.det(body.deformation(q)).min())
    assert max(iterations) == 16
    assert sum(iterations[3:]) == 192
    assert abs(min(determinants) - 0.9661699048673299) < 1e-12


DIFF_PD_SCENES = ["free_fall", "pinned", "planar", "arc", "history", "external"]
DIFF_PD_FORCES = {
    "planar": [("planar_contact", [0.0, 0.0, 2.0, 0.0, 3, 1.0e6, 1.0, 0.1])],
    "arc": [("arc_contact", [0.0, 0.0, 1.0, 0.0, 2.0, 0.0, np.sin(np.radians(30.0)), 0.0, -np.cos(np.radians(30.0)),
                             1.0, np.radians(32.0), 3, 1.0e6, 1.0, 0.1])],
}


@pytest.mark.parametrize("scene", DIFF_PD_SCENES)
def test_diff_pd_oracle_matches_the_reference_oracle(scene):
    from oracle.diff_pd_oracle import DiffPdStep

    g = golden("diff_pd.npz")
    key = scene + "__"
    step = DiffPdStep(g[key + "rest"], g[key + "tets"], 1000.0, 4.0e4, 5.0e4, g[key + "free"], (0.0, 0.0, -9.81),
                      DIFF_PD_FORCES.get(scene, []))
    dt = float(g[key + "dt"])
    for t in range(len(g[key + "iterations"])):
        x, v, iterations = step.step(g[key + "q_in"][t], g[key + "v_in"][t], g[key + "f"][t], dt)
        assert iterations == int(g[key + "iterations"][t])
        assert step.halvings == int(g[key + "halvings"][t])
        assert step.fallbacks == int(g[key + "fallbacks"][t])
        np.testing.assert_allclose(x, g[key + "q_out"][t], rtol=0.0, atol=1e-12)
        np.testing.assert_allclose(v, g[key + "v_out"][t], rtol=0.0, atol=1e-10)
