"""Parity fixtures in the reference's newton.diff_phd_parity.v1 exchange format."""

import numpy as np
import pytest

from newton_solver_diff_phd_b200 import meshes, parity
from oracle import pd_oracle

pytestmark = pytest.mark.gpu


def _fixture(contact=False):
    vertices, tets, _ = meshes.tet_grid(3, 2, 2, 0.1, origin=(0.0, 0.0, 0.001 if contact else 1.0))
    rng = np.random.default_rng(3)
    n, steps = len(vertices), 3
    fixture = {
        "schema": np.asarray(parity.SCHEMA),
        "rest_vertices": vertices, "tets": tets, "density": 1000.0, "material": np.asarray("pd"),
        "mu": np.full(len(tets), 2.0e4), "lambda": np.full(len(tets), 5.0e4),
        "dirichlet": (vertices[:, 0] <= 1.0e-12) if not contact else np.zeros(n, dtype=bool),
        "q": vertices, "v": np.tile([0.0, 0.0, -1.0], (n, 1)) if contact else np.zeros((n, 3)),
        "f_ext": 0.1 * rng.standard_normal((steps, n, 3)), "gravity": np.array([0.0, 0.0, -9.81]), "dt": 0.004,
        "max_iterations": 2000, "abs_tol": 1.0e-12, "rel_tol": 1.0e-11,
        "objective_q": rng.standard_normal((n, 3)), "objective_v": 0.01 * rng.standard_normal((n, 3)),
    }
    if contact:
        fixture.update({"contact_kind": np.asarray("planar"), "contact_parameters": np.array([0.0, 0.0, 1.0, 0.0]),
                        "contact_vertices": np.unique(meshes.boundary_faces_tet(tets)), "friction": 0.4,
                        "restitution": 0.0})
    return fixture


def test_fixture_rollout_matches_the_oracle_and_round_trips(tmp_path):
    fixture = _fixture()
    out = parity.run(fixture)
    assert out["schema"] == parity.SCHEMA and out["q_next"].shape == (3,) + fixture["q"].shape
    assert np.all(out["converged"]) and out["dL_dmu"].shape == (len(fixture["tets"]),)
    # The first step against the oracle on the float32-rounded inputs.
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)  # noqa: E731
    poses = meshes.tet_rest_poses(f32(fixture["rest_vertices"]), fixture["tets"]).astype(np.float32)
    body = pd_oracle.Body.tet(fixture["tets"], poses, ~fixture["dirichlet"], f32(fixture["mu"]),
                              f32(fixture["lambda"]), 1000.0)
    x, iterations, converged = pd_oracle.step(body, f32(fixture["q"]), f32(fixture["v"]), f32(fixture["f_ext"][0]),
                                              f32(fixture["gravity"]), 0.004, max_iterations=2000, abs_tol=1e-12,
                                              rel_tol=1e-11)
    assert converged and iterations == int(out["iterations"][0])
    np.testing.assert_allclose(out["q_next"][0], x, rtol=0.0, atol=1.0e-6)
    path = tmp_path / "case.npz"
    parity.save(path, fixture, out)
    inputs, outputs = parity.load(path)
    assert str(inputs["schema"]) == parity.SCHEMA
    for key, value in out.items():
        np.testing.assert_array_equal(np.asarray(outputs[key]), np.asarray(value))
    bad = dict(fixture, schema=np.asarray("other.v0"))
    with pytest.raises(ValueError):
        parity.run(bad)


def test_contact_fixture_records_multipliers_and_gaps():
    out = parity.run(_fixture(contact=True))
    assert out["contact_multipliers"].shape[0] == 3 and out["planar_gaps"].shape == out["contact_multipliers"].shape
    active = out["contact_multipliers"] > 0
    assert active.any()
    np.testing.assert_allclose(out["planar_gaps"][active], 0.0, atol=1.0e-9)
    assert np.all(np.isfinite(out["dL_dq"])) and np.all(np.isfinite(out["dL_dmu"]))
