"""Batched rollouts against the single-instance path, instance by instance."""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200 import SolverDiffPhD
from newton_solver_diff_phd_b200.batch import BatchedSolver
from newton_solver_diff_phd_b200.scenes import Cantilever, cantilever_model
from tests.helpers import tet_grid_model

pytestmark = pytest.mark.gpu

DT = 0.01
STEPS = 4


def _specs():
    rng = np.random.default_rng(5)
    sizes = [(4, 2), (7, 2), (12, 3), (9, 2), (5, 2)]
    youngs = [3e5, 2e6, 1e6, 5e6, 1e5]
    poissons = [0.35, 0.4, 0.45, 0.3, 0.42]
    return [Cantilever(nx, ny, ny, e, nu, rng.uniform(0.0, 5.0, (ny + 1) ** 2))
            for (nx, ny), e, nu in zip(sizes, youngs, poissons)]


def _instances(precision, window=5, with_tet=False):
    out = []
    for spec in _specs():
        model, mesh, materials, forces = cantilever_model(spec)
        solver = SolverDiffPhD(model, density=1000.0, hex_mesh=mesh, hex_materials=materials, precision=precision,
                               anderson_window=window, rel_tol=1e-6, abs_tol=1e-9, max_iterations=3000)
        out.append((model, solver, torch.as_tensor(forces, device="cuda")))
    if with_tet:
        model = tet_grid_model(gravity=0.0)
        solver = SolverDiffPhD(model, density=1000.0, precision=precision, anderson_window=window, rel_tol=1e-6,
                               abs_tol=1e-9, max_iterations=3000)
        forces = torch.zeros_like(model.particle_q)
        forces[:, 2] = 0.5
        out.append((model, solver, forces))
    return out


def _plain(model, solver, forces):
    state, out = model.state(), model.state()
    trajectory, iterations = [], []
    for _ in range(STEPS):
        state.particle_f.copy_(forces)
        solver.step(state, out, None, None, DT)
        trajectory.append(out.particle_q.clone())
        iterations.append(int(solver.iterations[0]))
        state, out = out, state
    solver.check_status()
    return torch.stack(trajectory), iterations


def _batched(instances, **options):
    batch = BatchedSolver([s for _, s, _ in instances], DT, **options)
    q0 = batch.concat([m.particle_q for m, _, _ in instances])
    qd0 = torch.zeros_like(q0)
    forces = batch.concat([f for _, _, f in instances])
    q, qd, x = batch.rollout(q0, qd0, forces, STEPS)
    status, iterations = batch.read()
    return batch, q, qd, x, status, iterations


SCHEDULES = ["teams", "phases"]


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_batched_fp64_matches_single_instance_steps(schedule):
    plain = [_plain(*inst) for inst in _instances("fp64", with_tet=True)]
    instances = _instances("fp64", with_tet=True)
    batch, q, qd, x, status, iterations = _batched(instances, schedule=schedule)
    assert np.all(status == 0), status
    for i, (trajectory, its) in enumerate(plain):
        got = batch.split(q)[i]
        scale = float(trajectory.abs().max())
        err = float((got - trajectory).abs().max())
        # Same algorithm, different reduction order: equal to rounding when the
        # iteration counts agree, within the convergence tolerance otherwise.
        assert np.all(np.abs(iterations[:, i] - np.asarray(its)) <= 1), (i, iterations[:, i], its)
        assert err <= 1e-6 * scale, (i, err, scale)
        np.testing.assert_allclose(batch.split(x)[i][-1].float().cpu(), got[-1].cpu(), rtol=0, atol=1e-6 * scale)


def _instances64(precision, rel_tol, max_iterations, abs_tol=1e-12):
    """The cantilevers with float64 states (no state rounding between steps)."""
    out = []
    for spec in _specs():
        model, mesh, materials, forces = cantilever_model(spec)
        solver = SolverDiffPhD(model, density=1000.0, hex_mesh=mesh, hex_materials=materials, precision=precision,
                               anderson_window=5, rel_tol=rel_tol, abs_tol=abs_tol, max_iterations=max_iterations,
                               state_dtype=torch.float64)
        out.append((model, solver, torch.as_tensor(forces, device="cuda", dtype=torch.float64)))
    return out


def _plain64(model, solver, forces):
    state, out = model.state(), model.state()
    for s in (state, out):
        s.particle_q, s.particle_qd, s.particle_f = s.particle_q.double(), s.particle_qd.double(), s.particle_f.double()
    trajectory = []
    for _ in range(STEPS):
        state.particle_f.copy_(forces)
        solver.step(state, out, None, None, DT)
        trajectory.append(solver._x.clone())
        state, out = out, state
    return torch.stack(trajectory)


def _relative(a, b):
    return float((a - b).abs().max()) / float(b.abs().max())


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_batched_fp32_refine_arithmetic_error_below_1e6(schedule):
    """Same iterations (no convergence stop): float32 factor products with
    float64 residual refinement stay within 1e-6 of the float64 iterates."""
    plain = [_plain64(*inst) for inst in _instances64("fp64", 0.0, 40, abs_tol=0.0)]
    batch, q, qd, x, status, iterations = _batched(_instances64("fp32+refine", 0.0, 40, abs_tol=0.0), schedule=schedule)
    assert np.all(iterations == 40), iterations
    for i, reference in enumerate(plain):
        assert _relative(batch.split(x)[i], reference) <= 1e-6, i


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_batched_fp32_refine_fixed_point_is_the_fp64_solution(schedule):
    """Converged tightly, float32 factor products reach the float64 solution
    (within 1e-6); at the working tolerance they land as close to it as the
    float64 solver itself. Float32 local projections move the fixed point by
    about cond(A) * 6e-8, bounded here at 1e-4."""
    truth = [_plain64(*inst) for inst in _instances64("fp64", 1e-12, 50000, abs_tol=0.0)]
    fp64 = [_plain64(*inst) for inst in _instances64("fp64", 1e-6, 20000)]
    tight = _batched(_instances64("fp32+refine", 1e-10, 50000, abs_tol=0.0), schedule=schedule)
    loose = _batched(_instances64("fp32+refine", 1e-6, 20000), schedule=schedule)
    fast = _batched(_instances64("fp32", 1e-8, 20000, abs_tol=0.0), schedule=schedule)
    assert np.all(tight[4] == 0) and np.all(loose[4] == 0) and np.all(fast[4] == 0)
    for i, (t, r) in enumerate(zip(truth, fp64)):
        assert _relative(tight[0].split(tight[3])[i], t) <= 1e-6, i
        e32 = _relative(loose[0].split(loose[3])[i], t)
        e64 = _relative(r, t)
        assert e32 <= 2.0 * e64 + 1e-6, (i, e32, e64)
        assert _relative(fast[0].split(fast[3])[i], t) <= 1e-4, i


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_batched_rollout_is_bitwise_deterministic_and_graph_is_reused(schedule):
    instances = _instances("fp32+refine", window=3)
    batch = BatchedSolver([s for _, s, _ in instances], DT, schedule=schedule)
    q0 = batch.concat([m.particle_q for m, _, _ in instances])
    qd0 = torch.zeros_like(q0)
    forces = batch.concat([f for _, _, f in instances])
    first = batch.rollout(q0, qd0, forces, STEPS)
    snapshot = [t.clone() for t in first]
    second = batch.rollout(q0, qd0, forces, STEPS, out=first)
    for a, b in zip(snapshot, second):
        assert torch.equal(a, b)


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_batched_per_step_forces_and_cold_svd(schedule):
    instances = _instances("fp64", window=0)
    batch = BatchedSolver([s for _, s, _ in instances], DT, schedule=schedule, svd_warm_start=False, task_nnz=512,
                          team_nnz=2048, team_samples=64)
    q0 = batch.concat([m.particle_q for m, _, _ in instances])
    qd0 = torch.zeros_like(q0)
    forces = batch.concat([f for _, _, f in instances])
    per_step = torch.stack([forces * (t + 1) / STEPS for t in range(STEPS)]).contiguous()
    q, _, _ = batch.rollout(q0, qd0, per_step, STEPS)
    for i, (model, solver, f) in enumerate(instances):
        state, out = model.state(), model.state()
        for t in range(STEPS):
            state.particle_f.copy_(f * (t + 1) / STEPS)
            solver.step(state, out, None, None, DT)
            state, out = out, state
        expected = state.particle_q
        scale = float(expected.abs().max())
        assert float((batch.split(q)[i][-1] - expected).abs().max()) <= 1e-6 * scale


def test_stepwise_launches_equal_the_graph():
    instances = _instances("fp32+refine")
    batch = BatchedSolver([s for _, s, _ in instances], DT, schedule="phases")
    q0 = batch.concat([m.particle_q for m, _, _ in instances])
    qd0 = torch.zeros_like(q0)
    forces = batch.concat([f for _, _, f in instances])
    graph = [t.clone() for t in batch.rollout(q0, qd0, forces, STEPS)]
    graph_iterations = batch.read()[1]
    stepwise = batch.rollout(q0, qd0, forces, STEPS, stepwise=True)
    assert np.array_equal(batch.read()[1], graph_iterations)
    for a, b in zip(graph, stepwise):
        assert torch.equal(a, b)


def test_teams_form_from_factor_and_sample_counts():
    instances = _instances("fp64")
    batch = BatchedSolver([s for _, s, _ in instances], DT, team_nnz=2048, team_samples=64)
    sizes, grid = batch.team_sizes()
    assert grid >= 1 and np.all(sizes >= 1) and np.all(sizes <= grid)
    assert sizes[2] > sizes[0]  # the 12x3x3 cantilever gets a larger team than the 4x2x2 one


@pytest.mark.parametrize("precision", ["fp64", "fp32+refine"])
def test_batched_adjoint_matches_single_instance_rollouts(precision):
    """Gradients of a loss on the final positions w.r.t. the initial state,
    every step's forces and the per-element Lame parameters: the teams
    adjoint against each instance's own Rollout backward."""
    from newton_solver_diff_phd_b200.rollout import Rollout

    def make():
        out = []
        for spec in _specs():
            model, mesh, materials, forces = cantilever_model(spec)
            solver = SolverDiffPhD(model, density=1000.0, hex_mesh=mesh, hex_materials=materials, precision=precision,
                                   anderson_window=5, rel_tol=1e-8, abs_tol=1e-12, max_iterations=20000,
                                   adjoint="exact", state_dtype=torch.float64)
            out.append((model, solver, torch.as_tensor(forces, device="cuda", dtype=torch.float64)))
        return out

    rng = np.random.default_rng(11)
    reference = []
    for model, solver, forces in make():
        driver = Rollout(solver, STEPS, DT)
        q0 = model.particle_q.double()
        final = driver.forward(q0, torch.zeros_like(q0), forces)
        weights = torch.as_tensor(rng.standard_normal(final.particle_q.shape), device="cuda")
        gq0, gqd0, gf, gm = driver.backward(weights, None)
        reference.append((weights, final.particle_q.clone(), gq0.clone(), gqd0.clone(), gf.clone(), gm.clone()))
    instances = make()
    batch = BatchedSolver([s for _, s, _ in instances], DT)
    q0 = batch.concat([m.particle_q for m, _, _ in instances])
    qd0 = torch.zeros_like(q0)
    forces = batch.concat([f for _, _, f in instances])
    q, qd, x = batch.rollout(q0, qd0, forces, STEPS)
    weights = batch.concat([r[0] for r in reference])
    gq0, gqd0, gf, gm, iterations = batch.backward(x, weights)
    assert np.all(iterations > 0)
    status, _ = batch.read()
    assert np.all((status & 8) == 0), status
    eo = batch.element_offsets
    for i, (w, final, rq, rqd, rf, rm) in enumerate(reference):
        for got, want in ((batch.split(q)[i][-1], final), (batch.split(gq0)[i], rq), (batch.split(gqd0)[i], rqd),
                          (batch.split(gf)[i], rf), (gm[eo[i]:eo[i + 1]], rm)):
            scale = float(want.abs().max())
            assert float((got - want).abs().max()) <= 1e-5 * scale + 1e-30, (i, float((got - want).abs().max()), scale)


def test_anderson_window_can_change_after_construction():
    """A solver switched to window 8 steps exactly like one built with it."""
    results = []
    for switch in (False, True):
        spec = _specs()[2]
        model, mesh, materials, forces = cantilever_model(spec)
        solver = SolverDiffPhD(model, density=1000.0, hex_mesh=mesh, hex_materials=materials,
                               anderson_window=3 if switch else 8, rel_tol=1e-6, abs_tol=1e-9)
        if switch:
            solver.set_anderson_window(8)
        results.append(_plain(model, solver, torch.as_tensor(forces, device="cuda")))
    assert torch.equal(results[0][0], results[1][0])
    assert results[0][1] == results[1][1]
    with pytest.raises(ValueError):
        solver.set_anderson_window(9)


def test_autotune_picks_a_probed_setting():
    from newton_solver_diff_phd_b200.batch import autotune

    instances = _instances("fp32+refine")
    solvers = [s for _, s, _ in instances]
    probe = BatchedSolver(solvers, DT)
    q0 = probe.concat([m.particle_q for m, _, _ in instances])
    forces = probe.concat([f for _, _, f in instances])
    del probe
    batch, report = autotune(solvers, DT, q0, torch.zeros_like(q0), forces, steps=1, windows=(3, 5),
                             teams=((65536, 512), (2048, 64)))
    assert len(report["probes"]) == 3
    chosen = report["chosen"]
    assert chosen["window"] in (3, 5) and all(s.anderson_window == chosen["window"] for s in solvers)
    assert min(p["ms"] for p in report["probes"]) == [p["ms"] for p in report["probes"]
                                                      if (p["window"], p["team_nnz"]) == (chosen["window"],
                                                                                          chosen["team_nnz"])][0]
    q, qd, x = batch.rollout(q0, torch.zeros_like(q0), forces, STEPS)
    status, _ = batch.read()
    assert np.all(status == 0)


def test_autotune_gives_a_stalling_instance_its_own_window():
    """Instance 203 of the family (6x2x2 cells, E 1.96e5 Pa, 219 N at the tip, nominal strain
    2.8) reaches the iteration limit with Anderson window 5 already in its second step, while
    plain local/global iterations (window 0) converge in under 1,000; instance 0 converges
    with either. The per-instance autotuner keeps mixing for the instance it helps and gives
    the stalling one window 0, and the tuned batch converges in every step."""
    from newton_solver_diff_phd_b200.batch import autotune
    from newton_solver_diff_phd_b200.scenes import cantilever_family

    family = cantilever_family(256, seed=0)
    instances = []
    for spec in (family[0], family[203]):
        model, mesh, materials, forces = cantilever_model(spec)
        solver = SolverDiffPhD(model, density=1000.0, hex_mesh=mesh, hex_materials=materials,
                               precision="fp32+refine", anderson_window=5, rel_tol=1e-6, abs_tol=1e-9,
                               max_iterations=5000)
        instances.append((model, solver, torch.as_tensor(forces, device="cuda")))
    solvers = [s for _, s, _ in instances]
    probe = BatchedSolver(solvers, DT)
    q0 = probe.concat([m.particle_q for m, _, _ in instances])
    forces = probe.concat([f for _, _, f in instances])
    del probe
    batch, report = autotune(solvers, DT, q0, torch.zeros_like(q0), forces, steps=2, windows=(0, 5),
                             teams=((65536, 512),), replan_steps=6, instance_windows=True)
    stalled_probe = [p for p in report["probes"] if p.get("window") == 5]
    assert stalled_probe and stalled_probe[0]["instances_at_limit"] == 1
    assert solvers[1].anderson_window == 0
    batch.rollout(q0, torch.zeros_like(q0), forces, 6)
    status, iterations = batch.read()
    assert np.all(status == 0) and iterations[:, 1].max() < 5000


def test_measured_replan_keeps_the_results():
    """A batch planned from a previous rollout's measured costs (team sizes and
    lanes) solves the same problems: single-instance results within 1e-6."""
    plain = [_plain(*inst) for inst in _instances("fp64")]
    instances = _instances("fp64")
    batch, q, _, _, status, _ = _batched(instances, team_nnz=2048, team_samples=64)
    us, iterations, teams, adjoint_us = batch.measurement()
    assert us.shape == iterations.shape == teams.shape == (len(instances),) and adjoint_us is None
    assert np.all(us > 0) and np.all(iterations >= STEPS)
    replanned, q2, _, _, status2, _ = _batched(instances, team_nnz=2048, team_samples=64,
                                               measured=(us, iterations, teams))
    sizes, grid = replanned.team_sizes()
    assert np.all(status2 == 0) and grid >= 1
    assert np.all((sizes & (sizes - 1)) == 0) and np.all(sizes <= 64)
    for i, (trajectory, _) in enumerate(plain):
        scale = float(trajectory.abs().max())
        assert float((replanned.split(q2)[i] - trajectory).abs().max()) <= 1e-6 * scale
    with pytest.raises(ValueError):
        BatchedSolver([s for _, s, _ in instances], DT, measured=(us[:2], iterations, teams))


def test_adjoint_lanes_from_measured_adjoint_durations_keep_the_gradients():
    """A batch re-planned with the adjoint's own measured durations (its own lanes) returns
    the adjoint of the first plan: same team sizes, so the same arithmetic."""
    instances = _instances("fp64")
    batch, q, qd, x, status, _ = _batched(instances, team_nnz=2048, team_samples=64)
    weight = torch.as_tensor(np.random.default_rng(8).standard_normal(tuple(q.shape[1:])), dtype=torch.float32,
                             device="cuda")
    first = [t.clone() for t in batch.backward(x, weight)[:4]]
    us, iterations, teams, adjoint_us = batch.measurement()
    assert adjoint_us is not None and adjoint_us.shape == (len(instances),) and np.all(adjoint_us > 0)
    replanned, q2, _, x2, status2, _ = _batched(instances, team_nnz=2048, team_samples=64,
                                                measured=(us, iterations, teams, adjoint_us))
    sizes, _ = replanned.team_sizes()
    second = replanned.backward(x2, weight)[:4]
    assert np.all(status2 == 0)
    if np.array_equal(sizes, teams):
        for a, b in zip(first, second):
            assert torch.equal(a, b)
    else:
        for a, b in zip(first, second):
            scale = float(a.abs().max())
            assert float((a - b).abs().max()) <= 1e-6 * max(scale, 1e-30)



def test_a_second_batch_over_the_same_solvers_leaves_the_first_valid():
    """Each batch owns its instances' team plans: building another batch (other team
    sizes) over the same solvers, or stepping a solver alone, does not disturb it."""
    instances = _instances("fp64")
    first, q, _, _, status, _ = _batched(instances, team_nnz=2048, team_samples=64)
    second, q2, _, _, _, _ = _batched(instances, team_nnz=1 << 20, team_samples=1 << 20)
    assert not np.array_equal(first.team_sizes()[0], second.team_sizes()[0])
    _plain(*instances[0])  # the solver plans its single-instance launch again
    q0 = first.concat([m.particle_q for m, _, _ in instances])
    forces = first.concat([f for _, _, f in instances])
    again, _, _ = first.rollout(q0, torch.zeros_like(q0), forces, STEPS)
    assert torch.equal(again, q)


def test_a_batch_refuses_to_run_after_its_solvers_were_resized():
    instances = _instances("fp64", window=3)
    batch, *_ = _batched(instances)
    instances[0][1].set_anderson_window(8)  # grows (reallocates) the history
    q0 = batch.concat([m.particle_q for m, _, _ in instances])
    with pytest.raises(RuntimeError):
        batch.rollout(q0, torch.zeros_like(q0), batch.concat([f for _, _, f in instances]), STEPS)
