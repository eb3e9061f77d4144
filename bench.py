#!/usr/bin/env python
"""Benchmark of the DiffPhD projective-dynamics step and its adjoint on B200.

Metric: PD forward+adjoint steps per second (one PD time step forward plus its
adjoint), on the Tet4 block workload: a 32x8x8 block of 0.01 m cubes split
into 5 tetrahedra each (10,240 Tet4, 2,673 particles), per-tet Young's modulus
log-uniform in [1e5, 1e7] Pa (seed 0), nu 0.4, density 1000 kg/m^3, gravity
-9.81 m/s^2, the x=0 face pinned, 50 steps of dt 5e-3 s at relative tolerance
1e-6, float64. The loss is the squared distance of the final positions to the
rest pose plus a seeded 1 mm Gaussian displacement; the backward pass returns
its gradient with respect to every tet's Young's modulus (and the initial
state and forces). One bench step is one 50-step rollout forward and back.

``--gpus N`` (under torchrun) runs N independent replicas, one per GPU; a
single instance does not shard (its inverse factor is dense-ish and every
iteration would need an all-gather). ``value`` is the whole-job rate.

A second leg (N=1, ``--no-batched`` skips it) times the batched path on the
uneven Hex8 cantilever family (256 instances, nx uniform in [4, 40], ny =
nz = max(2, nx // 4), 25 steps of dt 0.01 s, fp32+refine, forward + adjoint
w.r.t. every instance's E) against the plain path stepping each instance on
its own, and reports both under ``batched``.

``--impl reference`` times the CPU port of the reference's sparse algorithm
(oracle/sparse_port.py; the reference's Warp CPU path needs warp-lang and
newton, which are not installed) on this host's cores, on the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

STEPS_PER_ROLLOUT = 50
DT = 5.0e-3
REL_TOL = 1.0e-6
ABS_TOL = 1.0e-9
NX, NY, NZ, EDGE = 32, 8, 8, 0.01
METRIC = "PD fwd+adjoint steps/s on 1 B200 at <=1e-6 rel err vs FP64; batched vs plain"
UNIT = "PD steps/s"
WORKLOAD = "tet4_block_32x8x8_fwd_adjoint_50steps"


def workload_arrays(seed=0):
    from newton_solver_diff_phd_b200 import meshes

    vertices, tets, _ = meshes.tet_grid(NX, NY, NZ, EDGE)
    rng = np.random.default_rng(seed)
    young = np.exp(rng.uniform(np.log(1.0e5), np.log(1.0e7), len(tets)))
    poisson = 0.4
    target = vertices + rng.normal(0.0, 1.0e-3, vertices.shape)
    return vertices, tets, young, poisson, target


def build_model(device):
    import torch

    from newton_solver_diff_phd_b200 import ModelBuilder, meshes

    vertices, tets, young, poisson, target = workload_arrays()
    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=NX, dim_y=NY, dim_z=NZ,
                          cell_x=EDGE, cell_y=EDGE, cell_z=EDGE, density=1000.0, k_mu=1.0, k_lambda=1.0, k_damp=0.0,
                          fix_left=True)
    model = builder.finalize(device)
    mu, lam = meshes.lame_from_young(young, poisson)
    with torch.no_grad():
        model.tet_materials.copy_(torch.tensor(np.column_stack((mu, lam, np.zeros_like(mu))), dtype=torch.float32))
    return model, young, poisson, target


def workload_config(args, nnz_s, world):
    """The workload both arms run (identical in both lines; measured values go elsewhere)."""
    return {
        "workload": WORKLOAD,
        "particles": (NX + 1) * (NY + 1) * (NZ + 1),
        "tets": 5 * NX * NY * NZ,
        "rollout_steps": STEPS_PER_ROLLOUT,
        "dt": DT,
        "rel_tol": REL_TOL,
        "abs_tol": ABS_TOL,
        "anderson_window": 5,
        "adjoint": f"{args.adjoint} (dL/dE of every tet; CG preconditioned by the factor)",
        "nnz_S": int(nnz_s),
        "l2": "GPU arm: 256 MiB write between timed rollouts (flush); the factor re-enters L2 within a rollout",
        "parallelism": f"replicas x{world}",
    }


def algorithmic_bytes_per_iteration(n, elements, nnz_s, corners=4, window=5, value_bytes=8):
    """Bytes one local/global iteration must move: factor values and indices of S and S^T, the vectors
    around the two products, element contributions, the Anderson history and the convergence norms
    (b = value bytes)."""
    b = value_bytes
    return (2 * (nnz_s * (b + 4) + 4 * (n + 1)) + 2 * (3 * n * b) * 2 + elements * corners * 4 + 3 * elements * 8
            + 3 * n * b + 3 * n * b + (2 * window + 4) * 3 * n * b + 4 * 3 * n * b)


class ClockSampler:
    """nvidia-smi clock/throttle sampling while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        self.file.flush()
        rows = []
        try:
            for line in Path(self.file.name).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        max_sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        loaded = sorted(sm)[len(sm) // 4:] if len(sm) >= 4 else sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(max_sm) if max_sm else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """Per-launch DRAM bytes of the forward step kernel from the committed ncu summary, if any."""
    path = ROOT / "profiles" / "forward_step_kernel_tet4_block.md"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch_scaled:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def run_b200(args):
    import torch

    from newton_solver_diff_phd_b200 import SolverDiffPhD, meshes
    from newton_solver_diff_phd_b200.rollout import Rollout

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    from newton_solver_diff_phd_b200 import distributed

    # One process per GPU; the group has a bounded collective timeout.
    ranks = distributed.setup("nccl", timeout_s=600.0, device=device)
    model, young, poisson, target = build_model(device)
    solver = SolverDiffPhD(model, density=1000.0, rel_tol=REL_TOL, abs_tol=ABS_TOL, adjoint=args.adjoint,
                           precision=args.precision)
    driver = Rollout(solver, STEPS_PER_ROLLOUT, DT)
    q0 = model.particle_q.clone()
    qd0 = torch.zeros_like(q0)
    target_t = torch.tensor(target, dtype=torch.float32, device=device)
    dmu_de, dlam_de, _, _ = meshes.lame_young_derivatives(poisson)
    dmu_de_t = torch.tensor(dmu_de, dtype=torch.float64, device=device)
    dlam_de_t = torch.tensor(dlam_de, dtype=torch.float64, device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    def one_rollout():
        final = driver.forward(q0, qd0)
        diff = final.particle_q - target_t
        loss = (diff.double() ** 2).sum()
        _, _, _, gml = driver.backward((2.0 * diff).float().contiguous())
        grad_e = gml[:, 0] * dmu_de_t + gml[:, 1] * dlam_de_t
        return loss, grad_e

    # Untimed build and warm-up.
    for _ in range(args.warmup):
        loss, grad_e = one_rollout()
    torch.cuda.synchronize()
    status = solver.read_status()
    stream = torch.cuda.current_stream()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    distributed.barrier(ranks)
    torch.cuda.synchronize()
    with ClockSampler(local) as sampler:
        for k in range(args.steps):
            flush.fill_(float(k))  # evict the factor from L2 between timed rollouts (untimed)
            starts[k].record(stream)
            loss, grad_e = one_rollout()
            ends[k].record(stream)
        torch.cuda.synchronize()
    clocks = sampler.summary()
    elapsed_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    elapsed_ms = distributed.max_over_ranks(elapsed_ms, ranks)
    status |= solver.read_status()
    errors = rollout_errors(driver, grad_e)
    total_steps = STEPS_PER_ROLLOUT * args.steps * world
    value = total_steps / (elapsed_ms / 1000.0)

    if args.no_extras:
        distributed.barrier(ranks)
        distributed.teardown(ranks)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "profiling_run": True}))
        return
    # Kernel-level timing of the persistent forward and adjoint launches (outside the timed region).
    rows, nnz_s, _ = solver.factor_stats()
    fwd_ms, fwd_iters, bwd_ms, bwd_iters = [], [], [], []
    import ctypes

    from newton_solver_diff_phd_b200 import _lib

    lib = _lib.library()
    state_a, state_b = model.state(), model.state()
    for state in (state_a, state_b):
        state.requires_grad_(True)
    with torch.no_grad():
        state_a.particle_q.copy_(q0)
    record = torch.zeros((solver._n, 3), dtype=torch.float64, device=device)
    for t in range(8):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.step(state_a, state_b, None, None, DT, record=record)
        e1.record(stream)
        torch.cuda.synchronize()
        fwd_ms.append(e0.elapsed_time(e1))
        fwd_iters.append(int(solver.iterations[0]))
        state_b.particle_q.grad.normal_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.backward_step(record, DT, state_a, state_b)
        e1.record(stream)
        torch.cuda.synchronize()
        bwd_ms.append(e0.elapsed_time(e1))
        bwd_iters.append(solver.backward_iterations)
        state_a, state_b = state_b, state_a
    solver.read_status()
    per_iter = algorithmic_bytes_per_iteration(rows, solver._element_count, nnz_s)
    fwd_bytes = per_iter * float(np.mean(fwd_iters))
    fwd_launch_ms = float(np.mean(fwd_ms))
    bwd_launch_ms = float(np.mean(bwd_ms))
    peak, peak_kind = measured_peak()
    achieved = fwd_bytes / (fwd_launch_ms / 1000.0) / 1e9
    traffic = profile_traffic()

    result = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": elapsed_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64-refine",
        "data": "synthetic (seeded Tet4 block; materials log-uniform from default_rng(0))",
        "config": workload_config(args, nnz_s, world),
        "bench_step": f"one {STEPS_PER_ROLLOUT}-step rollout forward and its adjoint ({STEPS_PER_ROLLOUT} PD steps)",
        "precision": args.precision,
        "errors": errors,
        "measured": {
            "sample_forward_iterations_mean": float(np.mean(fwd_iters)),
            "sample_backward_iterations_mean": float(np.mean(bwd_iters)),
            "status_bits": int(status),
        },
        "gpu_launches": 2 * STEPS_PER_ROLLOUT * args.steps,
        "clocks": clocks,
        "roofline": {
            "bound": "hbm",
            "kernel": "forward_step_kernel<double,double> (one launch = one PD step, all iterations)",
            "achieved": achieved,
            "peak": peak,
            "peak_kind": f"{peak_kind} burst copy GB/s",
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "algorithmic_bytes_per_launch": fwd_bytes,
            "launch_ms": fwd_launch_ms,
            "adjoint_launch_ms": bwd_launch_ms,
        },
    }
    if rank == 0:
        result["e2e"] = run_e2e(args, solver, driver, q0, target, young, dmu_de, dlam_de, device)
        result["cpu_baseline"] = cpu_baseline(args)
        if world == 1 and not args.no_batched:
            result["batched"] = run_batched(args, device)
        if world == 1 and not args.no_contact:
            result["contact"] = run_contact(args, device)
        if world == 1 and args.twist:
            result["twist"] = run_twist(args, device)
        if world == 1 and not args.no_cantilever:
            result["cantilever"] = run_cantilever(args, device)
        if world == 1 and not args.no_diffpd:
            result["diffpd"] = run_diffpd(args, device)
        if world == 1:
            result["factor_build"] = run_factor_build(device)
            if args.factor_twist:
                result["factor_build_twist"] = run_factor_build(device, twist=True)
    distributed.barrier(ranks)
    distributed.teardown(ranks)
    if rank == 0:
        print(json.dumps(result), flush=True)


def rollout_errors(driver, grad_e):
    """Errors of the last timed rollout against the CPU oracle's rollout of the same workload
    (tests/golden/tet_block_rollout.npz): final positions and dL/dE, relative in the 2-norm."""
    g = np.load(FIXTURE)
    final = driver.checkpoints[-1].particle_q.double().cpu().numpy()
    grad = grad_e.double().cpu().numpy()
    return {
        "position_rel_vs_fp64_oracle": float(np.linalg.norm(final - g["q_final"]) / np.linalg.norm(g["q_final"])),
        "position_max_abs_m": float(np.abs(final - g["q_final"]).max()),
        "grad_E_rel_vs_fp64_oracle": float(np.linalg.norm(grad - g["grad_young"]) / np.linalg.norm(g["grad_young"])),
        "oracle": "the reference algorithm in float64 on the CPU (oracle/sparse_port.py, exact inverse factor of "
                  "oracle/factor_port.py), same inputs; both stop at rel 1e-6",
    }


def run_e2e(args, solver, driver, q0, target, young, dmu_de, dlam_de, device):
    """The same metric through the public API with host buffers (pinned H2D in, D2H out, timed)."""
    import torch

    from newton_solver_diff_phd_b200.rollout import rollout

    host_q0 = q0.cpu().pin_memory()
    host_qd0 = torch.zeros_like(host_q0).pin_memory()
    host_target = torch.tensor(target, dtype=torch.float32).pin_memory()
    host_young = torch.tensor(young, dtype=torch.float64).pin_memory()
    out_loss = torch.empty(1, dtype=torch.float64).pin_memory()
    out_grad = torch.empty(len(young), dtype=torch.float64).pin_memory()
    nu = 0.4
    stream = torch.cuda.current_stream()
    steps = max(1, args.steps)

    def once():
        q = host_q0.to(device, non_blocking=True)
        qd = host_qd0.to(device, non_blocking=True)
        tgt = host_target.to(device, non_blocking=True)
        e = host_young.to(device, non_blocking=True).requires_grad_(True)
        mu = e / (2.0 * (1.0 + nu))
        lam = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        q_t, _ = rollout(driver, q, qd, None, torch.stack((mu, lam), dim=1))
        loss = ((q_t.double() - tgt.double()) ** 2).sum()
        loss.backward()
        out_loss.copy_(loss.detach().reshape(1), non_blocking=True)
        out_grad.copy_(e.grad, non_blocking=True)

    once()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        once()
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    h2d = host_q0.numel() * 4 * 3 + host_young.numel() * 8
    d2h = 8 + out_grad.numel() * 8
    return {"value": STEPS_PER_ROLLOUT * steps / (ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "grad_wrt": "per-tet Young's modulus (E), loss scalar"}


BATCH_COUNT = 256
BATCH_STEPS = 25
BATCH_DT = 0.01
BATCH_WORKLOAD = "hex8_cantilever_family_256_uneven_25steps_fwd_adjoint"


def batch_family(device, precision, count=BATCH_COUNT, rel_tol=REL_TOL, abs_tol=ABS_TOL, max_iterations=5000):
    """The uneven Hex8 cantilever family: solvers, per-instance forces and Poisson ratios."""
    import torch

    from newton_solver_diff_phd_b200 import SolverDiffPhD
    from newton_solver_diff_phd_b200.scenes import cantilever_family, cantilever_model

    out = []
    for spec in cantilever_family(count, seed=0):
        model, mesh, materials, forces = cantilever_model(spec, device=device)
        solver = SolverDiffPhD(model, density=1000.0, hex_mesh=mesh, hex_materials=materials, precision=precision,
                               anderson_window=5, rel_tol=rel_tol, abs_tol=abs_tol, max_iterations=max_iterations,
                               adjoint="exact")
        out.append((spec, model, solver, torch.as_tensor(forces, device=device)))
    return out


def build_all(solvers, dt):
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(os.cpu_count() or 4) as pool:  # the host factor builds release the GIL
        list(pool.map(lambda s: s._build(dt), solvers))


def precision_check(device, windows=None, stride=32, steps=BATCH_STEPS):
    """Errors of the batched leg on every `stride`-th instance of the family over the whole
    rollout, against batched fp64 converged to rel 1e-11: (1) fp32+refine converged to rel 1e-11
    as well, the error of the arithmetic alone; (2) fp32+refine at the bench's own stopping rule
    (rel 1e-6, abs 1e-9), the error the timed leg's results carry, instance by instance; (3)
    fp32+refine at rel 1e-9, the tightened rule of `accurate_batched`. Every run stops at 5,000
    iterations per step; instances that reach it in any run are left out of the maxima. `windows`
    gives every family instance's Anderson window (those of the timed batch; default 5)."""
    import torch

    from newton_solver_diff_phd_b200 import SolverDiffPhD
    from newton_solver_diff_phd_b200.batch import BatchedSolver
    from newton_solver_diff_phd_b200.scenes import cantilever_family, cantilever_model

    specs = cantilever_family(BATCH_COUNT, seed=0)[::stride]
    sample_windows = [5] * len(specs) if windows is None else list(windows)[::stride]
    runs = {"fp64": ("fp64", 1.0e-11, 1.0e-14, 5000), "fp32+refine": ("fp32+refine", 1.0e-11, 1.0e-14, 5000),
            "bench": ("fp32+refine", REL_TOL, ABS_TOL, 5000), "tight": ("fp32+refine", 1.0e-9, 1.0e-12, 5000)}
    results = {}
    for name, (precision, rel_tol, abs_tol, limit) in runs.items():
        solvers, models, forces = [], [], []
        for spec, window in zip(specs, sample_windows):
            model, mesh, materials, force = cantilever_model(spec, device=device)
            solvers.append(SolverDiffPhD(model, density=1000.0, hex_mesh=mesh, hex_materials=materials,
                                         precision=precision, anderson_window=window, rel_tol=rel_tol,
                                         abs_tol=abs_tol, max_iterations=limit, adjoint="exact"))
            models.append(model)
            forces.append(torch.as_tensor(force, device=device))
        build_all(solvers, BATCH_DT)
        batch = BatchedSolver(solvers, BATCH_DT)
        q0 = batch.concat([m.particle_q for m in models])
        q, _, x = batch.rollout(q0, torch.zeros_like(q0), batch.concat(forces), steps)
        rng = np.random.default_rng(2)
        weight = torch.as_tensor(rng.standard_normal((batch.particle_count, 3)), dtype=torch.float32, device=device)
        _, _, _, gm, _ = batch.backward(x, weight)
        status, _ = batch.read()
        eo = batch.element_offsets
        grad = [gm[eo[i]:eo[i + 1]].double().cpu().numpy() for i in range(batch.count)]
        results[name] = ([t.double().cpu().numpy() for t in batch.split(x[-1])], grad, (status & 1) == 0)
        del batch, solvers

    def errors(name):
        x, g, ok = results[name]
        x64, g64, ok64 = results["fp64"]
        keep = ok & ok64
        pos = np.array([np.abs(a - b).max() / np.abs(b).max() for a, b in zip(x, x64)])
        grad = np.array([np.abs(a - b).max() / np.abs(b).max() for a, b in zip(g, g64)])
        return pos, grad, keep

    pos, grad, keep = errors("fp32+refine")

    def per_instance(name, rel_tol, abs_tol):
        p, g, k = errors(name)
        k = k & keep
        return {"rel_tol": rel_tol, "abs_tol": abs_tol, "instances_converged": int(k.sum()),
                "rel_position_err_vs_fp64_1e-11": [float(e) if ok else None for e, ok in zip(p, k)],
                "rel_grad_err_vs_fp64_1e-11": [float(e) if ok else None for e, ok in zip(g, k)],
                "max_rel_position_err": float(p[k].max()) if k.any() else None,
                "max_rel_grad_err": float(g[k].max()) if k.any() else None,
                "instances_within_1e-6_position": int(np.count_nonzero(p[k] <= 1.0e-6))}

    return {"instances": [int(i) for i in range(0, BATCH_COUNT, stride)], "anderson_windows": sample_windows,
            "sample": f"every {stride}th instance of the family, all {steps} steps, final positions",
            "converged_both": int(keep.sum()), "steps": steps, "rel_tol": 1.0e-11,
            "max_rel_position_err_fp32_refine_vs_fp64": float(pos[keep].max()) if keep.any() else None,
            "max_rel_grad_mu_lambda_err_fp32_refine_vs_fp64": float(grad[keep].max()) if keep.any() else None,
            "at_bench_stopping_rule": per_instance("bench", REL_TOL, ABS_TOL),
            "at_rel_tol_1e-9": per_instance("tight", 1.0e-9, 1.0e-12),
            "note": "errors are max |x - x64| / max |x64| per instance (None: an instance that hit the iteration "
                    "limit in some run); the rel 1e-6 stop bounds the fixed-point step, not the distance to the "
                    "fixed point, which slow instances leave larger"}


def family_cpu_baseline(q_traj, qd_traj, offsets, forward_iterations, adjoint_iterations, strata=12, sample_step=12,
                        iterations=20):
    """The CPU port's cost of the whole family rollout. A single 4,961-particle Hex8 instance costs
    the NumPy port minutes, so the port is timed on a stratified sample and the timings are
    applied to the run's own iteration counts: the instances sorted by size, the median of each
    of `strata` strata plus both ends; for each, `iterations` forward local/global iterations and
    `iterations` adjoint CG iterations from its state at step `sample_step` of the batched rollout
    (one process per core, side by side; the inverse factor, bit-identical to
    oracle/factor_port.py's, is built beforehand and untimed). Per-iteration costs of the other
    instances are interpolated in the particle count (never extrapolated); the family's total is
    the sum over instances and steps of the recorded forward and adjoint iteration counts times
    those costs."""
    import multiprocessing

    import scipy.sparse as sp

    from newton_solver_diff_phd_b200 import _lib, meshes
    from newton_solver_diff_phd_b200.scenes import cantilever_family
    from oracle import pd_oracle
    from oracle.sparse_port import time_hex_iterations

    family = cantilever_family(BATCH_COUNT, seed=0)
    sizes = np.array([(s.nx + 1) * (s.ny + 1) * (s.nz + 1) for s in family])
    order = np.argsort(sizes, kind="stable")
    bounds = np.linspace(0, len(order), strata + 1)
    chosen = {int(order[int((lo + hi) // 2)]) for lo, hi in zip(bounds[:-1], bounds[1:])}
    chosen = sorted(chosen | {int(order[0]), int(order[-1])})  # the ends too: no extrapolation
    q_step = q_traj[sample_step - 1].double().cpu().numpy()
    qd_step = qd_traj[sample_step - 1].double().cpu().numpy()
    jobs = []
    for i in chosen:
        spec = family[i]
        vertices, hexes, _ = meshes.hex_grid(spec.nx, spec.ny, spec.nz, 0.01)
        free = vertices[:, 0] > 1.0e-12
        mu, lame = meshes.lame_from_young(np.full(len(hexes), spec.young), spec.poisson)
        tip = np.flatnonzero(np.abs(vertices[:, 0] - spec.nx * 0.01) <= 1.0e-12)
        forces = np.zeros_like(vertices)
        forces[tip, 0] = np.asarray(spec.tip_forces, dtype=np.float32)[: len(tip)]
        csr = sp.csr_matrix(pd_oracle.Body.hex(vertices, hexes, free, mu, lame, 1000.0).matrix(BATCH_DT))
        factor = _lib.inverse_factor((csr.indptr, csr.indices, csr.data))
        lo, hi = int(offsets[i]), int(offsets[i + 1])
        jobs.append((vertices, hexes, free, mu, lame, forces, factor, q_step[lo:hi], qd_step[lo:hi], BATCH_DT,
                     iterations))
    workers = max(1, min(os.cpu_count() or 1, len(jobs)))
    for name in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[name] = "1"
    jobs.sort(key=lambda job: -len(job[0]))
    start = time.perf_counter()
    with multiprocessing.get_context("spawn").Pool(workers) as pool:
        measured = sorted(pool.map(time_hex_iterations, jobs, chunksize=1))
    wall = time.perf_counter() - start
    n = np.array([m[0] for m in measured], dtype=np.float64)
    forward_cost = np.interp(sizes, n, [m[1] for m in measured])
    adjoint_cost = np.interp(sizes, n, [m[2] for m in measured])
    seconds = float(np.sum(forward_iterations * forward_cost[None, :]) + np.sum(adjoint_iterations * adjoint_cost[None, :]))
    steps = forward_iterations.shape[0] * forward_iterations.shape[1]
    return {"value": steps / seconds, "unit": "instance PD steps/s", "cores": 1, "kind": "port",
            "sample": f"per-iteration costs of oracle/sparse_port.py (one core each) "
                      f"measured on {len(chosen)} size-stratified instances {chosen} ({iterations} forward and "
                      f"{iterations} adjoint CG iterations from the batched rollout's step-{sample_step} state, "
                      f"{workers} processes side by side, {wall:.0f} s), interpolated in the particle count and "
                      f"applied to this run's {int(forward_iterations.sum())} forward and "
                      f"{int(adjoint_iterations.sum())} adjoint iterations: the family's rollout on one core",
            "estimated_single_core_seconds": seconds}


def batched_roofline(family, iterations, forward_ms):
    """HBM roofline of the batched forward launch: the algorithmic bytes of every local/global
    iteration of every instance, summed over the run's recorded iteration counts, per second of
    the launch. Per iteration of an instance (fp32+refine: float32 factor values and product
    vectors, float64 elsewhere): the two factor products 2 (nnz(S) (4 + 4) + 4 (N + 1)) and
    their vectors 2 (3N 4) 2, the element indices and contributions E 8 4 + 3E 8, the iterate
    and projection 2 (3N 8), the Anderson history (2m + 4) 3N 8, the convergence vectors
    4 (3N 8), and the float64 refinement residual nnz(A) (8 + 4) + 2 (3N 8); m is the instance's own
    Anderson window."""
    total = 0.0
    for i, (spec, _, solver, _) in enumerate(family):
        n = (spec.nx + 1) * (spec.ny + 1) * (spec.nz + 1)
        e = spec.nx * spec.ny * spec.nz
        nnz_s = solver.factor_stats()[1]
        counts = [np.array([1 + (k > 0) + (k < d) for k in range(d + 1)]) for d in (spec.nx, spec.ny, spec.nz)]
        nnz_a = int(np.einsum("i,j,k->", *counts))
        per_iteration = (2 * (nnz_s * 8 + 4 * (n + 1)) + 2 * (3 * n * 4) * 2 + e * 8 * 4 + 3 * e * 8 + 2 * 3 * n * 8
                         + (2 * solver.anderson_window + 4) * 3 * n * 8 + 4 * 3 * n * 8 + nnz_a * 12 + 2 * 3 * n * 8)
        total += float(iterations[:, i].sum()) * per_iteration
    peak, peak_kind = measured_peak()
    achieved = total / (forward_ms / 1000.0) / 1.0e9
    return {"bound": "hbm", "kernel": "team_forward_kernel<double,float> (one launch = the whole 25-step rollout)",
            "achieved": achieved, "peak": peak, "peak_kind": f"{peak_kind} burst copy GB/s", "unit": "GB/s",
            "frac": achieved / peak, "traffic": None, "algorithmic_bytes_per_launch": total,
            "traffic_note": "the 8-second launch is beyond the capture size rule; a small batch's DRAM traffic is "
                            "in profiles/team_forward_kernel_cantilever_batch.md"}


def stalled_instances(family, status):
    """The instances that hit the iteration limit in some step, with their nominal tip strain
    F / (E A) (total tip force over Young's modulus times the cross-section)."""
    out = []
    for i in np.flatnonzero(status & 1):
        spec = family[i][0]
        tip_force = float(np.sum(np.asarray(spec.tip_forces, dtype=np.float32)[: (spec.ny + 1) * (spec.nz + 1)]))
        area = spec.ny * spec.nz * 0.01 * 0.01
        out.append({"instance": int(i), "grid": [spec.nx, spec.ny, spec.nz], "young": spec.young,
                    "tip_force_n": tip_force, "nominal_strain": tip_force / (spec.young * area)})
    return out


def accurate_batched(family, chosen, measurement, q0, qd0, forces, weight, steps_total, rel_tol=1.0e-9,
                     abs_tol=1.0e-12):
    """The same batched forward + adjoint with the stopping rule tightened to `rel_tol`, the
    tolerance at which the final positions of the converged instances lie within 1e-6 of FP64
    solutions converged to rel 1e-11 (per-instance errors in `precision_check`). Same team sizes
    and lane plan as the timed run; one run, graph capture included."""
    import torch

    from newton_solver_diff_phd_b200.batch import BatchedSolver

    solvers = [s for _, _, s, _ in family]
    previous = [(s.rel_tol, s.abs_tol) for s in solvers]
    for s in solvers:
        s.set_tolerances(rel_tol=rel_tol, abs_tol=abs_tol)
    try:
        batch = BatchedSolver(solvers, BATCH_DT, team_nnz=chosen["team_nnz"], team_samples=chosen["team_samples"],
                              measured=measurement)
        batch.read()  # clears the status bits of the earlier runs
        stream = torch.cuda.current_stream()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        traj = batch.rollout(q0, qd0, forces, BATCH_STEPS)
        e1.record(stream)
        batch.backward(traj[2], weight)
        e2.record(stream)
        torch.cuda.synchronize()
        status, iterations = batch.read()
        fwd_ms, adj_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
        del batch, traj
    finally:
        for s, (rel, absolute) in zip(solvers, previous):
            s.set_tolerances(rel_tol=rel, abs_tol=absolute)
    return {"rel_tol": rel_tol, "abs_tol": abs_tol, "value": steps_total / ((fwd_ms + adj_ms) / 1000.0),
            "unit": "instance PD steps/s", "forward_ms": fwd_ms, "adjoint_ms": adj_ms,
            "forward_iterations": int(iterations.sum()),
            "instances_hitting_max_iterations": int(np.count_nonzero(status & 1)),
            "note": "one run with graph capture, same lanes as the timed run"}


def run_batched(args, device):
    """Batched vs plain on the uneven cantilever family (forward + adjoint w.r.t. every instance's E)."""
    import torch

    from newton_solver_diff_phd_b200 import meshes
    from newton_solver_diff_phd_b200.batch import BatchedSolver, autotune
    from newton_solver_diff_phd_b200.rollout import Rollout

    precision = "fp32+refine"
    family = batch_family(device, precision)
    build_all([s for _, _, s, _ in family], BATCH_DT)
    rng = np.random.default_rng(1)
    weights = [torch.as_tensor(rng.standard_normal((m.particle_count, 3)), dtype=torch.float32, device=device)
               for _, m, _, _ in family]
    # Autotuner (untimed): the Anderson window from 6-step probe rollouts
    # (3, 5, 8), the team sizing, and a re-plan of team sizes and lanes from
    # one measured 25-step rollout. (Per-instance windows with a window-0
    # fallback for stalled instances, `instance_windows=True`, converge more
    # of them but slow the batch by a third on this family and leave the
    # window-0 instances farther from the fixed point at rel 1e-6.)
    q0 = torch.cat([m.particle_q for _, m, _, _ in family]).contiguous()
    qd0 = torch.zeros_like(q0)
    forces = torch.cat([f for _, _, _, f in family]).contiguous()
    batch, tuning = autotune([s for _, _, s, _ in family], BATCH_DT, q0, qd0, forces, steps=6, windows=(3, 5, 8),
                             replan_steps=BATCH_STEPS)
    tuned = tuning["chosen"]
    tuned_plan = batch.measurement() if tuned.get("replanned") else None
    del batch
    # Plain path: every instance on its own, one cooperative launch per step
    # (default plans), with the tuned Anderson window.
    stream = torch.cuda.current_stream()
    plain_ms, plain_final = 0.0, []
    for (spec, model, solver, instance_forces), w in zip(family, weights):
        driver = Rollout(solver, BATCH_STEPS, BATCH_DT)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        final = driver.forward(model.particle_q, torch.zeros_like(model.particle_q), instance_forces)
        driver.backward(w, None)
        end.record(stream)
        torch.cuda.synchronize()
        plain_ms += start.elapsed_time(end)
        plain_final.append(final.particle_q.clone())
    plain_status = np.array([solver.read_status() for _, _, solver, _ in family])
    batch = BatchedSolver([s for _, _, s, _ in family], BATCH_DT, team_nnz=tuned["team_nnz"],
                          team_samples=tuned["team_samples"], measured=tuned_plan)
    sizes, grid = batch.team_sizes()
    weight = batch.concat(weights)
    eo = batch.element_offsets
    nu = torch.tensor(np.repeat([spec.poisson for spec, _, _, _ in family], np.diff(eo)), device=device)
    dmu_de = 1.0 / (2.0 * (1.0 + nu))
    dlam_de = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    index = torch.tensor(np.repeat(np.arange(batch.count), np.diff(eo)), device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    def one(out=None):
        traj = batch.rollout(q0, qd0, forces, BATCH_STEPS, out=out)
        gq0, gqd0, gf, gm, its = batch.backward(traj[2], weight)
        grad_e = torch.zeros(batch.count, dtype=torch.float64, device=device)
        grad_e.index_add_(0, index, gm[:, 0] * dmu_de + gm[:, 1] * dlam_de)
        return traj, grad_e, its

    def timed_one(out=None):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        result = one(out)
        b.record(stream)
        torch.cuda.synchronize()
        return result, a.elapsed_time(b)

    traj, grad_e, _ = one()  # captures the graphs
    (traj, grad_e, _), first_ms = timed_one(traj)
    # Re-plan the adjoint's lanes too, from this measured forward + adjoint (untimed).
    chosen = tuning["chosen"]
    replanned = BatchedSolver([s for _, _, s, _ in family], BATCH_DT, team_nnz=chosen["team_nnz"],
                              team_samples=chosen["team_samples"], measured=batch.measurement())
    one_batch = batch
    batch = replanned
    (traj2, _, _), _ = timed_one()
    (traj2, _, _), second_ms = timed_one(traj2)
    if second_ms < first_ms:
        traj = traj2
        tuning["chosen"]["adjoint_lanes"] = True
    else:
        batch = one_batch
    tuning["probes"].append({"adjoint_replan": True, "ms": first_ms, "replanned_ms": second_ms})
    del replanned, one_batch
    torch.cuda.synchronize()
    batch.read()  # clears the status bits of the untimed rollouts
    flush.fill_(1.0)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    traj = batch.rollout(q0, qd0, forces, BATCH_STEPS, out=traj)
    e1.record(stream)
    gq0, gqd0, gf, gm, adjoint_its = batch.backward(traj[2], weight)
    e2.record(stream)
    torch.cuda.synchronize()
    fwd_ms, adj_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    status, forward_its = batch.read()
    batched_ms = fwd_ms + adj_ms
    final = batch.split(traj[0][-1])
    converged = (status & 1) == 0
    errs = [float((a.double() - b.double()).abs().max() / b.double().abs().max()) for a, b in zip(final, plain_final)]
    err = max(e for e, ok in zip(errs, converged) if ok)
    # End to end through the public API with host buffers (pinned in, dL/dE out).
    host = {k: v.cpu().pin_memory() for k, v in (("q0", q0), ("forces", forces), ("weight", weight))}
    out_grad = torch.empty(batch.count, dtype=torch.float64).pin_memory()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    q0_d = host["q0"].to(device, non_blocking=True)
    forces_d = host["forces"].to(device, non_blocking=True)
    weight_d = host["weight"].to(device, non_blocking=True)
    traj_e = batch.rollout(q0_d, torch.zeros_like(q0_d), forces_d, BATCH_STEPS, out=traj)
    r = batch.backward(traj_e[2], weight_d)
    grad_e = torch.zeros(batch.count, dtype=torch.float64, device=device)
    grad_e.index_add_(0, index, r[3][:, 0] * dmu_de + r[3][:, 1] * dlam_de)
    out_grad.copy_(grad_e, non_blocking=True)
    end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = start.elapsed_time(end)
    steps_total = batch.count * BATCH_STEPS
    instances, particles = batch.count, int(batch.particle_count)
    batch_offsets = np.asarray(batch.particle_offsets)
    measurement = batch.measurement()
    del batch
    stalled = stalled_instances(family, status)
    roofline = batched_roofline(family, forward_its, fwd_ms)
    accurate = accurate_batched(family, chosen, measurement, q0, qd0, forces, weight, steps_total)
    precision = precision_check(device, windows=[s.anderson_window for _, _, s, _ in family])
    cpu = family_cpu_baseline(traj[0], traj[1], batch_offsets, forward_its, adjoint_its)
    return {
        "workload": BATCH_WORKLOAD,
        "metric": "instance PD steps/s (forward + adjoint w.r.t. every instance's E)",
        "value": steps_total / (batched_ms / 1000.0),
        "plain_value": steps_total / (plain_ms / 1000.0),
        "batched_vs_plain": plain_ms / batched_ms,
        "cpu_baseline": cpu,
        "batched_vs_cpu": (steps_total / (batched_ms / 1000.0)) / cpu["value"],
        "e2e": {"value": steps_total / (e2e_ms / 1000.0), "h2d_bytes_per_step": int(sum(v.numel() * v.element_size()
                                                                                         for v in host.values())),
                "d2h_bytes_per_step": int(out_grad.numel() * 8)},
        "forward_ms": fwd_ms,
        "adjoint_ms": adj_ms,
        "plain_ms": plain_ms,
        "precision": "fp32+refine",
        "precision_check": precision,
        "schedule": "teams",
        "autotune": tuning["chosen"],
        "autotune_probes": tuning["probes"],
        "plain_anderson_window": "the batch's",
        "plain_instances_with_status": int(np.count_nonzero(plain_status)),
        "instances": instances,
        "particles": particles,
        "team_sizes": {str(int(k)): int(v) for k, v in zip(*np.unique(sizes, return_counts=True))},
        "grid_blocks": int(grid),
        "forward_iterations": int(forward_its.sum()),
        "adjoint_iterations": int(adjoint_its.sum()),
        "max_iterations_per_step": 5000,
        "instances_hitting_max_iterations": int(np.count_nonzero(status & 1)),
        "stalled_instances": stalled,
        "roofline": roofline,
        "at_rel_tol_1e-9": accurate,
        "max_rel_position_err_vs_plain_same_precision": err,
        "err_note": "final positions, instances that converged within the iteration limit in every step; both paths "
                    "stop at rel 1e-6, so they differ by the stopping rule (the fixed point itself equals FP64's, "
                    "tests/test_gpu_batch.py)",
        "gpu_launches_per_rollout": 2,
        "data": "synthetic (cantilever_family(256, seed=0): nx uniform [4,40], ny=nz=max(2,nx//4), E log-uniform "
                "[1e5,1e7] Pa, nu uniform [0.3,0.45], tip +X forces uniform [0,50] N)",
    }


def run_contact(args, device):
    """The Tet4 contact workload (a 20x20x10 block of 1 mm cubes, 20,000 Tet4, on a frictional
    plane, poked by a meshed probe through the penalty mesh contact), twice:

    * as configured (dt 1 ms, probe 4 mm down over 200 steps): the first `contact_steps` steps
      forward, their state adjoint, and the contact projection of dL/d(mu, lambda) of the
      busiest converged step. At dt 1 ms the explicit penalty (kn 5e3 N/m on a 1.1 mg vertex)
      is outside its stability limit (dt < 2 / sqrt(kn / m) = 30 us), so this measures the
      contact machinery under chatter, not a physical poke;
    * a stable variant, all 200 steps: dt 20 us (omega dt = 1.35 < 2 for the penalty), the probe
      starting 0.6 mm above the block (outside the contact radius) and 1 mm down over the rollout
      (0.25 m/s), everything else the same.
    """
    from newton_solver_diff_phd_b200.scenes import Poke

    out = _contact_leg(Poke(offset=(0.0, 0.0)), args.contact_steps, device)
    if not args.no_contact_stable:
        stable = Poke(offset=(0.0, 0.0), dt=2.0e-5, probe_travel=1.0e-3, start_gap=0.6e-3)
        out["stable"] = _contact_leg(stable, stable.steps, device)
        out["stable"]["variant"] = ("dt 20 us (explicit penalty stable: omega dt = 1.35 < 2), the probe starting "
                                    "0.6 mm above the block (outside the 0.55 mm contact radius) and 1 mm down over "
                                    "200 steps; block, plane, probe and contact parameters as configured")
    return out


def _contact_leg(spec, steps, device):
    """One contact rollout of `steps` steps of `spec` (see `run_contact`)."""
    import torch

    from newton_solver_diff_phd_b200 import SolverDiffPhD, Tape
    from newton_solver_diff_phd_b200.scenes import poke_scene

    steps = min(steps, spec.steps)
    model, opt = poke_scene(spec, device=device)
    solver = SolverDiffPhD(model, density=spec.density, frictional_boundary=opt["frictional_boundary"],
                           frictional_vertices=opt["frictional_vertices"], mesh_contact=opt["mesh_contact"],
                           max_iterations=5000, rel_tol=REL_TOL, abs_tol=ABS_TOL)
    dirichlet = torch.as_tensor(opt["dirichlet"], device=device)
    rng = np.random.default_rng(0)
    chosen = rng.choice(np.unique(opt["surface"]), 64, replace=False)
    seed = torch.zeros((model.particle_count, 3), dtype=torch.float32, device=device)
    seed[chosen] = torch.as_tensor(rng.standard_normal((64, 3)), dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream()
    # Warm-up: the factor build, the panel of the plane's vertices and one step.
    warm_in, warm_out = model.state(), model.state()
    solver.step(warm_in, warm_out, None, None, spec.dt, dirichlet_positions=dirichlet[0])
    torch.cuda.synchronize()
    solver.read_status()
    states = [model.state(requires_grad=True) for _ in range(steps + 1)]
    iterations, active, pairs = [], [], []
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    forward_ms = 0.0
    with Tape() as tape:
        for t in range(steps):
            e0.record(stream)
            solver.step(states[t], states[t + 1], None, None, spec.dt, dirichlet_positions=dirichlet[t])
            e1.record(stream)
            torch.cuda.synchronize()
            forward_ms += e0.elapsed_time(e1)
            iterations.append(int(solver.iterations[0]))
            active.append(int((solver.contact_multipliers > 0).sum()))
            pairs.append(solver.mesh_contact_pairs)
    forward_status = solver.read_status()
    e0.record(stream)
    tape.backward(grads={states[-1].particle_q: seed})
    e1.record(stream)
    torch.cuda.synchronize()
    adjoint_ms = e0.elapsed_time(e1)
    adjoint_status = solver.read_status()
    # Parameter gradients through the contact projection, on the converged step
    # with the most active plane contacts: one call to plan and allocate, then
    # one timed call.
    converged = [t for t in range(steps) if iterations[t] < 5000]
    busiest = max(converged, key=lambda t: (active[t], -t)) if converged else steps - 1
    model.tet_materials.requires_grad_(True)
    woodbury = []
    for _ in range(2):
        model.tet_materials.grad = torch.zeros_like(model.tet_materials)
        step_in, step_out = model.state(requires_grad=True), model.state(requires_grad=True)
        with torch.no_grad():
            step_in.particle_q.copy_(states[busiest].particle_q)
            step_in.particle_qd.copy_(states[busiest].particle_qd)
        with Tape() as tape:
            solver.step(step_in, step_out, None, None, spec.dt, dirichlet_positions=dirichlet[busiest])
        rows = int((solver.contact_multipliers > 0).sum())
        e1.record(stream)
        tape.backward(grads={step_out.particle_q: seed})
        e2.record(stream)
        torch.cuda.synchronize()
        woodbury.append(e1.elapsed_time(e2))
    woodbury_status = solver.read_status()
    total_iterations = int(sum(iterations))
    return {
        "workload": "tet4_poke_block_20x20x10_plane_probe",
        "steps": steps,
        "forward_ms_per_step": forward_ms / steps,
        "forward_us_per_iteration": 1000.0 * forward_ms / max(total_iterations, 1),
        "forward_iterations": iterations,
        "steps_at_iteration_limit": int(sum(1 for i in iterations if i >= 5000)),
        "plane_contacts_active": active,
        "probe_pairs": pairs,
        "state_adjoint_ms_per_step": adjoint_ms / steps,
        "woodbury_step": {"step": busiest, "contact_rows_active": rows, "backward_ms": woodbury[1],
                          "first_call_ms": woodbury[0], "status": woodbury_status,
                          "note": "one step's whole backward with dL/d(mu, lambda) through the contact projection; "
                                  "the first call plans and allocates the column lanes"},
        "status_forward": forward_status,
        "status_adjoint": adjoint_status,
        "config": {"particles": model.particle_count, "tets": model.tet_count, "plane_vertices": 441,
                   "probe": f"icosphere r 3 mm (162 surface particles), prescribed {spec.probe_travel * 1e3:g} mm "
                            f"descent over {spec.steps} steps",
                   "mesh_contact": "radius 0.55 mm, kn 5e3 N/m, kf 50 N s/m, mu 0.5", "dt": spec.dt,
                   "rel_tol": REL_TOL, "precision": "fp64", "adjoint": "reference"},
        "data": "synthetic (block and probe built in scenes.poke_scene)",
    }


# The reference's own Hex8 cantilever (examples/_diff_phd_cantilever.py), whose
# port numbers the reference publishes for 0.016 m cells on a GB10:
# docs/validation/cantilever-performance-2026-11-02.json:43-46 (22 replayed
# steps in 41.9 ms of GPU graph time, 1.905 ms/step) and
# cantilever-reference-2026-11-02.json:264-265 (min Gauss det(F)
# 0.9661699048673299, at most 16 iterations).
PUBLISHED_CANTILEVER = {"gb10_graph_ms_per_step_replay": 1.905, "min_gauss_j": 0.9661699048673299,
                        "max_iterations": 16, "replay_iterations": 192}


def run_cantilever(args, device):
    """Forward steps of the reference cantilever (axial pull, 25 steps of dt 0.01 s, rel 1e-4) at the
    published 0.016 m cells and at BASELINE's 0.01 m cells, timed per step with CUDA events."""
    import torch

    from newton_solver_diff_phd_b200 import SolverDiffPhD
    from newton_solver_diff_phd_b200.scenes import ReferenceCantilever, reference_cantilever

    stream = torch.cuda.current_stream()
    out = {"workload": "reference Hex8 cantilever 20x5x5 (756 particles, 500 Hex8 x 8 samples), axial pull",
           "published_gb10": PUBLISHED_CANTILEVER}
    for edge in (0.016, 0.01):
        spec = ReferenceCantilever(edge=edge, motion="axial")
        model, options, q0, tip = reference_cantilever(spec, device=device)
        solver = SolverDiffPhD(model, **options)
        forces = torch.zeros((spec.steps, model.particle_count, 3), dtype=torch.float32, device=device)
        tip_index = torch.as_tensor(tip, device=device)
        for t in range(spec.steps):
            forces[t, tip_index, 0] = spec.tip_force(t)
        runs = []
        for _ in range(2):  # the first run builds the factor; the second is reported
            states = [model.state(), model.state()]
            states[0].particle_q.copy_(torch.as_tensor(q0, dtype=torch.float32, device=device))
            times, iterations, determinants = [], [], []
            for t in range(spec.steps):
                states[0].particle_f.copy_(forces[t])
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                solver.step(states[0], states[1], None, None, spec.dt)
                e1.record(stream)
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
                iterations.append(int(solver.iterations[0]))
                determinants.append(float(solver.deformation_determinants(states[1]).min()))
                states.reverse()
            runs.append((times, iterations, determinants, solver.read_status()))
        times, iterations, determinants, status = runs[-1]
        out[f"edge_{edge}"] = {
            "forward_ms_per_step": float(np.mean(times)),
            "forward_ms_per_step_steps_3_24": float(np.mean(times[3:])),
            "forward_us_per_iteration": 1000.0 * float(np.sum(times)) / max(1, sum(iterations)),
            "iterations": iterations,
            "min_gauss_det_F": min(determinants),
            "status": int(status),
        }
    published = PUBLISHED_CANTILEVER
    mine = out["edge_0.016"]
    out["vs_published_0.016"] = {
        "min_gauss_det_F_abs_diff": abs(mine["min_gauss_det_F"] - published["min_gauss_j"]),
        "max_iterations_equal": max(mine["iterations"]) == published["max_iterations"],
        "replay_iterations_equal": sum(mine["iterations"][3:]) == published["replay_iterations"],
        "replay_speedup_vs_gb10_graph_time": published["gb10_graph_ms_per_step_replay"]
        / mine["forward_ms_per_step_steps_3_24"],
    }
    return out


def run_diffpd(args, device):
    """The SolverDiffPD (L-BFGS) forward step on the Tet4 32x8x8 block of 1 cm cubes (the x = 0 face
    pinned, gravity, corotated 4e4 Pa and volume 5e4 Pa weights, density 1000 kg/m^3, a planar
    penalty contact with friction 0.5 m below the block, which the sagging beam does not reach in
    20 steps: at 2 cm the explicit penalty of the reference makes a step exhaust its 4,000
    iterations), `diffpd_steps` steps of dt 1e-2 at the
    reference's default tolerances (rel 1e-4, abs 1e-9, 10 history pairs): per-step device time
    and L-BFGS iterations, the first two steps checked against the NumPy restatement of the
    reference step (oracle/diff_pd_oracle.py, dense Cholesky of A), which is also timed on the host
    as the leg's CPU baseline."""
    import torch

    from newton_solver_diff_phd_b200 import ModelBuilder, SolverDiffPD
    from oracle.diff_pd_oracle import DiffPdStep

    builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=NX, dim_y=NY, dim_z=NZ,
                          cell_x=EDGE, cell_y=EDGE, cell_z=EDGE, density=1000.0, k_mu=2.0e4, k_lambda=5.0e4,
                          k_damp=0.0, fix_left=True)
    model = builder.finalize(device)
    forces = [("planar_contact", [0.0, 0.0, 1.0, 0.5, 3, 1.0e6, 1.0, 0.1])]
    solver = SolverDiffPD(model, density=1000.0, corotated_stiffness=4.0e4, volume_stiffness=5.0e4,
                          state_forces=forces, gravity=(0.0, 0.0, -9.81), recursion=args.diffpd_recursion)
    dt, steps = 1.0e-2, args.diffpd_steps
    states = [model.state(), model.state()]
    solver.step(states[0], states[1], None, None, dt)  # factor build and warm-up
    torch.cuda.synchronize()
    solver.check_status()
    states = [model.state(), model.state()]
    stream = torch.cuda.current_stream()
    ms, iterations, inputs, outputs = [], [], [], []
    for t in range(steps):
        if t < 2:
            inputs.append((states[0].particle_q.double().cpu().numpy(), states[0].particle_qd.double().cpu().numpy()))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.step(states[0], states[1], None, None, dt)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
        iterations.append(int(solver.iterations[0]))
        if t < 2:
            outputs.append(solver.positions.cpu().numpy())
        states.reverse()
    status = solver.read_status()
    oracle = DiffPdStep(model.particle_q.cpu().numpy().astype(np.float64),
                        model.tet_indices.cpu().numpy().reshape(-1, 4), 1000.0, 4.0e4, 5.0e4,
                        model.particle_inv_mass.cpu().numpy() > 0, (0.0, 0.0, -9.81), forces)
    errors, oracle_iterations, cpu_s = [], [], 0.0
    for (q, v), x in zip(inputs, outputs):
        start = time.perf_counter()
        x_ref, _, count = oracle.step(q, v, np.zeros_like(q), dt)
        cpu_s += time.perf_counter() - start
        errors.append(float(np.abs(x - x_ref).max()))
        oracle_iterations.append(int(count))
    return {"workload": "tet4_block_32x8x8_diffpd_lbfgs", "recursion": args.diffpd_recursion, "steps": steps,
            "ms_per_step": float(np.mean(ms)),
            "steps_per_s": 1000.0 * steps / float(np.sum(ms)),
            "us_per_iteration": 1000.0 * float(np.sum(ms)) / max(sum(iterations), 1), "iterations": iterations,
            "status": int(status), "first_steps_vs_oracle": {"max_abs_position_err_m": max(errors),
                                                             "iterations": iterations[:2],
                                                             "oracle_iterations": oracle_iterations},
            "cpu_baseline": {"value": len(inputs) / cpu_s, "unit": "DiffPD steps/s", "cores": os.cpu_count(),
                             "kind": "port", "sample": "the first two steps with oracle/diff_pd_oracle.py (NumPy, "
                                                       "dense Cholesky of A, threaded BLAS)"},
            "config": {"particles": model.particle_count, "tets": model.tet_count, "dt": dt, "rel_tol": 1.0e-4,
                       "abs_tol": 1.0e-9, "history": 10, "max_ls_iter": 10,
                       "state_forces": "gravity, planar_contact z = -0.5 m (p 3, kn 1e6, kf 1, mu 0.1)"}}


def run_factor_build(device, twist=False):
    """The exact inverse factor built on the host and with the numeric LDL^T and the rows of
    L^{-1} on the device: wall time of each build and whether every array is bit-identical. The
    matrix is the largest family instance's (Hex8 40x10x10 cells, 4,961 rows), or with `twist`
    the twist-release workload's (80x20x20 cells, 35,721 rows; the host build takes about a
    minute)."""
    import scipy.sparse as sp

    from newton_solver_diff_phd_b200 import _lib, meshes
    from newton_solver_diff_phd_b200.scenes import Twist
    from oracle import pd_oracle

    if twist:
        spec = Twist()
        vertices, hexes, cells = meshes.hex_grid(spec.nx, spec.ny, spec.nz, spec.edge)
        slab = np.asarray(cells)
        third = spec.nx // 3
        young = spec.young * np.where((slab > third) & (slab <= 2 * third), spec.stiff_ratio, 1.0)
        poisson, density, dt, name = spec.poisson, spec.density, spec.dt, "Hex8 twist release 80x20x20 cells, 35,721 rows"
    else:
        vertices, hexes, _ = meshes.hex_grid(40, 10, 10, 0.01)
        young = np.exp(np.random.default_rng(3).uniform(np.log(1.0e5), np.log(1.0e7), len(hexes)))
        poisson, density, dt, name = 0.45, 1000.0, BATCH_DT, "Hex8 cantilever 40x10x10 cells, 4,961 rows"
    free = vertices[:, 0] > 1.0e-12
    mu, lam = meshes.lame_from_young(young, poisson)
    matrix = sp.csr_matrix(pd_oracle.Body.hex(vertices, hexes, free, mu, lam, density).matrix(dt))
    matrix.sort_indices()
    csr = (matrix.indptr, matrix.indices, matrix.data)
    _lib.inverse_factor(csr, device=device.index or 0)  # context and module load, untimed
    start = time.perf_counter()
    host = _lib.inverse_factor(csr)
    host_s = time.perf_counter() - start
    start = time.perf_counter()
    on_device = _lib.inverse_factor(csr, device=device.index or 0)
    device_s = time.perf_counter() - start
    same = all(np.array_equal(host[k], on_device[k]) for k in host)
    return {"matrix": name, "nnz_S": int(len(host["s_values"])), "host_s": host_s, "device_s": device_s,
            "bit_identical": bool(same), "host_threads": os.cpu_count(),
            "note": "device build: numeric LDL^T and rows of L^{-1} on the GPU; ordering, symbolic fill and the "
                    "CSR assembly on the host threads in both builds"}


def run_twist(args, device):
    """The large Hex8 twist-release workload (80x20x20 cells, 35,721 particles): `twist_steps` steps
    of dt 1e-3 at rel 1e-6 forward, then the adjoint of the final tip rotation angle w.r.t. the
    initial positions and every cell's Young's modulus with a checkpoint every 10 steps (exact
    adjoint), in fp64 and in fp32+refine; the factor build is timed apart, on the host for the
    fp64 solver and with the numeric LDL^T and the rows of L^{-1} on the device for the fp32+refine
    solver (the two factors are bit-identical; tests/test_gpu_factor_device.py)."""
    import torch

    from newton_solver_diff_phd_b200 import SolverDiffPhD
    from newton_solver_diff_phd_b200.rollout import Rollout
    from newton_solver_diff_phd_b200.scenes import Twist, twist_cantilever

    spec = Twist()
    steps = min(args.twist_steps, spec.steps)
    model, mesh, materials, q0_host, tip = twist_cantilever(spec, device=device)
    q0 = torch.as_tensor(q0_host, dtype=torch.float32, device=device)
    qd0 = torch.zeros_like(q0)
    rest = torch.as_tensor(mesh.vertices[tip, 1:], dtype=torch.float64, device=device)
    rest = rest - rest.mean(dim=0)
    nu = spec.poisson
    dmu_de, dlam_de = 1.0 / (2.0 * (1.0 + nu)), nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    stream = torch.cuda.current_stream()
    out = {"workload": "hex8_twist_release_80x20x20", "steps": steps, "checkpoint_every": 10}
    results = {}
    for precision in ("fp64", "fp32+refine"):
        solver = SolverDiffPhD(model, density=spec.density, hex_mesh=mesh, hex_materials=materials,
                               precision=precision, rel_tol=REL_TOL, abs_tol=ABS_TOL, max_iterations=5000,
                               adjoint="exact")
        solver.set_factor_device(precision != "fp64")
        start = time.perf_counter()
        solver._build(spec.dt)
        build_s = time.perf_counter() - start
        driver = Rollout(solver, steps, spec.dt, checkpoint_every=10)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        final = driver.forward(q0, qd0)
        e1.record(stream)
        q = final.particle_q.detach().double().requires_grad_(True)
        tip_q = q[torch.as_tensor(tip, device=device), 1:]
        tip_q = tip_q - tip_q.mean(dim=0)
        cross = (rest[:, 0] * tip_q[:, 1] - rest[:, 1] * tip_q[:, 0]).sum()
        angle = torch.atan2(cross, (rest * tip_q).sum())
        (grad_q,) = torch.autograd.grad(angle, q)
        gq0, _, _, gm = driver.backward(grad_q.float().contiguous())
        e2.record(stream)
        torch.cuda.synchronize()
        status = solver.read_status()
        _, nnz_s, _ = solver.factor_stats()
        grad_e = (gm[:, 0] * dmu_de + gm[:, 1] * dlam_de).cpu().numpy()
        results[precision] = (final.particle_q.double().cpu().numpy(), grad_e, float(angle.detach()))
        out[precision] = {"factor_build_s": build_s, "factor_ldlt_and_inverse_rows_on": "host" if precision == "fp64"
                          else "device", "nnz_S": int(nnz_s), "forward_ms": e0.elapsed_time(e1),
                          "adjoint_ms": e1.elapsed_time(e2),
                          "fwd_adjoint_steps_per_s": steps / (e0.elapsed_time(e2) / 1000.0),
                          "final_tip_angle_deg": float(np.degrees(float(angle.detach()))), "status": int(status),
                          "max_abs_dangle_dE": float(np.abs(grad_e).max())}
        del driver, solver
        torch.cuda.empty_cache()
    x64, g64, _ = results["fp64"]
    x32, g32, _ = results["fp32+refine"]
    out["fp32_refine_vs_fp64"] = {
        "max_rel_position_err": float(np.abs(x32 - x64).max() / np.abs(x64).max()),
        "max_rel_grad_E_err": float(np.abs(g32 - g64).max() / np.abs(g64).max()) if np.abs(g64).max() > 0 else None,
        "note": "both stop at rel 1e-6 on the step rule; the arithmetic error alone is measured by the batched "
                "precision check at rel 1e-11",
    }
    return out


# ---------------------------------------------------------------------------
# The CPU side: the reference's algorithm for this path on the host cores.
# The reference's own CPU path (Warp CPU kernels) needs warp-lang and newton,
# which are not installed; oracle/sparse_port.py runs the same algorithm with
# NumPy/SciPy on a thread pool, with the inverse factor of
# oracle/factor_port.py (bit-identical to the reference's sparse.py setup).
# Nothing here loads this package's CUDA library.
#
# A PD step of the rollout costs between 4 and 900 local/global iterations
# (bursts where the pinned beam swings back), so a few consecutive steps are
# not a fair sample. tests/golden/tet_block_rollout.npz holds the oracle's own
# rollout of this workload: the input state of every second step and the loss
# gradient its adjoint receives. A CPU sample point is one of those 25 steps,
# forward then adjoint (conjugate gradients preconditioned by the factor, the
# same solver as the GPU arm's exact adjoint), from the recorded inputs.

FIXTURE = ROOT / "tests" / "golden" / "tet_block_rollout.npz"


class CpuWorkload:
    """The port on the bench's Tet4 block (built from the same arrays the solver gets)."""

    def __init__(self, threads):
        import scipy.sparse as sp

        from newton_solver_diff_phd_b200 import ModelBuilder, meshes
        from oracle import factor_port, pd_oracle
        from oracle.sparse_port import SparsePort

        vertices, tets, young, poisson, _ = workload_arrays()
        builder = ModelBuilder(gravity=(0.0, 0.0, -9.81))
        builder.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=None, vel=(0.0, 0.0, 0.0), dim_x=NX, dim_y=NY, dim_z=NZ,
                              cell_x=EDGE, cell_y=EDGE, cell_z=EDGE, density=1000.0, k_mu=1.0, k_lambda=1.0,
                              k_damp=0.0, fix_left=True)
        model = builder.finalize("cpu")
        mu, lam = meshes.lame_from_young(young, poisson)
        free = model.particle_inv_mass.numpy() > 0
        self.body = pd_oracle.Body.tet(model.tet_indices.numpy().reshape(-1, 4), model.tet_poses.numpy(), free,
                                       mu.astype(np.float32).astype(np.float64),
                                       lam.astype(np.float32).astype(np.float64), 1000.0)
        start = time.perf_counter()
        self.factor = factor_port.inverse_factor(sp.csr_matrix(self.body.matrix(DT)))
        self.setup_s = time.perf_counter() - start
        self.port = SparsePort(self.body, self.factor, DT, threads=threads)
        self.gravity = model.gravity.numpy()[0].astype(np.float64)
        self.fixture = np.load(FIXTURE)
        self.points = len(self.fixture["steps"])

    def run_point(self, k):
        """Forward then adjoint of sample point ``k``; returns ``(seconds, forward iterations, adjoint iterations)``."""
        g = self.fixture
        q = g["q_in"][k].astype(np.float64)
        v = g["qd_in"][k].astype(np.float64)
        start = time.perf_counter()
        x, forward, _ = self.port.step(q, v, np.zeros_like(q), self.gravity, max_iterations=10000, abs_tol=ABS_TOL,
                                       rel_tol=REL_TOL)
        _, _, backward = self.port.backward_cg(x, g["grad_q_out"][k].astype(np.float64),
                                               g["grad_qd_out"][k].astype(np.float64), max_iterations=10000,
                                               abs_tol=ABS_TOL, rel_tol=REL_TOL, mode="exact")
        return time.perf_counter() - start, forward, backward

    def stratified_points(self, count):
        """``count`` points that follow the rollout's iteration distribution: the points sorted by
        the oracle's forward iterations, the median of each of ``count`` equal strata."""
        iterations = self.fixture["iterations"][self.fixture["steps"]]
        order = np.argsort(iterations, kind="stable")
        bounds = np.linspace(0, len(order), count + 1)
        return [int(order[int((lo + hi) // 2)]) for lo, hi in zip(bounds[:-1], bounds[1:])]


def cpu_baseline(args, points=5):
    threads = os.cpu_count() or 1
    work = CpuWorkload(threads)
    chosen = work.stratified_points(points)
    total, forward, backward = 0.0, 0, 0
    for k in chosen:
        seconds, f, b = work.run_point(k)
        total += seconds
        forward += f
        backward += b
    steps = [int(work.fixture["steps"][k]) for k in chosen]
    return {"value": len(chosen) / total, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"PD steps {steps} of the 50-step rollout (the medians of {points} strata of the oracle's "
                      f"per-step iteration counts), each forward ({forward} iterations in all) then its exact adjoint "
                      f"by CG ({backward} iterations), from the oracle rollout's recorded inputs; "
                      "oracle/sparse_port.py on a thread pool, factor from oracle/factor_port.py "
                      f"({work.setup_s:.1f} s, untimed)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    work = CpuWorkload(threads)
    # Warm-up: the first step of the rollout (the cheapest, 40 iterations).
    for _ in range(args.warmup):
        work.run_point(0)
    # Timed step k: sample point (k * 25) // K, so the K steps spread evenly
    # over the rollout (all 25 points when K >= 25, cycling beyond).
    total, forward, backward, used = 0.0, 0, 0, []
    for k in range(args.steps):
        point = (k * work.points) // args.steps if args.steps <= work.points else k % work.points
        seconds, f, b = work.run_point(point)
        total += seconds
        forward += f
        backward += b
        used.append(int(work.fixture["steps"][point]))
    value = args.steps / total
    sample = (f"one PD step forward + exact adjoint per bench step, at rollout steps {used} "
              f"({forward} forward and {backward} adjoint CG iterations in all), from the oracle rollout's recorded "
              "inputs (tests/golden/tet_block_rollout.npz); oracle/sparse_port.py on a thread pool, the reference "
              "algorithm on the host cores (warp-lang and newton are not installed)")
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Tet4 block; materials log-uniform from default_rng(0))", "impl": "reference",
        "config": workload_config(args, nnz_s=len(work.factor["s_values"]), world=1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(result), flush=True)


def run_batch_profile(args):
    """A small batched rollout for profilers: the instances ``--profile-batch`` lists (indices into
    cantilever_family(256, seed=0)), ``--profile-steps`` steps, fp32+refine, teams schedule, run
    twice (the first rollout captures the graph)."""
    import torch

    from newton_solver_diff_phd_b200.batch import BatchedSolver

    device = torch.device("cuda", 0)
    chosen = [int(k) for k in args.profile_batch.split(",")]
    family = batch_family(device, "fp32+refine")
    family = [family[k] for k in chosen]
    build_all([s for _, _, s, _ in family], BATCH_DT)
    batch = BatchedSolver([s for _, _, s, _ in family], BATCH_DT)
    q0 = torch.cat([m.particle_q for _, m, _, _ in family]).contiguous()
    forces = torch.cat([f for _, _, _, f in family]).contiguous()
    traj = batch.rollout(q0, torch.zeros_like(q0), forces, args.profile_steps)
    traj = batch.rollout(q0, torch.zeros_like(q0), forces, args.profile_steps, out=traj)
    torch.cuda.synchronize()
    status, iterations = batch.read()
    print(json.dumps({"instances": chosen, "steps": args.profile_steps, "status": status.tolist(),
                      "iterations": iterations.sum(axis=0).tolist()}))


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["b200", "reference"], default="b200")
    parser.add_argument("--adjoint", choices=["reference", "exact"], default="exact")
    parser.add_argument("--precision", choices=["fp64", "fp32+refine"], default="fp64")
    parser.add_argument("--no-batched", action="store_true", help="skip the batched-vs-plain cantilever family leg")
    parser.add_argument("--no-contact", action="store_true", help="skip the Tet4 contact (poke) leg")
    parser.add_argument("--no-cantilever", action="store_true", help="skip the reference Hex8 cantilever leg")
    parser.add_argument("--contact-steps", type=int, default=30, help="steps of the contact leg's rollout")
    parser.add_argument("--no-contact-stable", action="store_true",
                        help="skip the contact leg's stable 200-step variant (dt 20 us)")
    parser.add_argument("--twist", action="store_true",
                        help="add the 35,721-particle Hex8 twist-release leg (minutes: its host factor build)")
    parser.add_argument("--twist-steps", type=int, default=100, help="steps of the twist-release leg")
    parser.add_argument("--no-diffpd", action="store_true", help="skip the SolverDiffPD (L-BFGS) leg")
    parser.add_argument("--diffpd-steps", type=int, default=20, help="steps of the SolverDiffPD leg")
    parser.add_argument("--diffpd-recursion", choices=("two_loop", "gram"), default="two_loop",
                        help="L-BFGS recursion of the SolverDiffPD leg (the reference's two loops or the Gram form)")
    parser.add_argument("--factor-device-rows", type=int, choices=(0, 1), default=0,
                        help="device rows of L^-1 in the factor-build legs: 0 chunked, 1 grouped dense segments")
    parser.add_argument("--profile-factor", action="store_true",
                        help="run only the factor-build leg (4,961 rows, or the twist matrix with --factor-twist; "
                             "host then device; for profilers)")
    parser.add_argument("--profile-diffpd", action="store_true",
                        help="run only the SolverDiffPD leg (for profilers; --diffpd-steps sets its length)")
    parser.add_argument("--factor-twist", action="store_true",
                        help="also time the twist-release matrix's factor build on the host and the device")
    parser.add_argument("--no-extras", action="store_true",
                        help="skip the e2e, CPU-baseline and per-launch timing legs (profiling runs)")
    parser.add_argument("--profile-batch", default=None,
                        help="comma-separated family instances: run only a small batched rollout (for profilers)")
    parser.add_argument("--profile-steps", type=int, default=2, help="steps of the --profile-batch rollout")
    args = parser.parse_args()
    if args.factor_device_rows:
        from newton_solver_diff_phd_b200 import _lib

        _lib.check(_lib.library().pd_factor_device_rows(args.factor_device_rows))
    if args.profile_batch:
        run_batch_profile(args)
        return
    if args.profile_diffpd:
        import torch

        print(json.dumps(run_diffpd(args, torch.device("cuda", 0))))
        return
    if args.profile_factor:
        import torch

        print(json.dumps(run_factor_build(torch.device("cuda", 0), twist=args.factor_twist)))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
