// Persistent forward step kernel, its helpers and small utility kernels.
#include <cuda_runtime.h>

#include "pd_forward.cuh"
#include "pd_friction.cuh"
#include "pd_kernels.h"
#include "pd_team.cuh"

// Phase timers of the persistent loop (rank 0 of the team, thread 0), compiled in only
// with -DPD_PHASE_TIMERS; the timing probe builds such a variant.
#ifdef PD_PHASE_TIMERS
#define PD_TIMER(slot)                                                              \
  do {                                                                             \
    if (team.rank == 0 && threadIdx.x == 0 && a.timers != nullptr) {              \
      unsigned long long now_;                                                     \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now_));                     \
      a.timers[slot] += now_ - timer_last_;                                        \
      timer_last_ = now_;                                                          \
    }                                                                              \
  } while (0)
#define PD_TIMER_START()                                                           \
  unsigned long long timer_last_ = 0;                                              \
  if (team.rank == 0 && threadIdx.x == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(timer_last_))
#else
#define PD_TIMER(slot) \
  do {                 \
  } while (0)
#define PD_TIMER_START() \
  do {                   \
  } while (0)
#endif

namespace pdb200 {

// Dual convergence gate of the previous iteration (kernels.py:354-401), by one
// warp while the other warps run the next local step: a fixed-order warp
// reduction of the per-block partials, then the decision. All blocks read it
// after the next barrier, so its latency leaves the critical path; a
// converged step costs one extra local step whose output is discarded.
__device__ void warp_convergence(const StepArgs& a, int blocks) {
  const int lane = threadIdx.x & 31;
  double sums[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double* row = a.partials + (48 + q) * blocks;
    double v = 0.0;
    for (int b = lane; b < blocks; b += 32) v += row[b];
    sums[q] = warp_sum(v);
  }
  if (lane == 0) {
    const double step_norm = sqrt(sums[0]);
    const double previous_norm = sqrt(sums[1]);
    const double change_norm = sqrt(sums[2]);
    const double projection_norm = sqrt(sums[3]);
    const int k = *a.iteration;
    *a.iteration = k + 1;
    if (k > 0 && step_norm <= a.rel_tol * previous_norm + a.abs_tol &&
        change_norm <= a.rel_tol * projection_norm + a.abs_tol) {
      *a.active = 0;
    } else if (k + 1 >= a.max_iterations) {
      *a.active = 0;
      atomicOr(a.status, kStatusNotConverged);
    } else {
      *a.active = 1;
    }
  }
}

// One projective-dynamics step of one instance by one team of blocks:
// prologue, every local/global iteration, epilogue. Returns false when a team
// barrier gave up (the status word says why).
// TL: precision of the local projections; TV: precision of the factor values;
// kContact: the frictional boundary is compiled in (single-instance launches).
template <typename TL, typename TV, bool kContact>
__device__ __forceinline__ bool forward_step_body(const StepArgs& a, const Team team, char* dyn_smem) {
  __shared__ double s_grad[8 * 8 * 3];
  __shared__ double s_scratch[kBlock];
  __shared__ double s_reduced[64];
  __shared__ double s_gamma[kMaxWindow];
  // Anderson state of the step, kept by every block: history count and start,
  // the count and start the last coefficients were solved for, acceptance.
  __shared__ int s_aa[5];
  __shared__ int s_control[8];
  const int gtid = team.rank * blockDim.x + threadIdx.x;
  const int gthreads = team.size * blockDim.x;
  const int n = a.n;
  if (a.hex) {
    for (int t = threadIdx.x; t < 8 * 8 * 3; t += blockDim.x) s_grad[t] = a.gradients[t];
  }
  // ---- Prologue: begin_step (kernels.py:155-190), explicit_boundary (:199-207),
  // read_activations (:136-152), begin_solve, Anderson reset.
  const double dt = a.dt;
  for (int i = gtid; i < n; i += gthreads) {
    const int f64 = a.state_f64;
    const V3<double> start =
        v3<double>(state_load(a.q_in, f64, 3 * i), state_load(a.q_in, f64, 3 * i + 1), state_load(a.q_in, f64, 3 * i + 2));
    const V3<double> velocity = v3<double>(state_load(a.qd_in, f64, 3 * i), state_load(a.qd_in, f64, 3 * i + 1),
                                           state_load(a.qd_in, f64, 3 * i + 2));
    store3(a.position, i, start);
    store3(a.velocity, i, velocity);
    V3<double> acceleration;
#pragma unroll
    for (int c = 0; c < 3; ++c) acceleration[c] = state_load(a.f_in, f64, 3 * i + c) / a.mass + a.gravity[c];
    V3<double> target;
#pragma unroll
    for (int c = 0; c < 3; ++c) target[c] = start[c] + dt * velocity[c] + dt * dt * acceleration[c];
    if (a.extra_force != nullptr) {
      // q~ += h^2/m f(q, v) of a state force (the reference's add_state_force).
#pragma unroll
      for (int c = 0; c < 3; ++c) target[c] = target[c] + dt * dt / a.mass * a.extra_force[3 * i + c];
    }
    store3(a.target, i, target);
    V3<double> boundary = v3<double>(0.0, 0.0, 0.0);
    if (a.free_[i] == 0) {
      if (a.dirichlet != nullptr) {
        boundary = v3<double>(state_load(a.dirichlet, f64, 3 * i), state_load(a.dirichlet, f64, 3 * i + 1),
                              state_load(a.dirichlet, f64, 3 * i + 2));
      } else {
        boundary = start;
        if (a.integrate_pinned) boundary = boundary + dt * velocity;
      }
    }
    store3(a.boundary, i, boundary);
    store3(a.x, i, start);
    store3(a.prev, i, start);
    store3(a.proj, i, v3<double>(0.0, 0.0, 0.0));
    store3(a.prev_proj, i, v3<double>(0.0, 0.0, 0.0));
  }
  if (a.activations != nullptr) {
    for (int e = gtid; e < a.ne; e += gthreads) {
      const double contraction = static_cast<double>(a.activations[e]);
      if (!isfinite(contraction) || contraction > 1.0 || (a.wm[e] == 0.0 && contraction != 0.0)) {
        atomicOr(a.status, kStatusActivation);
      }
      a.mtarget[e] = 1.0 - contraction;
    }
  }
  if (gtid == 0) {
    *a.iteration = 0;
    *a.active = 1;
  }
  if (threadIdx.x < 5) s_aa[threadIdx.x] = 0;
  // Factor slices of this block stay in shared memory for the whole step.
  const TV* s_values = sizeof(TV) == sizeof(double) ? reinterpret_cast<const TV*>(a.s_val)
                                                    : reinterpret_cast<const TV*>(a.s_val32);
  const TV* st_values = sizeof(TV) == sizeof(double) ? reinterpret_cast<const TV*>(a.st_val)
                                                     : reinterpret_cast<const TV*>(a.st_val32);
  if (a.resident) {
    load_slice<TV>(a.plan_s, s_values, dyn_smem, team.rank);
    load_slice<TV>(a.plan_st, st_values, dyn_smem, team.rank);
  }
  double* vector_smem = reinterpret_cast<double*>(dyn_smem + a.vector_smem_offset);
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  if constexpr (kContact) {
    if (a.fc.count > 0) {
      // Frictional boundary: frames, candidates, Delassus matrix (FrictionalContact.begin_step).
      fb_begin_frames(a, team);
      if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
      fb_begin_delassus(a, team);
    }
  }

  const int r0 = a.st_part[team.rank], r1 = a.st_part[team.rank + 1];
  // This block's partial-sum slots: my_partials[slot * team.size].
  double* my_partials = a.partials + team.rank;
  // Anderson history of the own rows: in shared memory when the plan made room.
  History history;
  if (a.hist_smem_offset >= 0) {
    history.x = reinterpret_cast<double*>(dyn_smem + a.hist_smem_offset);
    history.slot_stride = static_cast<size_t>(3) * a.hist_rows;
    history.g = history.x + (a.window + 1) * history.slot_stride;
    history.base = r0;
  } else {
    history.x = a.hist_x;
    history.g = a.hist_g;
    history.slot_stride = static_cast<size_t>(3) * n;
    history.base = 0;
  }

  PD_TIMER_START();
  for (int iter = 0;; ++iter) {
    // Decision for the previous iteration, overlapped with this local step.
    if (iter > 0 && team.rank == 0 && (threadIdx.x >> 5) == kWarps - 1) warp_convergence(a, team.size);
    // ---- P1: local step (warm-started SVD after the first iteration).
    if (a.hex) {
      local_step_hex<TL>(a, s_grad, iter > 0, team);
    } else {
      local_step_tet<TL>(a, iter > 0, team);
    }
    PD_TIMER(0);
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    PD_TIMER(5);
    if (iter > 0) {
      if (threadIdx.x == 0) s_control[0] = *reinterpret_cast<volatile int*>(a.active);
      __syncthreads();
      if (s_control[0] == 0) break;  // converged at iter - 1; x is that iterate
    }

    // ---- P2: fixed-order gather, vertex-plane energies, right-hand side.
    // Four lanes per particle: lane q sums entries q, q+4, ... of the
    // particle's element-ordered incidence list; a fixed shuffle tree joins
    // them, so the sum order is the same on every run.
    {
      const int sub = threadIdx.x & 3;
      const int groups_total = gthreads >> 2;
      const int lane_group = (threadIdx.x & 31) >> 2;
      const int warp_first = (gtid >> 5) * 8;
      for (int base = warp_first; base < n; base += groups_total) {
        const int i = base + lane_group;
        const bool valid = i < n;
        double px = 0.0, py = 0.0, pz = 0.0;
        double ax = 0.0, ay = 0.0, az = 0.0;
        if (valid) {
          const int k0 = a.inc_offsets[i], k1 = a.inc_offsets[i + 1];
#pragma unroll 4
          for (int k = k0 + sub; k < k1; k += 4) {
            const double* c = a.contrib + 3 * a.inc_entries[k];
            px += c[0];
            py += c[1];
            pz += c[2];
          }
          if (a.refine) {
            for (int k = a.a_off[i] + sub; k < a.a_off[i + 1]; k += 4) {
              const double v = a.a_val[k];
              const int j = a.a_col[k];
              ax += v * a.prev[3 * j];
              ay += v * a.prev[3 * j + 1];
              az += v * a.prev[3 * j + 2];
            }
          }
        }
#pragma unroll
        for (int mask = 1; mask < 4; mask <<= 1) {
          px += __shfl_xor_sync(0xffffffffu, px, mask);
          py += __shfl_xor_sync(0xffffffffu, py, mask);
          pz += __shfl_xor_sync(0xffffffffu, pz, mask);
          if (a.refine) {
            ax += __shfl_xor_sync(0xffffffffu, ax, mask);
            ay += __shfl_xor_sync(0xffffffffu, ay, mask);
            az += __shfl_xor_sync(0xffffffffu, az, mask);
          }
        }
        if (valid && sub == 0) {
          if (a.plane_weight != nullptr) {
            const double w = a.plane_weight[i];
            if (w != 0.0) {
              const double nx = a.plane[0], ny = a.plane[1], nz = a.plane[2];
              const double xx = a.x[3 * i], xy = a.x[3 * i + 1], xz = a.x[3 * i + 2];
              const double d = nx * xx + ny * xy + nz * xz + a.plane[3];
              const double m = fmin(0.0, d);
              px += w * ((xx - m * nx) - a.boundary[3 * i]);
              py += w * ((xy - m * ny) - a.boundary[3 * i + 1]);
              pz += w * ((xz - m * nz) - a.boundary[3 * i + 2]);
            }
          }
          a.proj[3 * i] = px;
          a.proj[3 * i + 1] = py;
          a.proj[3 * i + 2] = pz;
          // Residual form with refinement: b - A x_prev, in float64.
          a.rhs[3 * i] = a.inertia * a.target[3 * i] + px - ax;
          a.rhs[3 * i + 1] = a.inertia * a.target[3 * i + 1] + py - ay;
          a.rhs[3 * i + 2] = a.inertia * a.target[3 * i + 2] + pz - az;
        }
      }
    }
    PD_TIMER(1);
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    PD_TIMER(5);
    // ---- P3: y = S b (the residual in the refinement modes, in float32
    // when the slices and the float4 vector are resident).
    bool f32_vectors = false;
    if constexpr (sizeof(TV) == sizeof(float)) {
      f32_vectors = a.f32_vectors != 0;
      if (f32_vectors) {
        float4* staged = reinterpret_cast<float4*>(vector_smem);
        stage_vector_f32(a.plan_s, team.rank, a.rhs, staged, n);
        spmv_block_rows<TV>(a.plan_s, s_values, true, dyn_smem, VecF32{staged},
                            OutF32{reinterpret_cast<float4*>(a.y)}, team.rank);
      }
    }
    if (!f32_vectors) {
      const double* in = a.rhs;
      if (a.stage_vector) {
        stage_for(a.plan_s, team.rank, a.rhs, vector_smem, n);
        in = vector_smem;
      }
      spmv_block<TV>(a.plan_s, s_values, a.resident != 0, dyn_smem, in, a.y, team.rank);
    }
    PD_TIMER(2);
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    PD_TIMER(5);

    // ---- P4: x = S^T y, Dirichlet values, Anderson history and Gram partials.
    if constexpr (sizeof(TV) == sizeof(float)) {
      if (f32_vectors) {
        float4* staged = reinterpret_cast<float4*>(vector_smem);
        stage_float4(a.plan_st, team.rank, reinterpret_cast<const float4*>(a.y), staged, n);
        spmv_block_rows<TV>(a.plan_st, st_values, true, dyn_smem, VecF32{staged}, OutF64{a.x}, team.rank);
      }
    }
    if (!f32_vectors) {
      const double* in = a.y;
      if (a.stage_vector) {
        stage_for(a.plan_st, team.rank, a.y, vector_smem, n);
        in = vector_smem;
      }
      spmv_block<TV>(a.plan_st, st_values, a.resident != 0, dyn_smem, in, a.x, team.rank);
    }
    int contact_active = 0;
    if constexpr (kContact) {
      if (a.fc.count > 0) {
        // x = A^{-1} (b + J^T lambda): one Newton step on the multipliers (by
        // the first block for small contact sets, by the team for large ones),
        // then the correction through the panel columns.
        if (a.fc.kind == kBoundaryMesh && a.fc.restitution > 0.0) {
          for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) store3(a.fc.surface, i, load3d(a.prev, i));
        }
        if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
        if (a.fc.count <= kTeamContacts) {
          if (team.rank == 0) fb_newton(a);
          if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
        } else if (!fb_newton_team(a, team)) {
          return false;
        }
        contact_active = *reinterpret_cast<volatile int*>(a.fc.active);
      }
    }
    __syncthreads();
    const int count = a.window > 0 ? s_aa[0] : 0;
    const int start = a.window > 0 ? s_aa[1] : 0;
    const int capacity = a.window + 1;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      V3<double> value = load3d(a.x, i);
      if (a.refine) value = value + load3d(a.prev, i);
      if (contact_active > 0) value = value + fb_correction(a.fc, i, contact_active);
      if (a.free_[i] == 0) value = load3d(a.boundary, i);
      store3(a.x, i, value);
      if (a.window > 0) {
        const int slot = (start + count) % capacity;
        const V3<double> previous = load3d(a.prev, i);
        double* hx = history.xs(slot, i);
        double* hg = history.gs(slot, i);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          hx[c] = previous[c];
          hg[c] = value[c] - previous[c];
        }
      }
    }
    if (a.window > 0) {
      __syncthreads();
      gram_partials(history, a.window, r0, r1, count, start, my_partials, s_scratch, team.size);
      PD_TIMER(3);
      // Every block reduces the partials in the same fixed order and solves
      // the same small least-squares problem, so every block holds the same
      // coefficients and history state: no serial section, no release wait.
      if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
      reduce_partials(a.partials, 0, gram_entries(count), team.size, s_reduced, s_scratch);
      if (threadIdx.x == 0) aa_solve(s_aa, s_gamma, s_aa + 4, s_reduced, a.window, s_scratch);
      __syncthreads();
      PD_TIMER(6);
    }

    // ---- P5: Anderson apply, Dirichlet re-imposition, convergence partials.
    {
      int accept = 0, used_count = 0, used_start = 0;
      if (a.window > 0) {
        accept = s_aa[4];
        used_count = s_aa[2];
        used_start = s_aa[3];
      }
      double step2 = 0.0, prev2 = 0.0, change2 = 0.0, proj2 = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        V3<double> value = load3d(a.x, i);
        if (accept) value = aa_apply_row(history, a.window, i, used_count, used_start, s_gamma);
        if (a.free_[i] == 0) value = load3d(a.boundary, i);
        store3(a.x, i, value);
        const V3<double> previous = load3d(a.prev, i);
        const V3<double> p = load3d(a.proj, i);
        const V3<double> pp = load3d(a.prev_proj, i);
        const V3<double> step = value - previous;
        const V3<double> change = p - pp;
        step2 += dot(step, step);
        prev2 += dot(previous, previous);
        change2 += dot(change, change);
        proj2 += dot(pp, pp);
        store3(a.prev, i, value);
        store3(a.prev_proj, i, p);
      }
      step2 = block_sum(step2, s_scratch);
      prev2 = block_sum(prev2, s_scratch);
      change2 = block_sum(change2, s_scratch);
      proj2 = block_sum(proj2, s_scratch);
      PD_TIMER(4);
      if (threadIdx.x == 0) {
        my_partials[48 * team.size] = step2;
        my_partials[49 * team.size] = prev2;
        my_partials[50 * team.size] = change2;
        my_partials[51 * team.size] = proj2;
      }
      // The decision is taken by one warp during the next local step.
      if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
      PD_TIMER(7);
    }
  }

  if constexpr (kContact) {
    if (a.fc.count > 0 && a.fc.restitution > 0.0) {
      // FrictionalContact.finish_step: restitution on the converged positions.
      fb_restitution(a, team);
      if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    }
  }
  // ---- Epilogue: write_state (kernels.py:404-414) and the step record.
  for (int i = gtid; i < n; i += gthreads) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double value = a.x[3 * i + c];
      state_store(a.q_out, a.state_f64, 3 * i + c, value);
      state_store(a.qd_out, a.state_f64, 3 * i + c, (value - a.position[3 * i + c]) / dt);
      if (a.x_record != nullptr) a.x_record[3 * i + c] = value;
    }
  }
  return true;
}

// Plain launch: the whole cooperative grid is one team solving one instance.
template <typename TL, typename TV>
__global__ void __launch_bounds__(kBlock) forward_step_kernel(const StepArgs a) {
  extern __shared__ __align__(16) char dyn_smem[];
  forward_step_body<TL, TV, true>(a, Team{static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x)}, dyn_smem);
}

// Whole forward rollouts of many instances, each by a team of blocks: the
// single-instance step body with the team's rank and size, one step after
// the other, a team barrier between steps (the next step reads the states
// every member wrote).
template <typename TL, typename TV>
__global__ void __launch_bounds__(kBlock, 2) team_forward_kernel(const TeamLaunch launch) {
  extern __shared__ __align__(16) char dyn_smem[];
  __shared__ StepArgs s_args;
  Team lane_team;
  const int lane = lane_of_block(launch, lane_team);
  GridBarrier* barrier = &launch.lane_barrier[lane];
  const int f64 = launch.state_f64;
  const long long step_elements = 3 * launch.particles;
  bool solo = false;
  for (;;) {
    Team team;
    const int instance = next_work(launch, lane, lane_team, solo, team);
    if (instance < 0) return;
    copy_arguments(launch.forward + instance, &s_args);
    if (launch.timeline != nullptr && team.rank == 0 && threadIdx.x == 0) {
      unsigned long long now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      launch.timeline[2 * instance] = now;
    }
    const long long offset = 3 * launch.particle_offset[instance];
    __syncthreads();
    for (int t = 0; t < launch.steps; ++t) {
      if (threadIdx.x == 0) {
        s_args.barrier = barrier;
        s_args.q_in = t == 0 ? state_offset(launch.q0, f64, offset)
                             : state_offset(static_cast<const void*>(launch.q_traj), f64, (t - 1) * step_elements + offset);
        s_args.qd_in = t == 0 ? state_offset(launch.qd0, f64, offset)
                              : state_offset(static_cast<const void*>(launch.qd_traj), f64, (t - 1) * step_elements + offset);
        s_args.f_in = state_offset(launch.forces, f64, t * launch.force_stride + offset);
        s_args.dirichlet = nullptr;
        s_args.q_out = state_offset(launch.q_traj, f64, t * step_elements + offset);
        s_args.qd_out = state_offset(launch.qd_traj, f64, t * step_elements + offset);
        s_args.x_record = launch.x_record != nullptr ? launch.x_record + t * step_elements + offset : nullptr;
        s_args.dt = launch.dt;
        for (int c = 0; c < 3; ++c) s_args.gravity[c] = launch.gravity[c];
        s_args.timers = instance == launch.timer_instance ? launch.timers : nullptr;
      }
      __syncthreads();
      if (!forward_step_body<TL, TV, false>(s_args, team, dyn_smem)) return;
      if (team.rank == 0 && threadIdx.x == 0 && launch.iteration_log != nullptr)
        launch.iteration_log[t * launch.count + instance] = *s_args.iteration;
      // The next step reads the states every rank of the lane wrote.
      if (!grid_sync(barrier, s_args.status, team.size, team.rank)) return;
    }
    if (launch.timeline != nullptr && team.rank == 0 && threadIdx.x == 0) {
      unsigned long long now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      launch.timeline[2 * instance + 1] = now;
    }
  }
}

// Plain out = S^T (S rhs) with separate launches (SparseInverse.apply).
template <typename TV>
__global__ void __launch_bounds__(kBlock) spmv_kernel(const int* off, const int* col, const TV* val, const double* vec,
                                                      double* out, int rows) {
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int warps_total = (gridDim.x * blockDim.x) >> 5;
  for (int row = warp_global; row < rows; row += warps_total) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int k = off[row] + lane; k < off[row + 1]; k += 32) {
      const double value = static_cast<double>(val[k]);
      const int c = col[k];
      sx += value * vec[3 * c];
      sy += value * vec[3 * c + 1];
      sz += value * vec[3 * c + 2];
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    sz = warp_sum(sz);
    if (lane == 0) {
      out[3 * row] = sx;
      out[3 * row + 1] = sy;
      out[3 * row + 2] = sz;
    }
  }
}

__global__ void set_spin_limit_kernel(GridBarrier* barrier, unsigned limit) { barrier->spin_limit = limit; }

// Waits at a barrier that never completes: the team is `blocks + missing`
// blocks, only `blocks` are launched. The wait gives up after the barrier's
// poll budget (or when another block raised the abort flag) and the block
// counts itself out.
__global__ void __launch_bounds__(kBlock) barrier_probe_kernel(GridBarrier* barrier, int* status, int* returned,
                                                               int missing, int mode) {
  const int team = static_cast<int>(gridDim.x) + missing;
  bool ok;
  if (mode == 0) {
    ok = grid_sync(barrier, status, team, static_cast<int>(blockIdx.x));
  } else {
    unsigned generation;
    if (barrier_arrive(barrier, generation, team)) {
      barrier_release(barrier, generation, team);  // not reached while missing > 0
      ok = true;
    } else {
      ok = barrier_wait(barrier, generation, status);
    }
  }
  if (!ok && threadIdx.x == 0) atomicAdd(returned, 1);
}

__global__ void hex_determinants_kernel(const float* q, const int* indices, const double* gradients, int ne,
                                        double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ne * 8) return;
  const int e = t / 8;
  const int s = t % 8;
  M3<double> f = zero3<double>();
  for (int j = 0; j < 8; ++j) {
    const int v = indices[8 * e + j];
    const double* g = gradients + (8 * s + j) * 3;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) f.a[r][c] += static_cast<double>(q[3 * v + r]) * g[c];
  }
  out[t] = determinant(f);
}

// ---------------------------------------------------------------------------
// Host launchers.

// precision 0: FP64; 1: FP64 local step, FP32 factor products; 2: FP32 local step and factor.
static const void* forward_kernel(int precision) {
  if (precision == 0) return reinterpret_cast<const void*>(&forward_step_kernel<double, double>);
  if (precision == 1) return reinterpret_cast<const void*>(&forward_step_kernel<double, float>);
  return reinterpret_cast<const void*>(&forward_step_kernel<float, float>);
}

static const void* team_forward(int precision) {
  if (precision == 0) return reinterpret_cast<const void*>(&team_forward_kernel<double, double>);
  if (precision == 1) return reinterpret_cast<const void*>(&team_forward_kernel<double, float>);
  return reinterpret_cast<const void*>(&team_forward_kernel<float, float>);
}

cudaError_t launch_team_forward(const TeamLaunch& launch, int blocks, int precision, size_t smem, cudaStream_t stream) {
  void* params[] = {const_cast<TeamLaunch*>(&launch)};
  return cudaLaunchCooperativeKernel(team_forward(precision), dim3(blocks), dim3(kBlock), params, smem, stream);
}

cudaError_t team_forward_max_blocks(int precision, size_t smem, int* blocks_per_sm) {
  const void* kernel = team_forward(precision);
  int device = 0, optin = 0;
  cudaError_t status = cudaGetDevice(&device);
  if (status != cudaSuccess) return status;
  status = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (status != cudaSuccess) return status;
  cudaFuncAttributes attributes{};
  status = cudaFuncGetAttributes(&attributes, kernel);
  if (status != cudaSuccess) return status;
  status = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - static_cast<int>(attributes.sharedSizeBytes));
  if (status != cudaSuccess) return status;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kernel, kBlock, smem);
}

cudaError_t launch_forward_step(const StepArgs& args, int blocks, int precision, size_t smem, cudaStream_t stream) {
  void* params[] = {const_cast<StepArgs*>(&args)};
  return cudaLaunchCooperativeKernel(forward_kernel(precision), dim3(blocks), dim3(kBlock), params, smem, stream);
}

// Allows the device's largest dynamic shared memory for the kernel (an
// attribute of the function, shared by every solver on the device, so it is
// never lowered to one solver's need) and returns the occupancy at `smem`.
cudaError_t forward_step_max_blocks(int precision, size_t smem, int* blocks_per_sm) {
  const void* kernel = forward_kernel(precision);
  int device = 0, optin = 0;
  cudaError_t status = cudaGetDevice(&device);
  if (status != cudaSuccess) return status;
  status = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (status != cudaSuccess) return status;
  cudaFuncAttributes attributes{};
  status = cudaFuncGetAttributes(&attributes, kernel);
  if (status != cudaSuccess) return status;
  status = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - static_cast<int>(attributes.sharedSizeBytes));
  if (status != cudaSuccess) return status;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kernel, kBlock, smem);
}

cudaError_t launch_apply_inverse(const int* s_off, const int* s_col, const double* s_val, const int* st_off,
                                 const int* st_col, const double* st_val, int rows, const double* rhs, double* work,
                                 double* out, cudaStream_t stream) {
  const int blocks = (rows * 32 + kBlock - 1) / kBlock;
  spmv_kernel<double><<<blocks, kBlock, 0, stream>>>(s_off, s_col, s_val, rhs, work, rows);
  spmv_kernel<double><<<blocks, kBlock, 0, stream>>>(st_off, st_col, st_val, work, out, rows);
  return cudaGetLastError();
}

cudaError_t launch_set_spin_limit(GridBarrier* barrier, unsigned limit, cudaStream_t stream) {
  set_spin_limit_kernel<<<1, 1, 0, stream>>>(barrier, limit);
  return cudaGetLastError();
}

cudaError_t launch_barrier_probe(GridBarrier* barrier, int* status, int* returned, int blocks, int missing, int mode,
                                 cudaStream_t stream) {
  void* params[] = {&barrier, &status, &returned, &missing, &mode};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&barrier_probe_kernel), dim3(blocks), dim3(kBlock),
                                     params, 0, stream);
}

cudaError_t launch_hex_determinants(const float* q, const int* indices, const double* gradients, int ne, double* out,
                                    cudaStream_t stream) {
  const int threads = ne * 8;
  hex_determinants_kernel<<<(threads + 255) / 256, 256, 0, stream>>>(q, indices, gradients, ne, out);
  return cudaGetLastError();
}

}  // namespace pdb200
