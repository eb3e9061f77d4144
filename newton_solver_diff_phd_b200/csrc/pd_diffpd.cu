// The DiffPD pd_eigen forward step (L-BFGS on the projective-dynamics
// objective) as one persistent cooperative launch per step.
//
// Reference: src/newton_solver_diff_phd/_src/solvers/diff_pd/solver.py:65-591
// and kernels.py (the device loop of SolverDiffPD). Each step evaluates the
// explicit state forces on the start-of-step state (gravity, then planar and
// arc penalty contacts with velocity friction), rhs = q + h v + h^2/m (f_ext +
// f_state), and minimises Phi(x) = 1/2 m/h^2 |x - rhs|^2 + E_pd(x) from x = q
// by L-BFGS whose initial inverse Hessian is the exact inverse factor of the
// constant PD matrix A = S^T S (the solver's own factor, built with the
// corotated weight as 2 mu and the volume weight as lambda), a backtracking
// Armijo line search and the masked gradient as fallback, until
// |g| <= rel |m/h^2 rhs_free| + abs.
//
// The whole loop runs on the device in one team of blocks: particle rows are
// owned by the block of their S^T rows, elements are split in contiguous
// ranges, and every scalar of the iteration (dot products, the two-loop
// coefficients, the line-search test) is reduced by every block in the same
// fixed order, so all blocks take the same branches without a serial section.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/pd_b200.h"
#include "pd_forward.cuh"
#include "pd_kernels.h"
#include "solver_state.h"

namespace pdb200 {

constexpr int kDiffPdMaxHistory = 32;
constexpr int kStateForceWidth = 18;
constexpr int kPlanarContact = 0;
constexpr int kArcContact = 1;
constexpr int kDpNotConverged = 1;
constexpr int kDpSingular = 2;
constexpr int kDpLineSearch = 4;
// Slots of one group of the Gram recursion's batched team sums: g.g, s_j.g,
// the new row and column of the Gram matrix and y.s of the newest pair.
constexpr int kDpWideGroup = 3 * kDiffPdMaxHistory + 4;
// Blocks a DiffPD launch may use (the fixed-order reductions' limit).
constexpr int kDpMaxBlocks = 256;

struct DiffPdArgs {
  int n, ne;
  const int* indices;      // [ne][4]
  const double* gradients; // [ne][4][3]
  const int* free_;        // [n]
  const int* inc_offsets;  // [n+1]
  const int* inc_entries;  // element*4 + corner, element-major
  double volume;           // mean rest volume (every element's volume)
  int corotated, volumetric;
  double wc, wv;
  // The solver's factor and its launch plan.
  const double* s_val;
  const double* st_val;
  const int* st_part;
  SpmvPlan plan_s, plan_st;
  int resident, stage_vector, vector_smem_offset;
  // [n][3] float64 vectors.
  double *position, *velocity, *rhs, *x, *trial, *force, *gradient, *direction, *r, *x_last, *g_last, *product;
  double* next_velocity;
  double* s_hist;    // [history][n][3]
  double* y_hist;
  double* energy;    // [ne]
  double* contrib;   // [ne][4][3]
  double* partials;  // [kPartialStride][blocks]
  double* wide;      // [2 kDpWideGroup][blocks]: the Gram recursion's batched sums
  int* status;
  int* counters;     // [0] iterations of the last step, [1] singular flag
  GridBarrier* barrier;
  int history, max_pd_iter, max_ls_iter;
  double abs_tol, rel_tol;
  double mass, inertia, h2m, dt;
  double gravity[3];
  int force_count;
  const int* kinds;        // [force_count]
  const double* params;    // [force_count][18] packed rows
  const void* q_in;
  const void* qd_in;
  const void* f_in;
  void* q_out;
  void* qd_out;
  int state_f64;
};

// kn pow(-min(0, d), p - 1): the penalty of a signed distance d.
__device__ __forceinline__ double dp_penalty(double kn, double d, double p) { return kn * pow(-fmin(0.0, d), p - 1.0); }

// -min(kf, mu fn / (|us| + eps)) us with the tangential velocity us.
__device__ __forceinline__ V3<double> dp_friction(V3<double> v, V3<double> normal, double fn, double kf, double mu) {
  const V3<double> us = v - dot(v, normal) * normal;
  return (-fmin(kf, mu * fn / (length(us) + DBL_EPSILON))) * us;
}

// One packed contact state force at (q, v) (diff_pd/kernels.py:118-152).
__device__ __forceinline__ V3<double> dp_state_force(int kind, const double* c, V3<double> q, V3<double> v) {
  V3<double> force = v3<double>(0.0, 0.0, 0.0);
  if (kind == kPlanarContact) {
    const V3<double> normal = v3<double>(c[0], c[1], c[2]);
    const double fn = dp_penalty(c[5], dot(normal, q) + c[3], c[4]);
    force = fn * normal + dp_friction(v, normal, fn, c[6], c[7]);
  } else if (kind == kArcContact) {
    const V3<double> center = v3<double>(c[0], c[1], c[2]);
    const V3<double> axis = v3<double>(c[3], c[4], c[5]);
    const V3<double> start = v3<double>(c[6], c[7], c[8]);
    const V3<double> aux = v3<double>(c[9], c[10], c[11]);
    const V3<double> local = q - center;
    const V3<double> projected = local - dot(local, axis) * axis;
    const double angle = atan2(dot(projected, aux), dot(projected, start));
    if (0.0 < angle && angle < c[13]) {
      const double fn = dp_penalty(c[15], c[12] - length(projected), c[14]);
      const V3<double> normal = (-1.0 / (length(projected) + DBL_EPSILON)) * projected;
      force = fn * normal + dp_friction(v, normal, fn, c[16], c[17]);
    }
  }
  return force;
}

// Energy and corner forces of element e at the positions `vec`
// (diff_pd/kernels.py:231-271): -Vbar sum_E w_E (F - P_E) g_k, energies in order.
__device__ __forceinline__ void dp_element(const DiffPdArgs& a, int e, const double* vec) {
  double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int i = a.indices[4 * e + k];
    const double* g = a.gradients + (4 * e + k) * 3;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) m[r][c] += vec[3 * i + r] * g[c];
  }
  M3<double> f;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) f.a[r][c] = m[r][c];
  double total = 0.0;
  M3<double> stress_c = zero3<double>(), stress_v = zero3<double>();
  if (a.corotated || a.volumetric) {
    M3<double> u, v;
    V3<double> sigma;
    unsigned_svd(f, u, sigma, v);
    if (a.corotated) {
      const M3<double> difference = f - mul(u, transpose(v));
      double squared = 0.0;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) squared += difference.a[r][c] * difference.a[r][c];
      total += a.wc * 0.5 * squared * a.volume;
      stress_c = a.wc * difference;
    }
    if (a.volumetric) {
      bool singular;
      const V3<double> offset = volume_offset(sigma, singular);
      if (singular) atomicOr(a.counters + 1, 1);
      const M3<double> difference = f - udvt(u, sigma + offset, v);
      double squared = 0.0;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) squared += difference.a[r][c] * difference.a[r][c];
      total += a.wv * 0.5 * squared * a.volume;
      stress_v = a.wv * difference;
    }
  }
  a.energy[e] = total;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double* g = a.gradients + (4 * e + k) * 3;
    const V3<double> gk = v3<double>(g[0], g[1], g[2]);
    const V3<double> c = (-a.volume) * mul(stress_c, gk) + (-a.volume) * mul(stress_v, gk);
    double* out = a.contrib + (4 * e + k) * 3;
    out[0] = c.x;
    out[1] = c.y;
    out[2] = c.z;
  }
}

// Team-wide sums of `count` (<= 4) per-block values: this block's values go
// to its partial slots, a team barrier, then every block sums the slots of
// all blocks in the same fixed order into `out` (shared memory). Slots
// alternate between two groups: a block that runs ahead writes the next
// group while slower blocks still read this one, and the group it would
// overwrite next was read by everyone before the barrier in between.
__device__ __forceinline__ bool dp_team_sum(const DiffPdArgs& a, Team team, int& sequence, const double* values,
                                            int count, double* out, double* scratch) {
  const int base = (sequence & 1) * 4;
  ++sequence;
  if (threadIdx.x == 0) {
    for (int c = 0; c < count; ++c) a.partials[(base + c) * team.size + team.rank] = values[c];
  }
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  reduce_partials(a.partials, base, count, team.size, out, scratch);
  return true;
}


// Trial evaluation: element energies and forces at a.trial, the fixed-order
// gather of the forces into the own rows, and Phi(trial) reduced over the
// team (own-row inertia terms plus own-range element energies).
__device__ __forceinline__ bool dp_evaluate(const DiffPdArgs& a, Team team, int e0, int e1, int r0, int r1,
                                            int& sequence, double* objective, double* s_out, double* scratch) {
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) dp_element(a, e, a.trial);
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  double residual = 0.0, energy = 0.0;
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    V3<double> total = v3<double>(0.0, 0.0, 0.0);
    for (int k = a.inc_offsets[i]; k < a.inc_offsets[i + 1]; ++k) total = total + load3d(a.contrib, a.inc_entries[k]);
    store3(a.force, i, total);
    const V3<double> difference = load3d(a.trial, i) - load3d(a.rhs, i);
    residual += dot(difference, a.inertia * difference);
  }
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) energy += a.energy[e];
  double values[2] = {block_sum(residual, scratch), block_sum(energy, scratch)};
  if (!dp_team_sum(a, team, sequence, values, 2, s_out, scratch)) return false;
  *objective = 0.5 * s_out[0] + s_out[1];
  return true;
}

// x = A^{-1} r over the team: y = S r on the S rows, then S^T y on the own rows.
template <typename TV>
__device__ __forceinline__ bool dp_apply_inverse(const DiffPdArgs& a, Team team, const char* dyn_smem,
                                                 double* vector_smem) {
  const TV* s_values = reinterpret_cast<const TV*>(a.s_val);
  const TV* st_values = reinterpret_cast<const TV*>(a.st_val);
  {
    const double* in = a.r;
    if (a.stage_vector) {
      stage_for(a.plan_s, team.rank, a.r, vector_smem, a.n);
      in = vector_smem;
    }
    spmv_block<TV>(a.plan_s, s_values, a.resident != 0, dyn_smem, in, a.product, team.rank);
  }
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  const double* in = a.product;
  if (a.stage_vector) {
    stage_for(a.plan_st, team.rank, a.product, vector_smem, a.n);
    in = vector_smem;
  }
  spmv_block<TV>(a.plan_st, st_values, a.resident != 0, dyn_smem, in, a.direction, team.rank);
  __syncthreads();
  return true;
}

// What the start of a step leaves for the L-BFGS loop: this block's rows and
// elements, the stop threshold, Phi(q) and whether q met a singular F.
struct DpStart {
  int r0, r1, e0, e1;
  double threshold, objective;
  bool singular;
};

// begin_step (solver.py:689-720): the state forces of the start-of-step state
// and rhs, the stop threshold rel |(m/h^2 rhs) on the free rows| + abs, Phi at
// x = q, and x and the masked gradient on the own rows. Returns false when a
// team barrier gave up.
__device__ __forceinline__ bool dp_begin_step(const DiffPdArgs& a, const Team team, char* dyn_smem, int& sequence,
                                              double* s_out, double* s_scratch, DpStart* start) {
  const int n = a.n;
  const int gtid = team.rank * blockDim.x + threadIdx.x;
  const int gthreads = team.size * blockDim.x;
  const double dt = a.dt;
  for (int i = gtid; i < n; i += gthreads) {
    const int f64 = a.state_f64;
    V3<double> q, v, f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      q[c] = state_load(a.q_in, f64, 3 * i + c);
      v[c] = state_load(a.qd_in, f64, 3 * i + c);
      f[c] = state_load(a.f_in, f64, 3 * i + c);
    }
    store3(a.position, i, q);
    store3(a.velocity, i, v);
    V3<double> force = v3<double>(a.mass * a.gravity[0], a.mass * a.gravity[1], a.mass * a.gravity[2]);
    for (int k = 0; k < a.force_count; ++k)
      force = force + dp_state_force(a.kinds[k], a.params + kStateForceWidth * k, q, v);
    store3(a.rhs, i, q + dt * v + a.h2m * f + a.h2m * force);
    store3(a.trial, i, q);
  }
  if (gtid == 0) {
    a.counters[0] = 0;
    a.counters[1] = 0;
  }
  // rhs and the first trial were written by particle index across the team;
  // the threshold reads rhs by owned row and the first evaluation reads every
  // corner of its elements.
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  if (a.resident) {
    load_slice<double>(a.plan_s, a.s_val, dyn_smem, team.rank);
    load_slice<double>(a.plan_st, a.st_val, dyn_smem, team.rank);
  }
  const int r0 = a.st_part[team.rank], r1 = a.st_part[team.rank + 1];
  start->r0 = r0;
  start->r1 = r1;
  team_range(a.ne, team, start->e0, start->e1);
  {
    double partial = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      if (a.free_[i]) {
        const V3<double> value = a.inertia * load3d(a.rhs, i);
        partial += dot(value, value);
      }
    }
    const double values[1] = {block_sum(partial, s_scratch)};
    if (!dp_team_sum(a, team, sequence, values, 1, s_out, s_scratch)) return false;
    start->threshold = a.rel_tol * sqrt(s_out[0]) + a.abs_tol;
  }
  if (!dp_evaluate(a, team, start->e0, start->e1, r0, r1, sequence, &start->objective, s_out, s_scratch)) return false;
  start->singular = *reinterpret_cast<volatile int*>(a.counters + 1) != 0;
  if (start->singular) atomicOr(a.status, kDpSingular);
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const V3<double> x = load3d(a.trial, i);
    store3(a.x, i, x);
    V3<double> g = a.inertia * (x - load3d(a.rhs, i)) - load3d(a.force, i);
    if (!a.free_[i]) g = v3<double>(0.0, 0.0, 0.0);
    store3(a.gradient, i, g);
  }
  return true;
}

// Backtracking Armijo line search along -direction from x (the last trial is
// accepted untested): trial = x - step d, halved until
// Phi(trial) < Phi(x) - 1e-4 step slope + eps or a singular F stops it.
__device__ __forceinline__ bool dp_line_search(const DiffPdArgs& a, const Team team, const DpStart& start,
                                               int& sequence, double objective, double slope,
                                               double* trial_objective, bool* singular, bool* failed, double* s_out,
                                               double* s_scratch) {
  double step = 1.0;
  *failed = false;
  for (int evaluations = 1;; ++evaluations) {
    for (int i = start.r0 + threadIdx.x; i < start.r1; i += blockDim.x)
      store3(a.trial, i, load3d(a.x, i) - step * load3d(a.direction, i));
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    if (!dp_evaluate(a, team, start.e0, start.e1, start.r0, start.r1, sequence, trial_objective, s_out, s_scratch))
      return false;
    *singular = *reinterpret_cast<volatile int*>(a.counters + 1) != 0;
    if (*singular) break;
    if (evaluations > a.max_ls_iter) {
      *failed = true;
      break;
    }
    const double bound = objective - 1.0e-4 * step * slope;
    if (!isnan(*trial_objective) && *trial_objective < bound + DBL_EPSILON) break;
    step *= 0.5;
  }
  return true;
}

// write_state: the float64 results and the rounded state on the own rows.
__device__ __forceinline__ void dp_write_state(const DiffPdArgs& a, const Team team, const DpStart& start,
                                               int iterations) {
  const double dt = a.dt;
  for (int i = start.r0 + threadIdx.x; i < start.r1; i += blockDim.x) {
    const V3<double> x = load3d(a.x, i);
    const V3<double> v = (1.0 / dt) * (x - load3d(a.position, i));
    store3(a.next_velocity, i, v);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      state_store(a.q_out, a.state_f64, 3 * i + c, x[c]);
      state_store(a.qd_out, a.state_f64, 3 * i + c, (x[c] - a.position[3 * i + c]) / dt);
    }
  }
  if (team.rank == 0 && threadIdx.x == 0) a.counters[0] = iterations;
}

// One DiffPD step by one team (solver.py:689-786 with the device loop of
// kernels.py), the two-loop recursion as the reference writes it: one team
// sum per pair in each loop. Returns false when a team barrier gave up.
__device__ bool diffpd_step_body(const DiffPdArgs& a, const Team team, char* dyn_smem) {
  __shared__ double s_scratch[kBlock];
  __shared__ double s_out[64];
  __shared__ double s_rho[kDiffPdMaxHistory];
  __shared__ double s_alpha[kDiffPdMaxHistory];
  const int n = a.n;
  const int gtid = team.rank * blockDim.x + threadIdx.x;
  int sequence = 0;
  DpStart start;
  if (!dp_begin_step(a, team, dyn_smem, sequence, s_out, s_scratch, &start)) return false;
  double* vector_smem = reinterpret_cast<double*>(dyn_smem + a.vector_smem_offset);
  const int r0 = start.r0, r1 = start.r1;
  double objective = start.objective;
  bool singular = start.singular;
  int iterations = 0;
  const int m = a.history;
  int pairs = 0, newest = m - 1;
  while (!singular) {
    // ---- History push (s, y) = (x - x_last, g - g_last), rho = 1 / (y . s).
    const bool store = iterations > 0;
    if (store) {
      newest = (newest + 1) % m;
      pairs = min(pairs + 1, m);
    }
    {
      double ys = 0.0;
      double* s_new = a.s_hist + static_cast<size_t>(newest) * 3 * n;
      double* y_new = a.y_hist + static_cast<size_t>(newest) * 3 * n;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const V3<double> x = load3d(a.x, i);
        const V3<double> g = load3d(a.gradient, i);
        if (store) {
          const V3<double> step = x - load3d(a.x_last, i);
          const V3<double> change = g - load3d(a.g_last, i);
          store3(s_new, i, step);
          store3(y_new, i, change);
          ys += dot(change, step);
        }
        store3(a.x_last, i, x);
        store3(a.g_last, i, g);
        store3(a.r, i, g);
      }
      if (store) {
        const double values[1] = {block_sum(ys, s_scratch)};
        if (!dp_team_sum(a, team, sequence, values, 1, s_out, s_scratch)) return false;
        if (threadIdx.x == 0) s_rho[newest] = 1.0 / s_out[0];
      }
    }
    // ---- Two-loop recursion, newest to oldest (alpha), A^{-1}, oldest to newest.
    for (int age = 0; age < pairs; ++age) {
      const int slot = (newest - age + m) % m;
      const double* s_k = a.s_hist + static_cast<size_t>(slot) * 3 * n;
      const double* y_k = a.y_hist + static_cast<size_t>(slot) * 3 * n;
      double partial = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) partial += dot(load3d(s_k, i), load3d(a.r, i));
      const double values[1] = {block_sum(partial, s_scratch)};
      if (!dp_team_sum(a, team, sequence, values, 1, s_out, s_scratch)) return false;
      const double alpha = s_rho[slot] * s_out[0];
      if (threadIdx.x == 0) s_alpha[slot] = alpha;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) store3(a.r, i, load3d(a.r, i) - alpha * load3d(y_k, i));
    }
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    if (!dp_apply_inverse<double>(a, team, dyn_smem, vector_smem)) return false;
    for (int age = pairs - 1; age >= 0; --age) {
      const int slot = (newest - age + m) % m;
      const double* s_k = a.s_hist + static_cast<size_t>(slot) * 3 * n;
      const double* y_k = a.y_hist + static_cast<size_t>(slot) * 3 * n;
      double partial = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) partial += dot(load3d(y_k, i), load3d(a.direction, i));
      const double values[1] = {block_sum(partial, s_scratch)};
      if (!dp_team_sum(a, team, sequence, values, 1, s_out, s_scratch)) return false;
      const double coefficient = s_alpha[slot] - s_rho[slot] * s_out[0];
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x)
        store3(a.direction, i, load3d(a.direction, i) + coefficient * load3d(s_k, i));
    }
    // ---- Descent check: a direction that does not descend falls back to the masked gradient.
    double slope;
    {
      double dg = 0.0, gg = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const V3<double> g = load3d(a.gradient, i);
        dg += dot(load3d(a.direction, i), g);
        gg += dot(g, g);
      }
      const double values[2] = {block_sum(dg, s_scratch), block_sum(gg, s_scratch)};
      if (!dp_team_sum(a, team, sequence, values, 2, s_out, s_scratch)) return false;
      slope = s_out[0];
      if (!(slope > 0.0)) {
        slope = s_out[1];
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x)
          store3(a.direction, i, a.free_[i] ? load3d(a.gradient, i) : v3<double>(0.0, 0.0, 0.0));
      }
    }
    double trial_objective = objective;
    bool failed = false;
    if (!dp_line_search(a, team, start, sequence, objective, slope, &trial_objective, &singular, &failed, s_out,
                        s_scratch))
      return false;
    // ---- Accept the trial; gradient and its norm.
    objective = trial_objective;
    double gg = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const V3<double> x = load3d(a.trial, i);
      store3(a.x, i, x);
      V3<double> g = a.inertia * (x - load3d(a.rhs, i)) - load3d(a.force, i);
      if (!a.free_[i]) g = v3<double>(0.0, 0.0, 0.0);
      store3(a.gradient, i, g);
      gg += dot(g, g);
    }
    const double values[1] = {block_sum(gg, s_scratch)};
    if (!dp_team_sum(a, team, sequence, values, 1, s_out, s_scratch)) return false;
    if (failed && gtid == 0) atomicOr(a.status, kDpLineSearch);
    iterations += 1;
    if (singular) {
      if (gtid == 0) atomicOr(a.status, kDpSingular);
      break;
    }
    if (sqrt(s_out[0]) <= start.threshold) break;
    if (iterations >= a.max_pd_iter) {
      if (gtid == 0) atomicOr(a.status, kDpNotConverged);
      break;
    }
  }
  dp_write_state(a, team, start, iterations);
  return true;
}

// Team-wide sums of `count` (<= kDpWideGroup) dot products over the owned
// rows, dot_of(k, i) being product k's term of row i: warp w of every block
// takes products w, w + 8, ..., its lanes the rows in a fixed stride and a
// fixed shuffle tree, lane 0 writes the block's partial into the wide slots;
// then a team barrier and every block sums the slots of all blocks in the
// same fixed order into `out`. Groups alternate as in dp_team_sum.
template <typename DotOf>
__device__ __forceinline__ bool dp_wide_sums(const DiffPdArgs& a, Team team, int& sequence, int count, int r0, int r1,
                                             DotOf dot_of, double* out, double* scratch) {
  const int base = (sequence & 1) * kDpWideGroup;
  ++sequence;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  for (int k = warp; k < count; k += kBlock / 32) {
    double sum = 0.0;
    for (int i = r0 + lane; i < r1; i += 32) sum += dot_of(k, i);
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, offset);
    if (lane == 0) a.wide[(base + k) * team.size + team.rank] = sum;
  }
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  reduce_partials(a.wide, base, count, team.size, out, scratch);
  return true;
}

// One DiffPD step by one team with the two-loop recursion in Gram form. The
// block keeps G[i][j] = s_i . y_j of the stored pairs and sg_i = s_i . g in
// shared memory; the first loop's s_i . r_i = sg_i - sum_{j newer} alpha_j
// G[i][j] and the second loop's y_i . d_i = y_i . d_0 + sum_{j older} c_j
// G[j][i] are scalar recurrences every block runs in the same order, r and the
// direction are formed on the own rows in the reference's order (newest
// first for r, oldest first for d), and the slope d . g is d_0 . g +
// sum_j c_j sg_j. An iteration takes two batched team sums around the
// inverse product (y_j . d_0, d_0 . g, g . g before the line search; g . g,
// sg_j and the new Gram row and column after it) instead of one per pair and
// loop. Same status bits, history and line search as diffpd_step_body; the
// dot products are rounded in another order.
__device__ bool diffpd_gram_body(const DiffPdArgs& a, const Team team, char* dyn_smem) {
  __shared__ double s_scratch[kBlock];
  __shared__ double s_out[kDpWideGroup];
  __shared__ double s_gram[kDiffPdMaxHistory * kDiffPdMaxHistory];
  __shared__ double s_rho[kDiffPdMaxHistory];
  __shared__ double s_alpha[kDiffPdMaxHistory];
  __shared__ double s_coef[kDiffPdMaxHistory];
  __shared__ double s_sg[kDiffPdMaxHistory];
  __shared__ double s_scalars[2];  // slope, g . g
  const int n = a.n;
  const int gtid = team.rank * blockDim.x + threadIdx.x;
  int sequence = 0;
  DpStart start;
  if (!dp_begin_step(a, team, dyn_smem, sequence, s_out, s_scratch, &start)) return false;
  double* vector_smem = reinterpret_cast<double*>(dyn_smem + a.vector_smem_offset);
  const int r0 = start.r0, r1 = start.r1;
  double objective = start.objective;
  bool singular = start.singular;
  int iterations = 0;
  const int m = a.history;
  int pairs = 0, newest = m - 1;
  // Ring slot of the pair of a given age (0 = newest).
  auto slot_of = [&](int age) { return (newest - age + m) % m; };
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    store3(a.x_last, i, load3d(a.x, i));
    store3(a.g_last, i, load3d(a.gradient, i));
  }
  while (!singular) {
    // ---- First loop: alpha_i = rho_i (sg_i - sum_{j newer} alpha_j G[i][j]), newest first.
    if (threadIdx.x == 0) {
      for (int age = 0; age < pairs; ++age) {
        const int i = slot_of(age);
        double sr = s_sg[i];
        for (int newer = 0; newer < age; ++newer) {
          const int j = slot_of(newer);
          sr = sr - s_alpha[j] * s_gram[i * kDiffPdMaxHistory + j];
        }
        s_alpha[i] = s_rho[i] * sr;
      }
    }
    __syncthreads();
    // ---- r = g - alpha_j y_j, newest first, then d_0 = A^{-1} r.
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      V3<double> r = load3d(a.gradient, i);
      for (int age = 0; age < pairs; ++age) {
        const int j = slot_of(age);
        r = r - s_alpha[j] * load3d(a.y_hist + static_cast<size_t>(j) * 3 * n, i);
      }
      store3(a.r, i, r);
    }
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    if (!dp_apply_inverse<double>(a, team, dyn_smem, vector_smem)) return false;
    // ---- y_j . d_0 by age, d_0 . g and g . g in one team sum.
    {
      auto dot_of = [&](int k, int i) {
        const V3<double> d0 = load3d(a.direction, i);
        if (k < pairs) return dot(load3d(a.y_hist + static_cast<size_t>(slot_of(k)) * 3 * n, i), d0);
        const V3<double> g = load3d(a.gradient, i);
        return k == pairs ? dot(d0, g) : dot(g, g);
      };
      if (!dp_wide_sums(a, team, sequence, pairs + 2, r0, r1, dot_of, s_out, s_scratch)) return false;
    }
    // ---- Second loop: c_i = alpha_i - rho_i (y_i . d_0 + sum_{j older} c_j G[j][i]), oldest first;
    // slope = d_0 . g + sum_j c_j sg_j, oldest first.
    if (threadIdx.x == 0) {
      for (int age = pairs - 1; age >= 0; --age) {
        const int i = slot_of(age);
        double yd = s_out[age];
        for (int older = pairs - 1; older > age; --older) {
          const int j = slot_of(older);
          yd = yd + s_coef[j] * s_gram[j * kDiffPdMaxHistory + i];
        }
        s_coef[i] = s_alpha[i] - s_rho[i] * yd;
      }
      double slope = s_out[pairs];
      for (int age = pairs - 1; age >= 0; --age) slope = slope + s_coef[slot_of(age)] * s_sg[slot_of(age)];
      s_scalars[0] = slope;
      s_scalars[1] = s_out[pairs + 1];
    }
    __syncthreads();
    // ---- Direction d_0 + c_j s_j (oldest first), or the masked gradient when it does not descend.
    double slope = s_scalars[0];
    const bool descends = slope > 0.0;
    if (!descends) slope = s_scalars[1];
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      V3<double> d;
      if (descends) {
        d = load3d(a.direction, i);
        for (int age = pairs - 1; age >= 0; --age) {
          const int j = slot_of(age);
          d = d + s_coef[j] * load3d(a.s_hist + static_cast<size_t>(j) * 3 * n, i);
        }
      } else {
        d = a.free_[i] ? load3d(a.gradient, i) : v3<double>(0.0, 0.0, 0.0);
      }
      store3(a.direction, i, d);
    }
    double trial_objective = objective;
    bool failed = false;
    if (!dp_line_search(a, team, start, sequence, objective, slope, &trial_objective, &singular, &failed, s_out,
                        s_scratch))
      return false;
    // ---- Accept the trial; gradient, history push (s, y) = (x - x_last, g - g_last).
    objective = trial_objective;
    newest = (newest + 1) % m;
    pairs = min(pairs + 1, m);
    {
      double* s_new = a.s_hist + static_cast<size_t>(newest) * 3 * n;
      double* y_new = a.y_hist + static_cast<size_t>(newest) * 3 * n;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const V3<double> x = load3d(a.trial, i);
        store3(a.x, i, x);
        V3<double> g = a.inertia * (x - load3d(a.rhs, i)) - load3d(a.force, i);
        if (!a.free_[i]) g = v3<double>(0.0, 0.0, 0.0);
        store3(a.gradient, i, g);
        store3(s_new, i, x - load3d(a.x_last, i));
        store3(y_new, i, g - load3d(a.g_last, i));
        store3(a.x_last, i, x);
        store3(a.g_last, i, g);
      }
      // The products read rows that other threads of this block wrote.
      __syncthreads();
      // Products: 0 g . g; 1 + age: s_age . g; then for every older age the new Gram row
      // s_new . y_age and column s_age . y_new; last y_new . s_new.
      const int older = pairs - 1;
      auto dot_of = [&](int k, int i) {
        const V3<double> g = load3d(a.gradient, i);
        if (k == 0) return dot(g, g);
        if (k <= pairs) return dot(load3d(a.s_hist + static_cast<size_t>(slot_of(k - 1)) * 3 * n, i), g);
        if (k <= pairs + older) {
          const int j = slot_of(k - pairs);
          return dot(load3d(s_new, i), load3d(a.y_hist + static_cast<size_t>(j) * 3 * n, i));
        }
        if (k <= pairs + 2 * older) {
          const int j = slot_of(k - pairs - older);
          return dot(load3d(a.s_hist + static_cast<size_t>(j) * 3 * n, i), load3d(y_new, i));
        }
        return dot(load3d(y_new, i), load3d(s_new, i));
      };
      if (!dp_wide_sums(a, team, sequence, 3 * pairs, r0, r1, dot_of, s_out, s_scratch)) return false;
      if (threadIdx.x == 0) {
        for (int age = 0; age < pairs; ++age) s_sg[slot_of(age)] = s_out[1 + age];
        for (int age = 1; age <= older; ++age) {
          const int j = slot_of(age);
          s_gram[newest * kDiffPdMaxHistory + j] = s_out[pairs + age];
          s_gram[j * kDiffPdMaxHistory + newest] = s_out[pairs + older + age];
        }
        const double ys = s_out[3 * pairs - 1];
        s_gram[newest * kDiffPdMaxHistory + newest] = ys;
        s_rho[newest] = 1.0 / ys;
      }
    }
    const double gg = s_out[0];
    __syncthreads();
    if (failed && gtid == 0) atomicOr(a.status, kDpLineSearch);
    iterations += 1;
    if (singular) {
      if (gtid == 0) atomicOr(a.status, kDpSingular);
      break;
    }
    if (sqrt(gg) <= start.threshold) break;
    if (iterations >= a.max_pd_iter) {
      if (gtid == 0) atomicOr(a.status, kDpNotConverged);
      break;
    }
  }
  dp_write_state(a, team, start, iterations);
  return true;
}

__global__ void __launch_bounds__(kBlock) diffpd_step_kernel(const DiffPdArgs a) {
  extern __shared__ __align__(16) char dyn_smem[];
  diffpd_step_body(a, Team{static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x)}, dyn_smem);
}

__global__ void __launch_bounds__(kBlock) diffpd_gram_kernel(const DiffPdArgs a) {
  extern __shared__ __align__(16) char dyn_smem[];
  diffpd_gram_body(a, Team{static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x)}, dyn_smem);
}

}  // namespace pdb200

// ---------------------------------------------------------------------------
// Host entry points.

using pdb200::DiffPdArgs;

namespace {

int dp_fail(int code, const std::string& message) { return pd_set_error(code, message); }

// Doubles between consecutive DiffPD vectors: 3n rounded up to 32 (256 bytes).
size_t dp_vector_stride(int n) { return (static_cast<size_t>(3) * n + 31) / 32 * 32; }

}  // namespace

extern "C" {

int pd_diffpd_set_state_forces(PdSolver* s, int32_t count, const int32_t* kinds, const double* parameters) {
  if (s == nullptr || count < 0 || (count > 0 && (kinds == nullptr || parameters == nullptr)))
    return dp_fail(PD_ERR_INVALID, "null argument or negative count");
  for (int k = 0; k < count; ++k) {
    if (kinds[k] != pdb200::kPlanarContact && kinds[k] != pdb200::kArcContact)
      return dp_fail(PD_ERR_INVALID, "state force kinds are 'planar_contact' and 'arc_contact'");
    for (int c = 0; c < pdb200::kStateForceWidth; ++c)
      if (!std::isfinite(parameters[pdb200::kStateForceWidth * k + c]))
        return dp_fail(PD_ERR_INVALID, "state force parameters must be finite");
  }
  PD_CUDA(cudaSetDevice(s->device));
  std::vector<int32_t> k(kinds, kinds + count);
  std::vector<double> p(parameters, parameters + static_cast<size_t>(pdb200::kStateForceWidth) * count);
  if (k.empty()) k.push_back(0);
  if (p.empty()) p.assign(pdb200::kStateForceWidth, 0.0);
  PD_CUDA(s->dp_kinds.upload(k));
  PD_CUDA(s->dp_params.upload(p));
  s->dp_force_count = count;
  return PD_OK;
}

int pd_diffpd_step(PdSolver* s, const PdDiffPdOptions* o, const void* q, const void* qd, const void* f,
                   const double gravity[3], double dt, void* q_out, void* qd_out, void* stream) {
  if (s == nullptr || o == nullptr || q == nullptr || qd == nullptr || f == nullptr || gravity == nullptr ||
      q_out == nullptr || qd_out == nullptr)
    return dp_fail(PD_ERR_INVALID, "null argument");
  if (s->hex || s->corners != 4) return dp_fail(PD_ERR_UNSUPPORTED, "SolverDiffPD requires tetrahedral soft bodies");
  if (!std::isfinite(dt) || dt <= 0.0) return dp_fail(PD_ERR_INVALID, "dt must be finite and positive");
  if (q == q_out || qd == qd_out || q == qd_out || qd == q_out)
    return dp_fail(PD_ERR_INVALID, "DiffPD requires distinct input and output states");
  if (o->max_pd_iter < 1 || o->max_ls_iter < 1 || o->history < 2 || o->history > pdb200::kDiffPdMaxHistory)
    return dp_fail(PD_ERR_INVALID, "max_pd_iter >= 1, max_ls_iter >= 1 and bfgs_history_size in [2, 32] are required");
  if (!(o->abs_tol >= 0.0) || !(o->rel_tol >= 0.0) || !std::isfinite(o->abs_tol) || !std::isfinite(o->rel_tol))
    return dp_fail(PD_ERR_INVALID, "abs_tol and rel_tol must be finite and nonnegative");
  if (o->recursion != PD_DIFFPD_TWO_LOOP && o->recursion != PD_DIFFPD_GRAM)
    return dp_fail(PD_ERR_INVALID, "recursion must be PD_DIFFPD_TWO_LOOP or PD_DIFFPD_GRAM");
  if (!s->built || s->stale || s->built_dt != dt)
    return dp_fail(PD_ERR_STATE, "SolverDiffPD must rebuild its factor (pd_build) for this dt and model");
  PD_CUDA(cudaSetDevice(s->device));
  if (int status = pd_ensure_plan(s)) return status;
  if (s->blocks > pdb200::kDpMaxBlocks) return dp_fail(PD_ERR_INVALID, "SolverDiffPD launches at most 256 blocks");
  // Every [n][3] vector starts on a 256-byte boundary: the products stage
  // their input vector into shared memory with 16-byte loads, and a stride of
  // 3n doubles would leave odd slots only 8-byte aligned.
  const size_t vec = dp_vector_stride(s->n);
  constexpr int kVectors = 13;
  // After the vectors: the wide partial slots of the Gram recursion.
  const size_t wide = static_cast<size_t>(2) * pdb200::kDpWideGroup * pdb200::kDpMaxBlocks;
  if (s->dp_vectors.ptr == nullptr) {
    PD_CUDA(s->dp_vectors.allocate((kVectors * vec + wide) * sizeof(double)));
    PD_CUDA(s->dp_energy.allocate(static_cast<size_t>(s->ne) * sizeof(double)));
    PD_CUDA(s->dp_counters.allocate(4 * sizeof(int)));
  }
  if (s->dp_history < o->history) {
    PD_CUDA(s->dp_hist.allocate(2 * static_cast<size_t>(o->history) * vec * sizeof(double)));
    s->dp_history = o->history;
  }
  if (s->dp_kinds.ptr == nullptr) {
    if (int status = pd_diffpd_set_state_forces(s, 0, nullptr, nullptr)) return status;
  }
  DiffPdArgs a{};
  a.n = s->n;
  a.ne = s->ne;
  a.indices = s->d_indices.as<int>();
  a.gradients = s->d_gradients.as<double>();
  a.free_ = s->d_free.as<int>();
  a.inc_offsets = s->d_inc_offsets.as<int>();
  a.inc_entries = s->d_inc_entries.as<int>();
  a.volume = s->mean_volume;
  a.corotated = o->use_corotated ? 1 : 0;
  a.volumetric = o->use_volume ? 1 : 0;
  a.wc = o->corotated_weight;
  a.wv = o->volume_weight;
  a.s_val = s->d_s_val.as<double>();
  a.st_val = s->d_st_val.as<double>();
  a.st_part = s->d_st_part.as<int>();
  a.plan_s = s->plan_s;
  a.plan_st = s->plan_st;
  a.resident = s->resident;
  a.stage_vector = s->stage_vector;
  a.vector_smem_offset = s->vector_smem_offset;
  double* v = s->dp_vectors.as<double>();
  double** slots[kVectors] = {&a.position, &a.velocity, &a.rhs,    &a.x,      &a.trial,  &a.force,        &a.gradient,
                              &a.direction, &a.r,       &a.x_last, &a.g_last, &a.product, &a.next_velocity};
  for (int k = 0; k < kVectors; ++k) *slots[k] = v + k * vec;
  a.wide = v + kVectors * vec;
  a.s_hist = s->dp_hist.as<double>();
  a.y_hist = a.s_hist + static_cast<size_t>(o->history) * vec;
  a.energy = s->dp_energy.as<double>();
  a.contrib = s->d_contrib.as<double>();
  a.partials = s->d_partials.as<double>();
  a.status = s->d_status.as<int>();
  a.counters = s->dp_counters.as<int>();
  a.barrier = s->d_barrier.as<pdb200::GridBarrier>();
  a.history = o->history;
  a.max_pd_iter = o->max_pd_iter;
  a.max_ls_iter = o->max_ls_iter;
  a.abs_tol = o->abs_tol;
  a.rel_tol = o->rel_tol;
  a.mass = s->mass;
  a.inertia = s->mass / (dt * dt);
  a.h2m = dt * dt / s->mass;
  a.dt = dt;
  for (int c = 0; c < 3; ++c) a.gravity[c] = gravity[c];
  a.force_count = s->dp_force_count;
  a.kinds = s->dp_kinds.as<int>();
  a.params = s->dp_params.as<double>();
  a.q_in = q;
  a.qd_in = qd;
  a.f_in = f;
  a.q_out = q_out;
  a.qd_out = qd_out;
  a.state_f64 = s->options.state_precision;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PD_CUDA(cudaMemsetAsync(s->d_barrier.ptr, 0, sizeof(pdb200::GridBarrier), st));
  if (s->spin_limit != 0u) PD_CUDA(pdb200::launch_set_spin_limit(a.barrier, s->spin_limit, st));
  const void* kernel = o->recursion == PD_DIFFPD_GRAM ? reinterpret_cast<const void*>(&pdb200::diffpd_gram_kernel)
                                                      : reinterpret_cast<const void*>(&pdb200::diffpd_step_kernel);
  {
    int optin = 0;
    PD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
    cudaFuncAttributes attributes{};
    PD_CUDA(cudaFuncGetAttributes(&attributes, kernel));
    PD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 optin - static_cast<int>(attributes.sharedSizeBytes)));
  }
  void* params[] = {&a};
  PD_CUDA(cudaLaunchCooperativeKernel(kernel, dim3(s->blocks), dim3(pdb200::kBlock), params, s->smem, st));
  return PD_OK;
}

int pd_diffpd_results(PdSolver* s, double** positions, double** velocities, int32_t* iterations, void* stream) {
  if (s == nullptr) return dp_fail(PD_ERR_INVALID, "null solver");
  if (s->dp_vectors.ptr == nullptr) return dp_fail(PD_ERR_STATE, "no DiffPD step has run");
  const size_t vec = dp_vector_stride(s->n);
  if (positions) *positions = s->dp_vectors.as<double>() + 3 * vec;
  if (velocities) *velocities = s->dp_vectors.as<double>() + 12 * vec;
  if (iterations) {
    PD_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int value = 0;
    PD_CUDA(cudaMemcpyAsync(&value, s->dp_counters.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    *iterations = value;
  }
  return PD_OK;
}

}  // extern "C"
