// Persistent backward-step kernel: the reference DiffPhD adjoint of one step
// (Adjoint.backward, src/newton_solver_diff_phd/_src/solvers/diff_phd/adjoint.py:1088-1259),
// extended to Hex8 cells (eight Gauss samples, sample weight w Vbar/8) and to
// an exact mode whose K uses per-element weights.
//
//   prologue  seed g = dL/dq+ + dL/dv+/h (:70-81), local Jacobians dP/dF at x+
//             (9 directional derivatives per sample, :92-137), ||g||^2 partials
//   loop      A1 K mu per element -> A2 gather + g -> A3 S -> A4 S^T, Dirichlet
//             zeroing, non-finite scrub, Anderson history -> serial clip / Anderson
//             -> A5 Anderson apply -> serial clip, stopping rule (:184-321, :927-964)
//   epilogue  routing guard (:226-261), state gradients (:474-490), Dirichlet
//             coupling and gradients (:493-553), material and activation gradients
//             with the parameter guard (:556-659).
// The norm clip of 1e6 is rare; when it triggers, an extra phase rescales the
// affected vector and recomputes its partials, so the fast path stays at five
// grid barriers per iteration.
#include <cuda_runtime.h>

#include "pd_forward.cuh"
#include "pd_team.cuh"
#include "pd_kernels.h"

namespace pdb200 {

constexpr double kClipNorm = 1.0e6;

template <typename TL>
__device__ __forceinline__ TL* jacobian_ptr(const AdjointArgs& b);
template <>
__device__ __forceinline__ double* jacobian_ptr<double>(const AdjointArgs& b) { return b.jac64; }
template <>
__device__ __forceinline__ float* jacobian_ptr<float>(const AdjointArgs& b) { return b.jac32; }

// Directional derivative of the projection stress w.r.t. F, applied to e_r e_c^T,
// for the nine flattened directions c9 = r + 3 c (Eigen column-major order).
template <typename TL>
__device__ void sample_jacobian(const AdjointArgs& b, int e, const M3<TL>& f, TL* out /* [9][9] row-major per direction */) {
  M3<TL> u, v;
  V3<TL> sigma;
  unsigned_svd(f, u, sigma, v);
  const bool exact = b.exact != 0;
  const TL wc = static_cast<TL>(exact ? b.wc[e] : b.jwc);
  const TL wv = static_cast<TL>(exact ? b.wv[e] : b.jwv);
  const TL wn = static_cast<TL>(exact ? b.wn[e] : b.jwn);
  const TL mu = static_cast<TL>(b.nh_mu), lame = static_cast<TL>(b.nh_lame), penalty = static_cast<TL>(b.nh_penalty);
  V3<TL> offset = v3<TL>(TL(0), TL(0), TL(0));
  V3<TL> stretches = offset;
  if (b.material == 0) {
    bool singular;
    offset = volume_offset(sigma, singular);
  } else {
    stretches = nh_prox_stretches(sigma, mu, lame, penalty);
  }
  const TL wm = b.has_muscles ? static_cast<TL>(b.wm[e]) : TL(0);
  V3<TL> m = v3<TL>(TL(0), TL(0), TL(0));
  TL target = TL(0);
  if (wm != TL(0)) {
    m = load3<TL>(b.mdir, e);
    target = b.activations != nullptr ? static_cast<TL>(1.0 - static_cast<double>(b.activations[e]))
                                      : static_cast<TL>(b.mtarget[e]);
  }
  for (int c9 = 0; c9 < 9; ++c9) {
    M3<TL> df = zero3<TL>();
    df.a[c9 % 3][c9 / 3] = TL(1);
    M3<TL> dp = zero3<TL>();
    if (b.material == 0) {
      if (wc != TL(0)) dp = dp + wc * corotated_jvp(u, sigma, v, df);
      if (wv != TL(0)) dp = dp + wv * volume_jvp(u, sigma, v, offset, df);
    } else if (wn != TL(0)) {
      dp = dp + wn * nh_prox_jvp(u, sigma, v, stretches, df, mu, lame, penalty);
    }
    if (wm != TL(0)) dp = dp + wm * outer(muscle_jvp(f, m, target, df), m);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) out[c9 * 9 + r * 3 + c] = dp.a[r][c];
  }
}

// ds = sum_c dF[c % 3][c / 3] J_c.
template <typename TL>
__device__ __forceinline__ M3<double> apply_jacobian(const TL* jac, const double df[3][3]) {
  M3<double> ds = zero3<double>();
  for (int c9 = 0; c9 < 9; ++c9) {
    const double coefficient = df[c9 % 3][c9 / 3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) ds.a[r][c] += coefficient * static_cast<double>(jac[c9 * 9 + r * 3 + c]);
  }
  return ds;
}

__device__ __forceinline__ void deformation_from(const int* idx, const double* grad, int corners, const double* vec,
                                                 double out[3][3]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[r][c] = 0.0;
  for (int k = 0; k < corners; ++k) {
    const int v = idx[k];
    const double* g = grad + 3 * k;
    const double px = vec[3 * v], py = vec[3 * v + 1], pz = vec[3 * v + 2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      out[0][c] += px * g[c];
      out[1][c] += py * g[c];
      out[2][c] += pz * g[c];
    }
  }
}

// Deformation of the combination vec + beta * vec2 (a CG search direction formed on the fly).
__device__ __forceinline__ void deformation_combined(const int* idx, const double* grad, int corners, const double* vec,
                                                     const double* vec2, double beta, double out[3][3]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[r][c] = 0.0;
  for (int k = 0; k < corners; ++k) {
    const int v = idx[k];
    const double* g = grad + 3 * k;
    const double px = vec[3 * v] + beta * vec2[3 * v];
    const double py = vec[3 * v + 1] + beta * vec2[3 * v + 1];
    const double pz = vec[3 * v + 2] + beta * vec2[3 * v + 2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      out[0][c] += px * g[c];
      out[1][c] += py * g[c];
      out[2][c] += pz * g[c];
    }
  }
}

// Per-sample gradient rows: Tet4 element e, or Hex8 sample s (shared).
__device__ __forceinline__ const double* sample_gradients(const AdjointArgs& b, const double* grad_smem, int e, int s) {
  return b.hex ? grad_smem + 8 * 3 * s : b.gradients + 12 * e;
}

// Element phase writing corner contributions of the operator `op` applied to
// `vec`: op 0 -> K vec (local Jacobian), op 1 -> (A - K) vec without the mass
// term (Dirichlet coupling, adjoint.py:493-521).
template <typename TL>
__device__ void element_operator(const AdjointArgs& b, const double* grad_smem, const double* vec, int op, Team team,
                                 const double* vec2 = nullptr, double beta = 0.0) {
  const int samples = b.hex ? 8 : 1;
  const int corners = b.corners;
  const int total = b.ne * samples;
  // Hex8 contributions are summed over the eight samples of a cell in a fixed
  // order by the thread that owns the cell; Tet4 has one sample per element.
  const int gthreads = team.size * blockDim.x;
  for (int e = threadIdx.x * team.size + team.rank; e < b.ne; e += gthreads) {
    double acc[8][3];
    for (int k = 0; k < corners; ++k) acc[k][0] = acc[k][1] = acc[k][2] = 0.0;
    for (int s = 0; s < samples; ++s) {
      const double* g = sample_gradients(b, grad_smem, e, s);
      double df[3][3];
      if (vec2 != nullptr) {
        deformation_combined(b.indices + corners * e, g, corners, vec, vec2, beta, df);
      } else {
        deformation_from(b.indices + corners * e, g, corners, vec, df);
      }
      const TL* jac = jacobian_ptr<TL>(b) + static_cast<size_t>(e * samples + s) * 81;
      M3<double> ds = apply_jacobian<TL>(jac, df);
      if (op == 1) {
        const double w = b.wc[e] + b.wv[e] + b.wn[e];
        M3<double> a = zero3<double>();
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) a.a[r][c] = w * df[r][c];
        if (b.has_muscles && b.wm[e] != 0.0) {
          const V3<double> m = load3d(b.mdir, e);
          V3<double> dfm;
          for (int r = 0; r < 3; ++r) dfm[r] = df[r][0] * m.x + df[r][1] * m.y + df[r][2] * m.z;
          a = a + b.wm[e] * outer(dfm, m);
        }
        ds = a - ds;
      }
      for (int k = 0; k < corners; ++k) {
        const V3<double> gk = v3<double>(g[3 * k], g[3 * k + 1], g[3 * k + 2]);
        const V3<double> c = mul(ds, gk);
        acc[k][0] += c.x;
        acc[k][1] += c.y;
        acc[k][2] += c.z;
      }
    }
    (void)total;
    for (int k = 0; k < corners; ++k) {
      double* out = b.contrib + (corners * e + k) * 3;
      out[0] = acc[k][0];
      out[1] = acc[k][1];
      out[2] = acc[k][2];
    }
  }
}

__device__ __forceinline__ V3<double> gather_row(const AdjointArgs& b, int i) {
  double px = 0.0, py = 0.0, pz = 0.0;
  for (int k = b.inc_offsets[i]; k < b.inc_offsets[i + 1]; ++k) {
    const double* c = b.contrib + 3 * b.inc_entries[k];
    px += c[0];
    py += c[1];
    pz += c[2];
  }
  return v3<double>(px, py, pz);
}

// Block partial of the Anderson Gram entries (same layout as the forward).
__device__ void adjoint_gram_partials(const AdjointArgs& b, int r0, int r1, int count, int start, double* block_out,
                                      double* scratch, int blocks) {
  const int entries = count * (count + 1) / 2 + count;
  const int capacity = b.window + 1;
  const int groups = entries > 0 ? kBlock / entries : 0;
  const int t = threadIdx.x;
  double sum = 0.0;
  const size_t stride = static_cast<size_t>(3) * b.n;
  if (entries > 0 && t < groups * entries) {
    const int entry = t % entries;
    const int group = t / entries;
    const int pairs = count * (count + 1) / 2;
    if (entry < pairs) {
      int ea, eb;
      gram_entry_pair(entry, count, ea, eb);
      const double* ga1 = b.hist_g + ((start + ea + 1) % capacity) * stride;
      const double* ga0 = b.hist_g + ((start + ea) % capacity) * stride;
      const double* gb1 = b.hist_g + ((start + eb + 1) % capacity) * stride;
      const double* gb0 = b.hist_g + ((start + eb) % capacity) * stride;
      for (int i = r0 + group; i < r1; i += groups)
        for (int c = 0; c < 3; ++c) sum += (ga1[3 * i + c] - ga0[3 * i + c]) * (gb1[3 * i + c] - gb0[3 * i + c]);
    } else {
      const int ea = entry - pairs;
      const double* ga1 = b.hist_g + ((start + ea + 1) % capacity) * stride;
      const double* ga0 = b.hist_g + ((start + ea) % capacity) * stride;
      const double* gn = b.hist_g + ((start + count) % capacity) * stride;
      for (int i = r0 + group; i < r1; i += groups)
        for (int c = 0; c < 3; ++c) sum += (ga1[3 * i + c] - ga0[3 * i + c]) * gn[3 * i + c];
    }
  }
  scratch[t] = sum;
  __syncthreads();
  if (t < entries) {
    double total = 0.0;
    for (int g = 0; g < groups; ++g) total += scratch[g * entries + t];
    block_out[t * blocks] = total;
  }
  __syncthreads();
}

__device__ __forceinline__ V3<double> adjoint_aa_apply_row(const AdjointArgs& b, int i, int count, int start,
                                                           const double* gamma) {
  const int capacity = b.window + 1;
  const size_t stride = static_cast<size_t>(3) * b.n;
  const int slot = (start + count) % capacity;
  V3<double> value;
  for (int c = 0; c < 3; ++c) value[c] = b.hist_x[slot * stride + 3 * i + c] + b.hist_g[slot * stride + 3 * i + c];
  for (int k = 0; k < count; ++k) {
    const int low = (start + k) % capacity;
    const int high = (start + k + 1) % capacity;
    for (int c = 0; c < 3; ++c) {
      const size_t h = high * stride + 3 * i + c;
      const size_t l = low * stride + 3 * i + c;
      value[c] -= (b.hist_x[h] - b.hist_x[l] + b.hist_g[h] - b.hist_g[l]) * gamma[k];
    }
  }
  return value;
}

// Partial slots inside a block's kPartialStride doubles.
constexpr int kSlotGram = 0;      // .. 43
constexpr int kSlotRaw = 48;      // ||raw||^2 after the solve
constexpr int kSlotStep = 49;     // ||raw - prev||^2
constexpr int kSlotMixed = 50;    // ||raw||^2 after mixing
constexpr int kSlotRhs = 51;      // ||g||^2 (seed)
constexpr int kSlotMaterial = 52; // material gradient column sums (2)
constexpr int kSlotActivation = 54;
constexpr int kSlotRZ = 56;   // CG: r^T z
constexpr int kSlotZZ = 57;   // CG: z^T z (the fixed-point step norm)
constexpr int kSlotMM = 58;   // CG: mu^T mu
constexpr int kSlotPQ = 59;   // CG: p^T (A - K) p

// One adjoint step of one instance by one team of blocks. Returns false when
// a team barrier gave up (the status word says why).
template <typename TL, typename TV>
__device__ __forceinline__ bool adjoint_step_body(const AdjointArgs& b, const Team team, char* dyn_smem) {
  __shared__ double s_grad[8 * 8 * 3];
  __shared__ double s_scratch[kBlock];
  __shared__ double s_reduced[64];
  __shared__ int s_control[8];
  const int gtid = team.rank * blockDim.x + threadIdx.x;
  const int gthreads = team.size * blockDim.x;
  const int n = b.n;
  const int samples = b.hex ? 8 : 1;
  const int corners = b.corners;
  if (b.hex) {
    for (int t = threadIdx.x; t < 8 * 8 * 3; t += blockDim.x) s_grad[t] = b.gradients[t];
    __syncthreads();
  }
  const int r0 = b.st_part[team.rank], r1 = b.st_part[team.rank + 1];
  double* my_partials = b.partials + team.rank;  // slot-major: [slot * team.size]
  const size_t hstride = static_cast<size_t>(3) * n;
  const double dt = b.dt;

  // ---- Prologue: seed (own rows), local Jacobians (elements).
  if (b.mode != 2) {
    double rhs2 = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      V3<double> g;
      if (b.mode == 1) {
        g = load3d(b.seed, i);
      } else {
        for (int c = 0; c < 3; ++c) {
          const double velocity = state_load(b.gqd_out, b.state_f64, 3 * i + c) / dt;
          g[c] = state_load(b.gq_out, b.state_f64, 3 * i + c) + velocity;
          b.base[3 * i + c] = -velocity;
        }
      }
      store3(b.rhs, i, g);
      store3(b.solution, i, v3<double>(0.0, 0.0, 0.0));
      rhs2 += dot(g, g);
    }
    rhs2 = block_sum(rhs2, s_scratch);
    if (threadIdx.x == 0) my_partials[(kSlotRhs) * team.size] = rhs2;
  }
  for (int t = b.reuse_jacobian ? b.ne * samples : gtid; t < b.ne * samples; t += gthreads) {
    const int e = t / samples;
    const int s = t % samples;
    double fm[3][3];
    deformation_from(b.indices + corners * e, sample_gradients(b, s_grad, e, s), corners, b.x, fm);
    M3<TL> f;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) f.a[r][c] = static_cast<TL>(fm[r][c]);
    TL jac[81];
    sample_jacobian<TL>(b, e, f, jac);
    TL* out = jacobian_ptr<TL>(b) + static_cast<size_t>(t) * 81;
    for (int k = 0; k < 81; ++k) out[k] = jac[k];
  }
  if (gtid == 0) {
    b.aa_state[0] = b.aa_state[1] = b.aa_state[2] = b.aa_state[3] = 0;
    *b.aa_accept = 0;
    *b.iteration = 0;
    *b.active = 1;
  }
  const TV* s_values = sizeof(TV) == sizeof(double) ? reinterpret_cast<const TV*>(b.s_val)
                                                    : reinterpret_cast<const TV*>(b.s_val32);
  const TV* st_values = sizeof(TV) == sizeof(double) ? reinterpret_cast<const TV*>(b.st_val)
                                                     : reinterpret_cast<const TV*>(b.st_val32);
  if (b.resident) {
    load_slice<TV>(b.plan_s, s_values, dyn_smem, team.rank);
    load_slice<TV>(b.plan_st, st_values, dyn_smem, team.rank);
  }
  double* vector_smem = reinterpret_cast<double*>(dyn_smem + b.vector_smem_offset);
  if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;

  if (b.mode == 2) {
    // Parameters only: the solution buffer already holds z.
  } else if (b.pcg) {
    // ---- Preconditioned conjugate gradients on (A - K) mu = g over the free
    // rows, preconditioned by the factor A^{-1} = S^T S. The reference's
    // fixed-point step A^{-1}(g + K mu) - mu equals the preconditioned residual
    // z = A^{-1} r, so the stop rule ||z|| < rel ||mu|| + abs is the reference's.
    // Per iteration: S | S^T (+ serial: beta, stop) | K p | A p - K p (+ serial:
    // alpha) | updates; the new direction p = z + beta p is formed where read.
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      V3<double> g = load3d(b.rhs, i);
      if (b.free_[i] == 0) g = v3<double>(0.0, 0.0, 0.0);
      store3(b.work, i, g);                                  // r
      store3(b.prev, i, v3<double>(0.0, 0.0, 0.0));          // p
    }
    if (threadIdx.x == 0) my_partials[kSlotMM * team.size] = 0.0;
    if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;
    for (;;) {
      // z = A^{-1} r.
      {
        const double* in = b.work;
        if (b.stage_vector) {
          stage_for(b.plan_s, team.rank, b.work, vector_smem, n);
          in = vector_smem;
        }
        spmv_block<TV>(b.plan_s, s_values, b.resident != 0, dyn_smem, in, b.y, team.rank);
      }
      if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;
      {
        const double* in = b.y;
        if (b.stage_vector) {
          stage_for(b.plan_st, team.rank, b.y, vector_smem, n);
          in = vector_smem;
        }
        spmv_block<TV>(b.plan_st, st_values, b.resident != 0, dyn_smem, in, b.raw, team.rank);
      }
      __syncthreads();
      double rz = 0.0, zz = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        V3<double> z = load3d(b.raw, i);
        if (b.free_[i] == 0) z = v3<double>(0.0, 0.0, 0.0);
        for (int c = 0; c < 3; ++c) {
          if (!isfinite(z[c])) {
            z[c] = 0.0;
            atomicOr(b.status, kStatusAdjointSafeguard);
          }
        }
        store3(b.raw, i, z);
        rz += dot(load3d(b.work, i), z);
        zz += dot(z, z);
      }
      rz = block_sum(rz, s_scratch);
      zz = block_sum(zz, s_scratch);
      if (threadIdx.x == 0) {
        my_partials[kSlotRZ * team.size] = rz;
        my_partials[kSlotZZ * team.size] = zz;
      }
      {
        unsigned generation;
        if (barrier_arrive(b.barrier, generation, team.size)) {
          reduce_partials(b.partials, kSlotRZ, 3, team.size, s_reduced, s_scratch);
          if (threadIdx.x == 0) {
            const double rho = s_reduced[0];
            const double step_norm = sqrt(s_reduced[1]);
            const double mu_norm = sqrt(s_reduced[2]);
            const int k = *b.iteration;
            *b.iteration = k + 1;
            int active = 1;
            if (k > 0 && step_norm < b.rel_tol * mu_norm + b.abs_tol) {
              active = 0;
            } else if (k + 1 >= b.max_iterations) {
              active = 0;
              if (b.mode == 0) atomicOr(b.status, kStatusAdjointNotConverged);
            } else if (!(rho > 0.0) || !isfinite(rho)) {
              // Zero residual (exact solve) or a non-positive preconditioned norm.
              active = 0;
              if (!(rho == 0.0)) atomicOr(b.status, kStatusAdjointSafeguard);
            }
            const double previous_rho = b.control_d[5];
            b.control_d[6] = (k == 0 || !(previous_rho > 0.0)) ? 0.0 : rho / previous_rho;  // beta
            b.control_d[5] = rho;
            b.control_d[3] = mu_norm;
            *b.active = active;
          }
          barrier_release(b.barrier, generation, team.size);
          __syncthreads();
        } else if (!barrier_wait(b.barrier, generation, b.status)) {
          return false;
        }
      }
      if (threadIdx.x == 0) s_control[0] = *reinterpret_cast<volatile int*>(b.active);
      __syncthreads();
      if (s_control[0] == 0) break;
      const double beta = *reinterpret_cast<volatile double*>(b.control_d + 6);
      // K p with p = z + beta p_old formed on the fly.
      element_operator<TL>(b, s_grad, b.raw, 0, team, b.prev, beta);
      if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;
      // q = A p - K p on the free rows; p^T q partials.
      double pq = 0.0;
      {
        const int sub = threadIdx.x & 3;
        const int groups_total = gthreads >> 2;
        const int lane_group = (threadIdx.x & 31) >> 2;
        for (int base = (gtid >> 5) * 8; base < n; base += groups_total) {
          const int i = base + lane_group;
          const bool valid = i < n;
          double qx = 0.0, qy = 0.0, qz = 0.0;
          if (valid) {
            const int k0 = b.inc_offsets[i], k1 = b.inc_offsets[i + 1];
            for (int k = k0 + sub; k < k1; k += 4) {
              const double* c = b.contrib + 3 * b.inc_entries[k];
              qx -= c[0];
              qy -= c[1];
              qz -= c[2];
            }
            for (int q = b.a_off[i] + sub; q < b.a_off[i + 1]; q += 4) {
              const double v = b.a_val[q];
              const int j = b.a_col[q];
              qx += v * (b.raw[3 * j] + beta * b.prev[3 * j]);
              qy += v * (b.raw[3 * j + 1] + beta * b.prev[3 * j + 1]);
              qz += v * (b.raw[3 * j + 2] + beta * b.prev[3 * j + 2]);
            }
          }
#pragma unroll
          for (int mask = 1; mask < 4; mask <<= 1) {
            qx += __shfl_xor_sync(0xffffffffu, qx, mask);
            qy += __shfl_xor_sync(0xffffffffu, qy, mask);
            qz += __shfl_xor_sync(0xffffffffu, qz, mask);
          }
          if (valid && sub == 0) {
            if (b.free_[i] == 0) qx = qy = qz = 0.0;
            b.y[3 * i] = qx;
            b.y[3 * i + 1] = qy;
            b.y[3 * i + 2] = qz;
            pq += (b.raw[3 * i] + beta * b.prev[3 * i]) * qx + (b.raw[3 * i + 1] + beta * b.prev[3 * i + 1]) * qy +
                  (b.raw[3 * i + 2] + beta * b.prev[3 * i + 2]) * qz;
          }
        }
      }
      pq = block_sum(pq, s_scratch);
      if (threadIdx.x == 0) my_partials[kSlotPQ * team.size] = pq;
      {
        unsigned generation;
        if (barrier_arrive(b.barrier, generation, team.size)) {
          reduce_partials(b.partials, kSlotPQ, 1, team.size, s_reduced, s_scratch);
          if (threadIdx.x == 0) {
            const double curvature = s_reduced[0];
            double alpha = 0.0;
            if (curvature > 0.0 && isfinite(curvature)) {
              alpha = b.control_d[5] / curvature;
            } else {
              // (A - K) is not positive definite along p: keep mu and stop.
              atomicOr(b.status, kStatusAdjointSafeguard);
              *b.active = 0;
            }
            b.control_d[7] = alpha;
          }
          barrier_release(b.barrier, generation, team.size);
          __syncthreads();
        } else if (!barrier_wait(b.barrier, generation, b.status)) {
          return false;
        }
      }
      const double alpha = *reinterpret_cast<volatile double*>(b.control_d + 7);
      // mu += alpha p, r -= alpha q, p stored (own rows).
      double mm = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        V3<double> p = load3d(b.raw, i) + beta * load3d(b.prev, i);
        if (b.free_[i] == 0) p = v3<double>(0.0, 0.0, 0.0);
        const V3<double> mu = load3d(b.solution, i) + alpha * p;
        const V3<double> r = load3d(b.work, i) - alpha * load3d(b.y, i);
        store3(b.prev, i, p);
        store3(b.solution, i, mu);
        store3(b.work, i, r);
        mm += dot(mu, mu);
      }
      mm = block_sum(mm, s_scratch);
      if (threadIdx.x == 0) my_partials[kSlotMM * team.size] = mm;
      if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;
      if (threadIdx.x == 0) s_control[0] = *reinterpret_cast<volatile int*>(b.active);
      __syncthreads();
      if (s_control[0] == 0) break;
    }
  } else {
  for (;;) {
    // ---- A1: K solution per element.
    element_operator<TL>(b, s_grad, b.solution, 0, team);
    if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;

    // ---- A2: work = g + gather(K solution) (refinement: minus A solution),
    // four lanes per particle with a fixed shuffle tree.
    {
      const int sub = threadIdx.x & 3;
      const int groups_total = gthreads >> 2;
      const int lane_group = (threadIdx.x & 31) >> 2;
      for (int base = (gtid >> 5) * 8; base < n; base += groups_total) {
        const int i = base + lane_group;
        const bool valid = i < n;
        double px = 0.0, py = 0.0, pz = 0.0;
        if (valid) {
          const int k0 = b.inc_offsets[i], k1 = b.inc_offsets[i + 1];
#pragma unroll 4
          for (int k = k0 + sub; k < k1; k += 4) {
            const double* c = b.contrib + 3 * b.inc_entries[k];
            px += c[0];
            py += c[1];
            pz += c[2];
          }
          if (b.refine) {
            for (int q = b.a_off[i] + sub; q < b.a_off[i + 1]; q += 4) {
              const double v = b.a_val[q];
              const int j = b.a_col[q];
              px -= v * b.solution[3 * j];
              py -= v * b.solution[3 * j + 1];
              pz -= v * b.solution[3 * j + 2];
            }
          }
        }
#pragma unroll
        for (int mask = 1; mask < 4; mask <<= 1) {
          px += __shfl_xor_sync(0xffffffffu, px, mask);
          py += __shfl_xor_sync(0xffffffffu, py, mask);
          pz += __shfl_xor_sync(0xffffffffu, pz, mask);
        }
        if (valid && sub == 0) {
          b.work[3 * i] = px + b.rhs[3 * i];
          b.work[3 * i + 1] = py + b.rhs[3 * i + 1];
          b.work[3 * i + 2] = pz + b.rhs[3 * i + 2];
        }
      }
    }
    if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;

    // ---- A3: y = S work.
    {
      const double* in = b.work;
      if (b.stage_vector) {
        stage_for(b.plan_s, team.rank, b.work, vector_smem, n);
        in = vector_smem;
      }
      spmv_block<TV>(b.plan_s, s_values, b.resident != 0, dyn_smem, in, b.y, team.rank);
    }
    if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;

    // ---- A4: raw = S^T y; Dirichlet zeroing and scrub; history; partials.
    {
      const double* in = b.y;
      if (b.stage_vector) {
        stage_for(b.plan_st, team.rank, b.y, vector_smem, n);
        in = vector_smem;
      }
      spmv_block<TV>(b.plan_st, st_values, b.resident != 0, dyn_smem, in, b.raw, team.rank);
    }
    __syncthreads();
    const int count = b.window > 0 ? b.aa_state[0] : 0;
    const int start = b.window > 0 ? b.aa_state[1] : 0;
    const int capacity = b.window + 1;
    {
      double raw2 = 0.0, step2 = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        V3<double> value = load3d(b.raw, i);
        const V3<double> previous = load3d(b.solution, i);
        if (b.refine) value = value + previous;
        if (b.free_[i] == 0) value = v3<double>(0.0, 0.0, 0.0);
        for (int c = 0; c < 3; ++c) {
          if (!isfinite(value[c])) {
            value[c] = 0.0;
            atomicOr(b.status, kStatusAdjointSafeguard);
          }
        }
        store3(b.raw, i, value);
        store3(b.prev, i, previous);
        raw2 += dot(value, value);
        const V3<double> step = value - previous;
        step2 += dot(step, step);
        if (b.window > 0) {
          const int slot = (start + count) % capacity;
          double* hx = b.hist_x + slot * hstride + 3 * i;
          double* hg = b.hist_g + slot * hstride + 3 * i;
          for (int c = 0; c < 3; ++c) {
            hx[c] = previous[c];
            hg[c] = step[c];
          }
        }
      }
      raw2 = block_sum(raw2, s_scratch);
      step2 = block_sum(step2, s_scratch);
      if (threadIdx.x == 0) {
        my_partials[(kSlotRaw) * team.size] = raw2;
        my_partials[(kSlotStep) * team.size] = step2;
      }
      if (b.window > 0) {
        __syncthreads();
        adjoint_gram_partials(b, r0, r1, count, start, my_partials + kSlotGram * team.size, s_scratch, team.size);
      }
      // Serial: norm clip of the solve result (safe_clip, adjoint.py:184-223);
      // without clipping also the Anderson solve and the step norm.
      unsigned generation;
      if (barrier_arrive(b.barrier, generation, team.size)) {
        reduce_partials(b.partials, kSlotRaw, 2, team.size, s_reduced, s_scratch);
        const double len = sqrt(s_reduced[0]);
        const bool clip = isfinite(len) && len > kClipNorm;
        if (threadIdx.x == 0) {
          b.control_d[0] = clip ? kClipNorm / len : 1.0;
          b.control_d[1] = s_reduced[1];
          if (clip) atomicOr(b.status, kStatusAdjointSafeguard);
        }
        __syncthreads();
        if (!clip && b.window > 0) {
          const int entries = count * (count + 1) / 2 + count;
          reduce_partials(b.partials, kSlotGram, entries, team.size, s_reduced, s_scratch);
          if (threadIdx.x == 0) aa_solve(b.aa_state, b.aa_gamma, b.aa_accept, s_reduced, b.window, s_scratch);
        }
        barrier_release(b.barrier, generation, team.size);
        __syncthreads();
      } else if (!barrier_wait(b.barrier, generation, b.status)) {
        return false;
      }
    }
    const double clip1 = *reinterpret_cast<volatile double*>(b.control_d);
    if (clip1 != 1.0) {
      // Rare slow path: rescale, then redo the step norm, history and Gram.
      double step2 = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const V3<double> value = clip1 * load3d(b.raw, i);
        store3(b.raw, i, value);
        const V3<double> step = value - load3d(b.prev, i);
        step2 += dot(step, step);
        if (b.window > 0) {
          const int slot = (start + count) % capacity;
          double* hg = b.hist_g + slot * hstride + 3 * i;
          for (int c = 0; c < 3; ++c) hg[c] = step[c];
        }
      }
      step2 = block_sum(step2, s_scratch);
      if (threadIdx.x == 0) my_partials[(kSlotStep) * team.size] = step2;
      if (b.window > 0) {
        __syncthreads();
        adjoint_gram_partials(b, r0, r1, count, start, my_partials + kSlotGram * team.size, s_scratch, team.size);
      }
      unsigned generation;
      if (barrier_arrive(b.barrier, generation, team.size)) {
        if (b.window > 0) {
          const int entries = count * (count + 1) / 2 + count;
          reduce_partials(b.partials, kSlotGram, entries, team.size, s_reduced, s_scratch);
          if (threadIdx.x == 0) aa_solve(b.aa_state, b.aa_gamma, b.aa_accept, s_reduced, b.window, s_scratch);
          __syncthreads();
        }
        reduce_partials(b.partials, kSlotStep, 1, team.size, s_reduced, s_scratch);
        if (threadIdx.x == 0) b.control_d[1] = s_reduced[0];
        barrier_release(b.barrier, generation, team.size);
        __syncthreads();
      } else if (!barrier_wait(b.barrier, generation, b.status)) {
        return false;
      }
    }

    // ---- A5: Anderson apply, second clip, stopping rule.
    {
      int accept = 0, used_count = 0, used_start = 0;
      if (b.window > 0) {
        accept = *reinterpret_cast<volatile int*>(b.aa_accept);
        used_count = *reinterpret_cast<volatile int*>(b.aa_state + 2);
        used_start = *reinterpret_cast<volatile int*>(b.aa_state + 3);
        if (threadIdx.x < kMaxWindow) s_reduced[32 + threadIdx.x] = reinterpret_cast<volatile double*>(b.aa_gamma)[threadIdx.x];
        __syncthreads();
      }
      double mixed2 = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        V3<double> value = load3d(b.raw, i);
        if (accept) value = adjoint_aa_apply_row(b, i, used_count, used_start, s_reduced + 32);
        if (b.free_[i] == 0) value = v3<double>(0.0, 0.0, 0.0);
        for (int c = 0; c < 3; ++c) {
          if (!isfinite(value[c])) {
            value[c] = 0.0;
            atomicOr(b.status, kStatusAdjointSafeguard);
          }
        }
        store3(b.solution, i, value);
        mixed2 += dot(value, value);
      }
      mixed2 = block_sum(mixed2, s_scratch);
      if (threadIdx.x == 0) my_partials[(kSlotMixed) * team.size] = mixed2;
      unsigned generation;
      if (barrier_arrive(b.barrier, generation, team.size)) {
        reduce_partials(b.partials, kSlotMixed, 1, team.size, s_reduced, s_scratch);
        if (threadIdx.x == 0) {
          const double len = sqrt(s_reduced[0]);
          double scale = 1.0;
          double solution_norm = len;
          if (isfinite(len) && len > kClipNorm) {
            scale = kClipNorm / len;
            solution_norm = sqrt(scale * scale * s_reduced[0]);
            atomicOr(b.status, kStatusAdjointSafeguard);
          }
          b.control_d[2] = scale;
          const double step_norm = sqrt(b.control_d[1]);
          const int k = *b.iteration;
          *b.iteration = k + 1;
          int active = 1;
          if (k > 0 && step_norm < b.rel_tol * solution_norm + b.abs_tol) {
            active = 0;
          } else if (k + 1 >= b.max_iterations) {
            active = 0;
            if (b.mode == 0) atomicOr(b.status, kStatusAdjointNotConverged);
          }
          *b.active = active;
          b.control_d[3] = solution_norm;
        }
        barrier_release(b.barrier, generation, team.size);
        __syncthreads();
      } else if (!barrier_wait(b.barrier, generation, b.status)) {
        return false;
      }
      const double clip2 = *reinterpret_cast<volatile double*>(b.control_d + 2);
      if (clip2 != 1.0) {
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) store3(b.solution, i, clip2 * load3d(b.solution, i));
        if (!grid_sync(b.barrier, b.status, team.size, team.rank)) return false;
      }
      if (threadIdx.x == 0) s_control[0] = *reinterpret_cast<volatile int*>(b.active);
      __syncthreads();
      if (s_control[0] == 0) break;
    }
  }

  }

  if (b.mode == 1) return true;  // one Woodbury column in `solution`

  // ---- Routing guard (adjoint.py:1125-1138, :226-261), in one serial section.
  if (b.mode == 0) {
    unsigned generation;
    if (barrier_arrive(b.barrier, generation, team.size)) {
      reduce_partials(b.partials, kSlotRhs, 1, team.size, s_reduced, s_scratch);
      if (threadIdx.x == 0) {
        const double mu_norm = *reinterpret_cast<volatile double*>(b.control_d + 3);
        const bool failed = kClipNorm > 0.0 && mu_norm >= 0.999 * kClipNorm;
        double value = 1.0;
        if (failed) {
          value = 0.0;
          atomicOr(b.status, kStatusAdjointSafeguard);
        } else {
          const double cap = sqrt(s_reduced[0]) + 1.0;
          const double injection = b.inertia * mu_norm;
          if (injection > cap) {
            value = cap / injection;
            atomicOr(b.status, kStatusAdjointSafeguard);
          }
        }
        b.control_d[4] = value;
        b.control_i[0] = failed ? 1 : 0;
      }
      barrier_release(b.barrier, generation, team.size);
      __syncthreads();
    } else if (!barrier_wait(b.barrier, generation, b.status)) {
      return false;
    }
  }
  const double routing = *reinterpret_cast<volatile double*>(b.control_d + 4);
  const int diverged = *reinterpret_cast<volatile int*>(b.control_i);

  // ---- State gradients (own rows, adjoint.py:474-490).
  for (int i = b.mode == 0 ? r0 + threadIdx.x : r1; i < r1; i += blockDim.x) {
    for (int c = 0; c < 3; ++c) {
      const double mu = b.solution[3 * i + c];
      const double injection = routing * b.inertia * mu;
      state_add(b.gq, b.state_f64, 3 * i + c, b.base[3 * i + c] + injection);
      state_add(b.gqd, b.state_f64, 3 * i + c, dt * injection);
      state_add(b.gf, b.state_f64, 3 * i + c, routing * mu);
    }
  }

  // ---- Element epilogue: Dirichlet coupling contributions, material and
  // activation gradients from z = mu (no contact rows).
  if (b.has_dirichlet && b.mode == 0) {
    if (diverged) {
      for (int t = gtid; t < b.ne * corners * 3; t += gthreads) b.contrib[t] = 0.0;
    } else {
      element_operator<TL>(b, s_grad, b.solution, 1, team);
    }
  }
  double material0 = 0.0, material1 = 0.0, activation = 0.0;
  const bool want_material = b.gmaterials != nullptr;
  const bool want_activation = b.gactivations != nullptr && b.has_muscles;
  if (want_material || want_activation) {
    const double volume = b.sample_volume;
    for (int e = gtid; e < b.ne; e += gthreads) {
      double first_value = 0.0, second_value = 0.0, act_value = 0.0;
      for (int s = 0; s < samples; ++s) {
        const double* g = sample_gradients(b, s_grad, e, s);
        double fm[3][3];
        deformation_from(b.indices + corners * e, g, corners, b.x, fm);
        M3<double> f;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) f.a[r][c] = fm[r][c];
        M3<double> first = zero3<double>(), second = zero3<double>();
        if (want_material) {
          if (b.material == 0) {
            M3<double> u, v;
            V3<double> sigma;
            unsigned_svd(f, u, sigma, v);
            bool singular;
            const V3<double> offset = volume_offset(sigma, singular);
            first = f - mul(u, transpose(v));
            second = f - udvt(u, sigma + offset, v);
          } else {
            first = (1.0 / (2.0 * b.nh_mu)) * neo_hookean_stress(f, b.nh_mu, b.nh_lame);
          }
        }
        V3<double> fibre = v3<double>(0.0, 0.0, 0.0);
        double len = 0.0;
        V3<double> m = fibre;
        const bool fibre_on = want_activation && b.wm[e] != 0.0;
        if (fibre_on) {
          m = load3d(b.mdir, e);
          fibre = mul(f, m);
          len = length(fibre);
        }
        for (int k = 0; k < corners; ++k) {
          const int v = b.indices[corners * e + k];
          const V3<double> z = load3d(b.solution, v);
          const V3<double> gk = v3<double>(g[3 * k], g[3 * k + 1], g[3 * k + 2]);
          first_value -= dot(z, mul(first, gk));
          second_value -= dot(z, mul(second, gk));
          if (fibre_on && len > DBL_EPSILON) act_value += dot(z, (b.wm[e] / len * dot(m, gk)) * fibre);
        }
      }
      const double g0 = 2.0 * volume * first_value;
      const double g1 = b.material == 0 ? volume * second_value : 0.0;
      if (want_material) {
        b.material_scratch[2 * e] = g0;
        b.material_scratch[2 * e + 1] = g1;
        material0 += g0;
        material1 += g1;
      }
      if (want_activation) {
        b.activation_scratch[e] = -act_value;
        activation += -act_value;
      }
    }
  }
  material0 = block_sum(material0, s_scratch);
  material1 = block_sum(material1, s_scratch);
  activation = block_sum(activation, s_scratch);
  if (threadIdx.x == 0) {
    my_partials[(kSlotMaterial) * team.size] = material0;
    my_partials[(kSlotMaterial + 1) * team.size] = material1;
    my_partials[(kSlotActivation) * team.size] = activation;
  }
  // Parameter guard (adjoint.py:622-644).
  {
    unsigned generation;
    if (barrier_arrive(b.barrier, generation, team.size)) {
      reduce_partials(b.partials, kSlotMaterial, 3, team.size, s_reduced, s_scratch);
      if (threadIdx.x == 0) {
        const bool material_ok = !b.zero_energy_weight && isfinite(s_reduced[0]) && isfinite(s_reduced[1]);
        const bool activation_ok = isfinite(s_reduced[2]);
        b.control_i[1] = (diverged == 0 && material_ok) ? 1 : 0;
        b.control_i[2] = (diverged == 0 && activation_ok) ? 1 : 0;
        if ((want_material && !material_ok) || (want_activation && !activation_ok)) {
          atomicOr(b.status, kStatusAdjointSafeguard);
        }
      }
      barrier_release(b.barrier, generation, team.size);
      __syncthreads();
    } else if (!barrier_wait(b.barrier, generation, b.status)) {
      return false;
    }
  }
  const int material_valid = *reinterpret_cast<volatile int*>(b.control_i + 1);
  const int activation_valid = *reinterpret_cast<volatile int*>(b.control_i + 2);
  if (want_material && material_valid) {
    for (int e = gtid; e < b.ne; e += gthreads) {
      b.gmaterials[2 * e] += b.material_scratch[2 * e];
      b.gmaterials[2 * e + 1] += b.material_scratch[2 * e + 1];
    }
  }
  if (want_activation && activation_valid) {
    for (int e = gtid; e < b.ne; e += gthreads) {
      b.gactivations[e] = b.gactivations[e] + static_cast<float>(b.activation_scratch[e]);
    }
  }
  // Dirichlet gradients: dL/dx_D = g_D - (A - K)_DF mu_F (adjoint.py:524-553).
  if (b.has_dirichlet && b.mode == 0) {
    for (int i = gtid; i < n; i += gthreads) {
      if (b.free_[i] != 0) continue;
      const V3<double> coupling = gather_row(b, i);
      for (int c = 0; c < 3; ++c) {
        const double value = b.rhs[3 * i + c] - coupling[c];
        if (b.gdirichlet != nullptr) {
          state_add(b.gdirichlet, b.state_f64, 3 * i + c, value);
        } else {
          state_add(b.gq, b.state_f64, 3 * i + c, value);
          if (b.integrate_pinned) state_add(b.gqd, b.state_f64, 3 * i + c, dt * value);
        }
      }
    }
  }
  return true;
}

// Plain launch: the whole cooperative grid is one team solving one instance.
template <typename TL, typename TV>
__global__ void __launch_bounds__(kBlock) adjoint_step_kernel(const AdjointArgs b) {
  extern __shared__ __align__(16) char dyn_smem[];
  adjoint_step_body<TL, TV>(b, Team{static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x)}, dyn_smem);
}

// Whole adjoint rollouts (last step first) of many instances, each by a team
// of blocks: the single-instance adjoint body per step. dL/dq and dL/dqd of
// consecutive steps alternate between two buffers; a team clears its slice
// of the buffer a step accumulates into before the step.
template <typename TL, typename TV>
__global__ void __launch_bounds__(kBlock, 2) team_adjoint_kernel(const TeamLaunch launch) {
  extern __shared__ __align__(16) char dyn_smem[];
  __shared__ AdjointArgs s_args;
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
    copy_arguments(launch.adjoint + instance, &s_args);
    if (launch.timeline != nullptr && team.rank == 0 && threadIdx.x == 0) {
      unsigned long long now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      launch.timeline[2 * instance] = now;
    }
    const long long offset = 3 * launch.particle_offset[instance];
    const int n3 = 3 * launch.adjoint[instance].n;
    __syncthreads();
    for (int t = launch.steps - 1; t >= 0; --t) {
      const int write = (launch.steps - 1 - t) & 1;
      void* gq = state_offset(launch.grad_q, f64, write * step_elements + offset);
      void* gqd = state_offset(launch.grad_qd, f64, write * step_elements + offset);
      for (int k = team.rank * blockDim.x + threadIdx.x; k < n3; k += team.size * blockDim.x) {
        state_store(gq, f64, k, 0.0);
        state_store(gqd, f64, k, 0.0);
      }
      if (threadIdx.x == 0) {
        const bool last = t == launch.steps - 1;
        s_args.barrier = barrier;
        s_args.x = launch.x_record + t * step_elements + offset;
        s_args.gq_out = last ? state_offset(launch.grad_q_final, f64, offset)
                             : state_offset(static_cast<const void*>(launch.grad_q), f64, (1 - write) * step_elements + offset);
        s_args.gqd_out = last ? state_offset(launch.grad_qd_final, f64, offset)
                              : state_offset(static_cast<const void*>(launch.grad_qd), f64, (1 - write) * step_elements + offset);
        s_args.gq = gq;
        s_args.gqd = gqd;
        s_args.gf = state_offset(launch.grad_forces, f64, t * step_elements + offset);
        s_args.gdirichlet = nullptr;
        s_args.gmaterials = launch.grad_materials != nullptr ? launch.grad_materials + 2 * launch.element_offset[instance]
                                                             : nullptr;
        s_args.gactivations = nullptr;
        s_args.activations = nullptr;
        s_args.dt = launch.dt;
      }
      __syncthreads();
      // The cleared accumulators are complete before any rank adds into them.
      if (!grid_sync(barrier, s_args.status, team.size, team.rank)) return;
      if (!adjoint_step_body<TL, TV>(s_args, team, dyn_smem)) return;
      if (team.rank == 0 && threadIdx.x == 0 && launch.iteration_log != nullptr)
        launch.iteration_log[t * launch.count + instance] = *s_args.iteration;
      if (!grid_sync(barrier, s_args.status, team.size, team.rank)) return;
    }
    if (launch.timeline != nullptr && team.rank == 0 && threadIdx.x == 0) {
      unsigned long long now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      launch.timeline[2 * instance + 1] = now;
    }
  }
}

static const void* team_adjoint(int precision) {
  if (precision == 0) return reinterpret_cast<const void*>(&team_adjoint_kernel<double, double>);
  if (precision == 1) return reinterpret_cast<const void*>(&team_adjoint_kernel<double, float>);
  return reinterpret_cast<const void*>(&team_adjoint_kernel<float, float>);
}

cudaError_t launch_team_adjoint(const TeamLaunch& launch, int blocks, int precision, size_t smem, cudaStream_t stream) {
  void* params[] = {const_cast<TeamLaunch*>(&launch)};
  return cudaLaunchCooperativeKernel(team_adjoint(precision), dim3(blocks), dim3(kBlock), params, smem, stream);
}

cudaError_t team_adjoint_max_blocks(int precision, size_t smem, int* blocks_per_sm) {
  const void* kernel = team_adjoint(precision);
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

// Columns of the contact projection (W_T = (A - K)^{-1} J^T), one work item
// per column: the single-instance adjoint fixed point (mode 1) with the
// column's own vectors, by the lane's team, as many columns at once as there
// are lanes (the reference solves them in batches, adjoint.py:666-806).
template <typename TL, typename TV>
__global__ void __launch_bounds__(kBlock, 2) team_column_kernel(const TeamLaunch launch) {
  extern __shared__ __align__(16) char dyn_smem[];
  __shared__ AdjointArgs s_args;
  Team lane_team;
  const int lane = lane_of_block(launch, lane_team);
  GridBarrier* barrier = &launch.lane_barrier[lane];
  bool solo = false;
  for (;;) {
    Team team;
    const int instance = next_work(launch, lane, lane_team, solo, team);
    if (instance < 0) return;
    copy_arguments(launch.adjoint + instance, &s_args);
    __syncthreads();
    if (threadIdx.x == 0) s_args.barrier = barrier;
    __syncthreads();
    if (!adjoint_step_body<TL, TV>(s_args, team, dyn_smem)) return;
    if (!grid_sync(barrier, s_args.status, team.size, team.rank)) return;
  }
}

static const void* team_columns(int precision) {
  if (precision == 0) return reinterpret_cast<const void*>(&team_column_kernel<double, double>);
  if (precision == 1) return reinterpret_cast<const void*>(&team_column_kernel<double, float>);
  return reinterpret_cast<const void*>(&team_column_kernel<float, float>);
}

cudaError_t launch_team_columns(const TeamLaunch& launch, int blocks, int precision, size_t smem, cudaStream_t stream) {
  void* params[] = {const_cast<TeamLaunch*>(&launch)};
  return cudaLaunchCooperativeKernel(team_columns(precision), dim3(blocks), dim3(kBlock), params, smem, stream);
}

cudaError_t team_columns_max_blocks(int precision, size_t smem, int* blocks_per_sm) {
  const void* kernel = team_columns(precision);
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

// precision 0: FP64; 1: FP64 Jacobians, FP32 factor products; 2: FP32 Jacobians and factor.
static const void* adjoint_kernel(int precision) {
  if (precision == 0) return reinterpret_cast<const void*>(&adjoint_step_kernel<double, double>);
  if (precision == 1) return reinterpret_cast<const void*>(&adjoint_step_kernel<double, float>);
  return reinterpret_cast<const void*>(&adjoint_step_kernel<float, float>);
}

cudaError_t launch_adjoint_step(const AdjointArgs& args, int blocks, int precision, size_t smem, cudaStream_t stream) {
  void* params[] = {const_cast<AdjointArgs*>(&args)};
  return cudaLaunchCooperativeKernel(adjoint_kernel(precision), dim3(blocks), dim3(kBlock), params, smem, stream);
}

// Allows the device's largest dynamic shared memory for the kernel (an
// attribute of the function, shared by every solver on the device, so it is
// never lowered to one solver's need) and returns the occupancy at `smem`.
cudaError_t adjoint_step_max_blocks(int precision, size_t smem, int* blocks_per_sm) {
  const void* kernel = adjoint_kernel(precision);
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

}  // namespace pdb200
