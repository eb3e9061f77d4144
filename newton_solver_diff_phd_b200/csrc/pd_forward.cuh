// Phases of the forward projective-dynamics step (one persistent launch).
//
// Per iteration (reference: SolverDiffPhD._iterate, solver.py:582-659):
//   P1 local step       elements -> contributions          (kernels.py:222-272, hex.py:122-169)
//   P2 gather + rhs     particles: p, b = m/h^2 q~ + p       (kernels.py:75-91, hex.py:246-260, :275-284)
//   P3 y = S b          S rows, nnz-balanced block ranges    (sparse.py:209-227)
//   P4 x = S^T y        S^T rows + Dirichlet values + Anderson history and Gram partials
//                       (sparse.py:341-348, kernels.py:287-291, anderson.py:306-354)
//   every block         Anderson least squares on the reduced partials (anderson.py:410-475)
//   P5 Anderson apply + convergence partials                 (anderson.py:478-503, kernels.py:354-401)
//   one warp, next P1   dual convergence gate, loop decision
// Only P1->P2, P2->P3, P3->P4, P4->P5 and P5->P1 cross blocks; particle rows
// of P4/P5 are owned by one block, so history, previous iterate and previous
// projection of a particle are only ever touched by that block.
#pragma once

#include "pd_device.cuh"

namespace pdb200 {

// Deformation gradient of a Tet4 element from float64 positions, as a TL matrix.
template <typename TL, typename Args>
__device__ __forceinline__ void tet_deformation(const Args& a, int e, const double* vec, M3<TL>& f) {
  double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int v = a.indices[4 * e + k];
    const double* g = a.gradients + (4 * e + k) * 3;
    const double px = vec[3 * v], py = vec[3 * v + 1], pz = vec[3 * v + 2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      m[0][c] += px * g[c];
      m[1][c] += py * g[c];
      m[2][c] += pz * g[c];
    }
  }
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) f.a[r][c] = static_cast<TL>(m[r][c]);
}

// SVD of F, warm-started from the singular vectors of the same sample in the
// previous iteration of this step: B = U0^T F V0 is nearly diagonal, so the
// Jacobi sweeps on B converge in one rotation sweep; U = U0 Ub, V = V0 Vb. The
// first iteration of a step starts cold (Eigen's conventions on F itself).
// su, sv: this sample's stored U and V (row-major, TS precision), or nullptr
// for a cold SVD without stored state.
template <typename TL, typename TS>
__device__ __forceinline__ void warm_svd(TS* su, TS* sv, bool warm, const M3<TL>& f, M3<TL>& u, V3<TL>& sigma,
                                         M3<TL>& v) {
  if (su == nullptr) {
    unsigned_svd(f, u, sigma, v);
    return;
  }
  if (warm) {
    M3<TL> u0, v0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      u0.a[k / 3][k % 3] = static_cast<TL>(su[k]);
      v0.a[k / 3][k % 3] = static_cast<TL>(sv[k]);
    }
    const M3<TL> b = mul(mul(transpose(u0), f), v0);
    M3<TL> ub, vb;
    unsigned_svd(b, ub, sigma, vb);
    u = mul(u0, ub);
    v = mul(v0, vb);
  } else {
    unsigned_svd(f, u, sigma, v);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    su[k] = static_cast<TS>(u.a[k / 3][k % 3]);
    sv[k] = static_cast<TS>(v.a[k / 3][k % 3]);
  }
}

// Warm-start state pointers of element sample `sample` (nullptr when the
// solver keeps none or the lane is padding, sample < 0).
template <typename TS>
__device__ __forceinline__ TS* svd_state(TS* base, int sample) {
  return (base == nullptr || sample < 0) ? nullptr : base + 9 * static_cast<size_t>(sample);
}

// Projection stress sum_energies w (P(F) - F_D) of one element sample.
// Args: any argument block with the per-element weights, muscle data, the
// Neo-Hookean parameters and the status word (StepArgs, BatchInstance).
template <typename TL, typename Args, typename TS>
__device__ __forceinline__ M3<TL> sample_stress(const Args& a, int e, TS* su, TS* sv, bool warm, const M3<TL>& f,
                                                const M3<TL>& fd) {
  M3<TL> stress = zero3<TL>();
  const TL wc = static_cast<TL>(a.wc[e]);
  const TL wv = static_cast<TL>(a.wv[e]);
  const TL wn = static_cast<TL>(a.wn[e]);
  if (wc != TL(0) || wv != TL(0) || wn != TL(0)) {
    M3<TL> u, v;
    V3<TL> sigma;
    warm_svd<TL, TS>(su, sv, warm, f, u, sigma, v);
    if (wc != TL(0)) stress = stress + wc * (mul(u, transpose(v)) - fd);
    if (wv != TL(0)) {
      bool singular;
      const V3<TL> offset = volume_offset(sigma, singular);
      if (singular) atomicOr(a.status, kStatusSingular);
      stress = stress + wv * (udvt(u, sigma + offset, v) - fd);
    }
    if (wn != TL(0)) {
      const V3<TL> stretches =
          nh_prox_stretches(sigma, static_cast<TL>(a.nh_mu), static_cast<TL>(a.nh_lame), static_cast<TL>(a.nh_penalty));
      stress = stress + wn * (udvt(u, stretches, v) - fd);
    }
  }
  if (a.has_muscles) {
    const TL wm = static_cast<TL>(a.wm[e]);
    if (wm != TL(0)) {
      const V3<TL> m = load3<TL>(a.mdir, e);
      const V3<TL> fibre = muscle_projection(f, m, static_cast<TL>(a.mtarget[e]));
      stress = stress + wm * outer(fibre - mul(fd, m), m);
    }
  }
  return stress;
}

// Local step of Tet4 element e: corner contributions stress g_k.
template <typename TL, typename Args, typename TS>
__device__ __forceinline__ void tet_element(const Args& a, int e, bool warm, TS* svd_u, TS* svd_v) {
  M3<TL> f, fd;
  tet_deformation<TL>(a, e, a.x, f);
  tet_deformation<TL>(a, e, a.boundary, fd);
  const M3<TL> stress = sample_stress<TL>(a, e, svd_state(svd_u, e), svd_state(svd_v, e), warm, f, fd);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double* g = a.gradients + (4 * e + k) * 3;
    const V3<TL> gk = v3<TL>(static_cast<TL>(g[0]), static_cast<TL>(g[1]), static_cast<TL>(g[2]));
    const V3<TL> c = mul(stress, gk);
    double* out = a.contrib + (4 * e + k) * 3;
    out[0] = static_cast<double>(c.x);
    out[1] = static_cast<double>(c.y);
    out[2] = static_cast<double>(c.z);
  }
}

// Contiguous range [first, last) of `count` work items of this block: the
// items are split evenly (sizes differ by at most one) over the team.
__device__ __forceinline__ void team_range(int count, Team team, int& first, int& last) {
  const int share = count / team.size, extra = count % team.size;
  first = team.rank * share + min(team.rank, extra);
  last = first + share + (team.rank < extra ? 1 : 0);
}

// P1 for Tet4: one thread per element, each block a contiguous range of
// elements, so the loads of indices, gradients and warm-start vectors of a
// warp are contiguous.
template <typename TL>
__device__ void local_step_tet(const StepArgs& a, bool warm, Team team) {
  int first, last;
  team_range(a.ne, team, first, last);
  for (int e = first + threadIdx.x; e < last; e += blockDim.x) tet_element<TL>(a, e, warm, a.svd_u, a.svd_v);
}

// Local step of Hex8 cell e by the eight lanes (lane & 7 = Gauss sample) of
// one lane group: the per-corner contributions sum_s stress_s g_sj are
// reduce-scattered across the eight lanes with shuffles (fixed tree), so lane
// s ends with corner j = s. Every lane of the warp must call this (the
// shuffles span the warp); lanes with e >= ne compute on a clamped cell,
// neither read nor write warm-start state and store nothing.
template <typename TL, typename Args, typename TS>
__device__ __forceinline__ void hex_cell(const Args& a, const double* grad_smem, int e, bool warm, TS* svd_u,
                                         TS* svd_v) {
  const int s = threadIdx.x & 7;
  const bool valid = e < a.ne;
  const int ec = valid ? e : a.ne - 1;
  double fm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double fdm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int v = a.indices[8 * ec + j];
    const double* g = grad_smem + (8 * s + j) * 3;
    const double px = a.x[3 * v], py = a.x[3 * v + 1], pz = a.x[3 * v + 2];
    const double bx = a.boundary[3 * v], by = a.boundary[3 * v + 1], bz = a.boundary[3 * v + 2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      fm[0][c] += px * g[c];
      fm[1][c] += py * g[c];
      fm[2][c] += pz * g[c];
      fdm[0][c] += bx * g[c];
      fdm[1][c] += by * g[c];
      fdm[2][c] += bz * g[c];
    }
  }
  M3<TL> f, fd;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      f.a[r][c] = static_cast<TL>(fm[r][c]);
      fd.a[r][c] = static_cast<TL>(fdm[r][c]);
    }
  const int sample = valid ? 8 * ec + s : -1;
  const M3<TL> stress = sample_stress<TL>(a, ec, svd_state(svd_u, sample), svd_state(svd_v, sample), warm, f, fd);
  // v[j] = stress_s g_sj for the eight corners.
  double vx[8], vy[8], vz[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const double* g = grad_smem + (8 * s + j) * 3;
    const V3<TL> c = mul(stress, v3<TL>(static_cast<TL>(g[0]), static_cast<TL>(g[1]), static_cast<TL>(g[2])));
    vx[j] = static_cast<double>(c.x);
    vy[j] = static_cast<double>(c.y);
    vz[j] = static_cast<double>(c.z);
  }
  // Reduce-scatter over the eight sample lanes: masks 4, 2, 1.
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const bool upper = (s & 4) != 0;
    const double sx = upper ? vx[t] : vx[4 + t];
    const double sy = upper ? vy[t] : vy[4 + t];
    const double sz = upper ? vz[t] : vz[4 + t];
    const double rx = __shfl_xor_sync(0xffffffffu, sx, 4);
    const double ry = __shfl_xor_sync(0xffffffffu, sy, 4);
    const double rz = __shfl_xor_sync(0xffffffffu, sz, 4);
    vx[t] = (upper ? vx[4 + t] : vx[t]) + rx;
    vy[t] = (upper ? vy[4 + t] : vy[t]) + ry;
    vz[t] = (upper ? vz[4 + t] : vz[t]) + rz;
  }
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const bool upper = (s & 2) != 0;
    const double sx = upper ? vx[t] : vx[2 + t];
    const double sy = upper ? vy[t] : vy[2 + t];
    const double sz = upper ? vz[t] : vz[2 + t];
    const double rx = __shfl_xor_sync(0xffffffffu, sx, 2);
    const double ry = __shfl_xor_sync(0xffffffffu, sy, 2);
    const double rz = __shfl_xor_sync(0xffffffffu, sz, 2);
    vx[t] = (upper ? vx[2 + t] : vx[t]) + rx;
    vy[t] = (upper ? vy[2 + t] : vy[t]) + ry;
    vz[t] = (upper ? vz[2 + t] : vz[t]) + rz;
  }
  {
    const bool upper = (s & 1) != 0;
    const double sx = upper ? vx[0] : vx[1];
    const double sy = upper ? vy[0] : vy[1];
    const double sz = upper ? vz[0] : vz[1];
    const double rx = __shfl_xor_sync(0xffffffffu, sx, 1);
    const double ry = __shfl_xor_sync(0xffffffffu, sy, 1);
    const double rz = __shfl_xor_sync(0xffffffffu, sz, 1);
    vx[0] = (upper ? vx[1] : vx[0]) + rx;
    vy[0] = (upper ? vy[1] : vy[0]) + ry;
    vz[0] = (upper ? vz[1] : vz[0]) + rz;
  }
  if (valid) {
    double* out = a.contrib + (8 * e + s) * 3;
    out[0] = vx[0];
    out[1] = vy[0];
    out[2] = vz[0];
  }
}

// P1 for Hex8: eight lanes per cell, four cells per warp, each block a
// contiguous range of cells. Every lane of a warp takes part in each pass
// (the sample reduction shuffles span the warp); lanes past the range work
// on a clamped cell and store nothing.
template <typename TL>
__device__ void local_step_hex(const StepArgs& a, const double* grad_smem, bool warm, Team team) {
  int first, last;
  team_range(a.ne, team, first, last);
  const int group = threadIdx.x >> 3;  // cell slot of this lane group in the block, 0..31
  for (int base = first; base < last; base += kBlock / 8) {
    const int e = base + group;
    hex_cell<TL>(a, grad_smem, e < last ? e : a.ne, warm, a.svd_u, a.svd_v);
  }
}

// Row-parallel CSR product out = M vec for rows [r0, r1) of this block,
// one warp per row, lanes strided over the row, fixed shuffle tree.
template <typename TV>
__device__ __forceinline__ void spmv_rows(const int* off, const int* col, const TV* val, const double* vec, double* out,
                                          int r0, int r1) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int row = r0 + warp; row < r1; row += kWarps) {
    const int begin = off[row];
    const int end = off[row + 1];
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll 4
    for (int k = begin + lane; k < end; k += 32) {
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

// Copies this block's rows of one product into shared memory (once per launch).
template <typename TV>
__device__ void load_slice(const SpmvPlan& plan, const TV* global_values, char* smem, int rank) {
  const int r0 = plan.part[rank], r1 = plan.part[rank + 1];
  const int k0 = plan.off[r0], k1 = plan.off[r1];
  const int nnz = k1 - k0, rows = r1 - r0;
  char* base = smem + plan.smem_offset;
  TV* val = reinterpret_cast<TV*>(base);
  int* col = reinterpret_cast<int*>(base + align16(plan.max_nnz * static_cast<int>(sizeof(TV))));
  int* off = col + align16(plan.max_nnz * 4) / 4;
  int* rowlist = off + align16((plan.max_rows + 1) * 4) / 4;
  const int* columns = plan.col_local != nullptr ? plan.col_local : plan.col;
  for (int k = threadIdx.x; k < nnz; k += blockDim.x) {
    val[k] = global_values[k0 + k];
    col[k] = columns[k0 + k];
  }
  for (int r = threadIdx.x; r <= rows; r += blockDim.x) off[r] = plan.off[r0 + r] - k0;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) rowlist[r] = plan.rowlist[r0 + r] - r0;
}

// Copies a particle vector [n][3] float64 into shared memory.
__device__ __forceinline__ void stage_vector(const double* vec, double* smem_vec, int n) {
  const int count = 3 * n;
  const double2* src = reinterpret_cast<const double2*>(vec);
  double2* dst = reinterpret_cast<double2*>(smem_vec);
  const int pairs = count / 2;
#pragma unroll 4
  for (int k = threadIdx.x; k < pairs; k += blockDim.x) dst[k] = src[k];
  if ((count & 1) && threadIdx.x == 0) smem_vec[count - 1] = vec[count - 1];
  __syncthreads();
}

// Stages the vector a product's slice reads into shared memory: the block's
// subset of entries (renumbered, when the plan has one) or the whole [n][3]
// vector. Ends with __syncthreads.
__device__ __forceinline__ void stage_for(const SpmvPlan& plan, int rank, const double* vec, double* smem_vec, int n) {
  if (plan.stage_cols == nullptr) {
    stage_vector(vec, smem_vec, n);
    return;
  }
  const int first = plan.stage_off[rank], count = plan.stage_off[rank + 1] - first;
  const int* cols = plan.stage_cols + first;
  for (int t = threadIdx.x; t < 3 * count; t += blockDim.x) {
    const int j = t / 3, c = t - 3 * j;
    smem_vec[t] = vec[3 * cols[j] + c];
  }
  __syncthreads();
}

// Four consecutive padded entries of a streamed row.
template <typename TV>
struct Group4;
template <>
struct Group4<float> {
  float v[4];
  __device__ __forceinline__ void load(const void* base, int g) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(base) + g);
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
  }
};
template <>
struct Group4<double> {
  double v[4];
  __device__ __forceinline__ void load(const void* base, int g) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(base) + 2 * g);
    const double2 b = __ldg(reinterpret_cast<const double2*>(base) + 2 * g + 1);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
  }
};

template <typename TV>
__device__ __forceinline__ void group_fma(const Group4<TV>& values, const int4 cols, const double* vec, double& sx,
                                          double& sy, double& sz) {
  const int c[4] = {cols.x, cols.y, cols.z, cols.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double value = static_cast<double>(values.v[k]);
    sx += value * vec[3 * c[k]];
    sy += value * vec[3 * c[k] + 1];
    sz += value * vec[3 * c[k] + 2];
  }
}

// out = M vec over the padded streaming layout (plans that are not resident):
// the same row-to-unit assignment as the resident path, four entries per
// 16-byte load, eight groups in flight per lane of a long row.
template <typename TV>
__device__ void spmv_block_streamed(const SpmvPlan& plan, const double* vec, double* out, const int* rowlist, int nshort,
                                    int rows) {
  for (int t = threadIdx.x; t < nshort; t += blockDim.x) {
    const int r = rowlist[t];
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll 4
    for (int g = plan.off4[r]; g < plan.off4[r + 1]; ++g) {
      Group4<TV> values;
      values.load(plan.val4, g);
      group_fma<TV>(values, __ldg(plan.col4 + g), vec, sx, sy, sz);
    }
    out[3 * r] = sx;
    out[3 * r + 1] = sy;
    out[3 * r + 2] = sz;
  }
  // Long rows: eight lanes per row, four rows per warp in flight, so a row of
  // a few hundred entries keeps every lane busy with several loads at once.
  const int lane = threadIdx.x & 7;
  const int slot = threadIdx.x >> 3;  // 32 row slots per block
  const int longs = rows - nshort;
  for (int base = 0; base < longs; base += kBlock / 8) {
    const int w = base + slot;
    const bool valid = w < longs;
    const int r = valid ? rowlist[nshort + w] : 0;
    const int begin = valid ? plan.off4[r] : 0;
    const int end = valid ? plan.off4[r + 1] : 0;
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll 8
    for (int g = begin + lane; g < end; g += 8) {
      Group4<TV> values;
      values.load(plan.val4, g);
      group_fma<TV>(values, __ldg(plan.col4 + g), vec, sx, sy, sz);
    }
#pragma unroll
    for (int offset = 4; offset > 0; offset >>= 1) {
      sx += __shfl_xor_sync(0xffffffffu, sx, offset);
      sy += __shfl_xor_sync(0xffffffffu, sy, offset);
      sz += __shfl_xor_sync(0xffffffffu, sz, offset);
    }
    if (valid && lane == 0) {
      out[3 * r] = sx;
      out[3 * r + 1] = sy;
      out[3 * r + 2] = sz;
    }
  }
}

// Readers of the product's input vector and writers of its output. The
// float64 pair keeps xyz triples of doubles and accumulates in double; the
// float32 pair (the refinement modes' residual products) keeps one float4
// (x, y, z, 0) per particle, a single 16-byte shared-memory load per entry,
// and accumulates in float: the residual form corrects the rounding.
struct VecF64 {
  const double* v;
  using Acc = double;
  template <typename TV>
  __device__ __forceinline__ void fma(TV value, int c, double& sx, double& sy, double& sz) const {
    const double w = static_cast<double>(value);
    sx += w * v[3 * c];
    sy += w * v[3 * c + 1];
    sz += w * v[3 * c + 2];
  }
};
struct VecF32 {
  const float4* v;
  using Acc = float;
  __device__ __forceinline__ void fma(float value, int c, float& sx, float& sy, float& sz) const {
    const float4 q = v[c];
    sx = fmaf(value, q.x, sx);
    sy = fmaf(value, q.y, sy);
    sz = fmaf(value, q.z, sz);
  }
};
struct OutF64 {
  double* o;
  template <typename A>
  __device__ __forceinline__ void store(int row, A x, A y, A z) const {
    o[3 * row] = static_cast<double>(x);
    o[3 * row + 1] = static_cast<double>(y);
    o[3 * row + 2] = static_cast<double>(z);
  }
};
struct OutF32 {
  float4* o;
  __device__ __forceinline__ void store(int row, float x, float y, float z) const { o[row] = make_float4(x, y, z, 0.0f); }
};

// Stages a float64 [n][3] vector into shared memory as float4 per particle
// (the block's subset when the plan has one).
__device__ __forceinline__ void stage_vector_f32(const SpmvPlan& plan, int rank, const double* vec, float4* smem_vec,
                                                 int n) {
  const int first = plan.stage_cols != nullptr ? plan.stage_off[rank] : 0;
  const int count = plan.stage_cols != nullptr ? plan.stage_off[rank + 1] - first : n;
  for (int j = threadIdx.x; j < count; j += blockDim.x) {
    const int i = plan.stage_cols != nullptr ? plan.stage_cols[first + j] : j;
    smem_vec[j] = make_float4(static_cast<float>(vec[3 * i]), static_cast<float>(vec[3 * i + 1]),
                              static_cast<float>(vec[3 * i + 2]), 0.0f);
  }
  __syncthreads();
}
// Copies a float4-per-particle vector into shared memory (the block's subset
// when the plan has one).
__device__ __forceinline__ void stage_float4(const SpmvPlan& plan, int rank, const float4* vec, float4* smem_vec, int n) {
  const int first = plan.stage_cols != nullptr ? plan.stage_off[rank] : 0;
  const int count = plan.stage_cols != nullptr ? plan.stage_off[rank + 1] - first : n;
#pragma unroll 4
  for (int j = threadIdx.x; j < count; j += blockDim.x)
    smem_vec[j] = vec[plan.stage_cols != nullptr ? plan.stage_cols[first + j] : j];
  __syncthreads();
}

// out = M vec for this block's rows of one resident or global CSR slice.
// Short rows (<= 32 nnz) are summed sequentially by one thread, long rows by
// one warp when a block has few of them, else by eight lanes (lane-strided,
// fixed shuffle trees); each row always by the same unit, so the result is
// bitwise reproducible. Slice data comes from shared memory when resident.
template <typename TV, typename Vec, typename Out>
__device__ void spmv_block_rows(const SpmvPlan& plan, const TV* global_values, bool resident, const char* smem,
                                const Vec vec, const Out out, int rank) {
  using Acc = typename Vec::Acc;
  const int r0 = plan.part[rank], r1 = plan.part[rank + 1];
  const int rows = r1 - r0;
  const int nshort = plan.nshort[rank];
  // Resident: row ids, offsets and entries are relative to the block's first
  // row and first entry. Global: absolute.
  const TV* val;
  const int* col;
  const int* off;
  const int* rowlist;
  int row_shift;
  if (resident) {
    const char* base = smem + plan.smem_offset;
    val = reinterpret_cast<const TV*>(base);
    col = reinterpret_cast<const int*>(base + align16(plan.max_nnz * static_cast<int>(sizeof(TV))));
    off = col + align16(plan.max_nnz * 4) / 4;
    rowlist = off + align16((plan.max_rows + 1) * 4) / 4;
    row_shift = r0;
  } else {
    val = global_values;
    col = plan.col;
    off = plan.off;
    rowlist = plan.rowlist + r0;
    row_shift = 0;
  }
  for (int t = threadIdx.x; t < nshort; t += blockDim.x) {
    const int r = rowlist[t];
    const int begin = off[r], end = off[r + 1];
    Acc sx = Acc(0), sy = Acc(0), sz = Acc(0);
    for (int k = begin; k < end; ++k) vec.fma(val[k], col[k], sx, sy, sz);
    out.store(r + row_shift, sx, sy, sz);
  }
  const int longs = rows - nshort;
  if (longs <= 4 * kWarps) {
    // Few long rows: one warp each (lane-strided, fixed shuffle tree).
    const int lane = threadIdx.x & 31;
    for (int w = nshort + (threadIdx.x >> 5); w < rows; w += kWarps) {
      const int r = rowlist[w];
      Acc sx = Acc(0), sy = Acc(0), sz = Acc(0);
#pragma unroll 4
      for (int k = off[r] + lane; k < off[r + 1]; k += 32) vec.fma(val[k], col[k], sx, sy, sz);
#pragma unroll
      for (int offset = 16; offset > 0; offset >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, offset);
        sy += __shfl_xor_sync(0xffffffffu, sy, offset);
        sz += __shfl_xor_sync(0xffffffffu, sz, offset);
      }
      if (lane == 0) out.store(r + row_shift, sx, sy, sz);
    }
    return;
  }
  // Many long rows: eight lanes per row, four rows per warp at once
  // (lane-strided entries, fixed three-level shuffle tree).
  const int lane = threadIdx.x & 7;
  const int slot = threadIdx.x >> 3;
  for (int base = 0; base < longs; base += kBlock / 8) {
    const int w = base + slot;
    const bool valid = w < longs;
    const int r = valid ? rowlist[nshort + w] : 0;
    const int begin = valid ? off[r] : 0;
    const int end = valid ? off[r + 1] : 0;
    Acc sx = Acc(0), sy = Acc(0), sz = Acc(0);
#pragma unroll 8
    for (int k = begin + lane; k < end; k += 8) vec.fma(val[k], col[k], sx, sy, sz);
#pragma unroll
    for (int offset = 4; offset > 0; offset >>= 1) {
      sx += __shfl_xor_sync(0xffffffffu, sx, offset);
      sy += __shfl_xor_sync(0xffffffffu, sy, offset);
      sz += __shfl_xor_sync(0xffffffffu, sz, offset);
    }
    if (valid && lane == 0) out.store(r + row_shift, sx, sy, sz);
  }
}

// out = M vec (float64 vectors) for this block's rows of one product; plans
// that are not resident stream the padded layout.
template <typename TV>
__device__ void spmv_block(const SpmvPlan& plan, const TV* global_values, bool resident, const char* smem,
                           const double* vec, double* out, int rank) {
  if (!resident && plan.off4 != nullptr) {
    const int r0 = plan.part[rank], r1 = plan.part[rank + 1];
    spmv_block_streamed<TV>(plan, vec, out, plan.rowlist + r0, plan.nshort[rank], r1 - r0);
    return;
  }
  spmv_block_rows<TV>(plan, global_values, resident, smem, VecF64{vec}, OutF64{out}, rank);
}

// Anderson Gram entries for history state (count, start): entries
// [0, count*(count+1)/2) are dG_a . dG_b (a <= b), then count entries dG_a . g.
__device__ __forceinline__ int gram_entries(int count) { return count * (count + 1) / 2 + count; }

__device__ __forceinline__ void gram_entry_pair(int entry, int count, int& a, int& b) {
  // Enumerate (a, b) with a <= b row by row.
  int k = entry;
  a = 0;
  while (k >= count - a) {
    k -= count - a;
    ++a;
  }
  b = a + k;
}

// Anderson history of the particle rows a block owns: slot k of row i is at
// x + k * slot_stride + 3 * (i - base) (and likewise g). Either the whole
// history in global memory (base 0, slot stride 3n) or the block's own rows in
// shared memory (base = first own row).
struct History {
  double* x;
  double* g;
  size_t slot_stride;
  int base;
  __device__ __forceinline__ double* xs(int slot, int i) const { return x + slot * slot_stride + 3 * (i - base); }
  __device__ __forceinline__ double* gs(int slot, int i) const { return g + slot * slot_stride + 3 * (i - base); }
};

// Block partial of the Gram entries over this block's particle rows [r0, r1).
inline __device__ void gram_partials(const History& h, int window, int r0, int r1, int count, int start,
                                     double* block_out, double* scratch, int blocks) {
  const int entries = gram_entries(count);
  const int capacity = window + 1;
  const int groups = entries > 0 ? kBlock / entries : 0;
  const int t = threadIdx.x;
  double sum = 0.0;
  if (entries > 0 && t < groups * entries) {
    const int entry = t % entries;
    const int group = t / entries;
    const int pairs = count * (count + 1) / 2;
    if (entry < pairs) {
      int ea, eb;
      gram_entry_pair(entry, count, ea, eb);
      const int a1 = (start + ea + 1) % capacity, a0 = (start + ea) % capacity;
      const int b1 = (start + eb + 1) % capacity, b0 = (start + eb) % capacity;
      for (int i = r0 + group; i < r1; i += groups) {
        const double* ga1 = h.gs(a1, i);
        const double* ga0 = h.gs(a0, i);
        const double* gb1 = h.gs(b1, i);
        const double* gb0 = h.gs(b0, i);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double da = ga1[c] - ga0[c];
          const double db = gb1[c] - gb0[c];
          sum += da * db;
        }
      }
    } else {
      const int ea = entry - pairs;
      const int a1 = (start + ea + 1) % capacity, a0 = (start + ea) % capacity, top = (start + count) % capacity;
      for (int i = r0 + group; i < r1; i += groups) {
        const double* ga1 = h.gs(a1, i);
        const double* ga0 = h.gs(a0, i);
        const double* gn = h.gs(top, i);
#pragma unroll
        for (int c = 0; c < 3; ++c) sum += (ga1[c] - ga0[c]) * gn[c];
      }
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

// Anderson coefficients for a history of exactly M columns: the regularised
// Gram system (anderson.py:424-447) solved by Eigen's pivoted LDL^T
// (anderson.py:357-407: largest remaining diagonal as pivot, full row and
// column swaps, pseudo-inverse of D), with every index fixed at compile time
// so the matrix lives in registers on this serial path. Returns |gamma|^2.
template <int M>
__device__ __forceinline__ double aa_coefficients(const double* reduced, double* gamma) {
  double g[M][M], b[M];
  {
    int entry = 0;
#pragma unroll
    for (int i = 0; i < M; ++i)
#pragma unroll
      for (int j = i; j < M; ++j) g[i][j] = reduced[entry++];
  }
  constexpr int pairs = M * (M + 1) / 2;
#pragma unroll
  for (int i = 0; i < M; ++i) b[i] = reduced[pairs + i];
  double trace = 0.0;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    trace += g[i][i];
#pragma unroll
    for (int j = i + 1; j < M; ++j) g[j][i] = g[i][j];
  }
  const double regularization = fmax(1.0e-6 * trace / static_cast<double>(M), 1.0e-12);
#pragma unroll
  for (int i = 0; i < M; ++i) g[i][i] = g[i][i] + regularization;
  int perm[M];
#pragma unroll
  for (int i = 0; i < M; ++i) perm[i] = i;
#pragma unroll
  for (int k = 0; k < M; ++k) {
    int biggest = k;
    double largest = fabs(g[k][k]);
#pragma unroll
    for (int i = k + 1; i < M; ++i) {
      const double value = fabs(g[i][i]);
      if (value > largest) {
        biggest = i;
        largest = value;
      }
    }
#pragma unroll
    for (int i = k + 1; i < M; ++i) {
      if (biggest == i) {
#pragma unroll
        for (int j = 0; j < M; ++j) {
          const double t = g[k][j];
          g[k][j] = g[i][j];
          g[i][j] = t;
        }
#pragma unroll
        for (int r = 0; r < M; ++r) {
          const double t = g[r][k];
          g[r][k] = g[r][i];
          g[r][i] = t;
        }
        const int t = perm[k];
        perm[k] = perm[i];
        perm[i] = t;
      }
    }
#pragma unroll
    for (int j = 0; j < k; ++j) g[k][k] = g[k][k] - g[k][j] * g[k][j] * g[j][j];
#pragma unroll
    for (int i = k + 1; i < M; ++i) {
#pragma unroll
      for (int j = 0; j < k; ++j) g[i][k] = g[i][k] - g[i][j] * g[j][j] * g[k][j];
      if (g[k][k] != 0.0) g[i][k] = g[i][k] / g[k][k];
    }
  }
  double y[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    y[i] = 0.0;
#pragma unroll
    for (int r = 0; r < M; ++r)
      if (perm[i] == r) y[i] = b[r];
  }
#pragma unroll
  for (int i = 0; i < M; ++i)
#pragma unroll
    for (int j = 0; j < i; ++j) y[i] = y[i] - g[i][j] * y[j];
#pragma unroll
  for (int i = 0; i < M; ++i) y[i] = fabs(g[i][i]) > DBL_MIN ? y[i] / g[i][i] : 0.0;
#pragma unroll
  for (int r = 0; r < M; ++r) {
    const int i = M - 1 - r;
#pragma unroll
    for (int j = i + 1; j < M; ++j) y[i] = y[i] - g[j][i] * y[j];
  }
  double norm = 0.0;
#pragma unroll
  for (int r = 0; r < M; ++r) {
    double x = 0.0;
#pragma unroll
    for (int i = 0; i < M; ++i)
      if (perm[i] == r) x = y[i];
    gamma[r] = x;
    norm += x * x;
  }
  return norm;
}

// Serial Anderson step (one thread) from the reduced Gram entries (anderson.py:424-475).
// work: unused scratch kept for the callers' signature.
__device__ __forceinline__ void aa_solve(int* state, double* gamma, int* accept, const double* reduced, int window,
                                double* work) {
  (void)work;
  int count = state[0];
  int start = state[1];
  const int capacity = window + 1;
  state[2] = count;
  state[3] = start;
  *accept = 0;
  if (count >= 1) {
    double norm = 0.0;
    switch (count) {
      case 1: norm = aa_coefficients<1>(reduced, gamma); break;
      case 2: norm = aa_coefficients<2>(reduced, gamma); break;
      case 3: norm = aa_coefficients<3>(reduced, gamma); break;
      case 4: norm = aa_coefficients<4>(reduced, gamma); break;
      case 5: norm = aa_coefficients<5>(reduced, gamma); break;
      case 6: norm = aa_coefficients<6>(reduced, gamma); break;
      case 7: norm = aa_coefficients<7>(reduced, gamma); break;
      default: norm = aa_coefficients<8>(reduced, gamma); break;
    }
    if (sqrt(norm) >= 10.0) {
      count = 0;
      start = 0;
    } else {
      *accept = 1;
      count += 1;
    }
  } else {
    count += 1;
  }
  while (count > window) {
    start = (start + 1) % capacity;
    count -= 1;
  }
  state[0] = count;
  state[1] = start;
}

// Anderson-mixed value of particle i (anderson.py:478-503), given the history
// before trimming (count_used, start_used) and the coefficients.
__device__ __forceinline__ V3<double> aa_apply_row(const History& h, int window, int i, int count, int start,
                                                   const double* gamma) {
  const int capacity = window + 1;
  const int slot = (start + count) % capacity;
  V3<double> value;
  {
    const double* hx = h.xs(slot, i);
    const double* hg = h.gs(slot, i);
#pragma unroll
    for (int c = 0; c < 3; ++c) value[c] = hx[c] + hg[c];
  }
  // Fully unrolled and predicated so every history load is issued up front.
#pragma unroll
  for (int k = 0; k < kMaxWindow; ++k) {
    if (k < count) {
      const int low = (start + k) % capacity;
      const int high = (start + k + 1) % capacity;
      const double* xh = h.xs(high, i);
      const double* xl = h.xs(low, i);
      const double* gh = h.gs(high, i);
      const double* gl = h.gs(low, i);
#pragma unroll
      for (int c = 0; c < 3; ++c) value[c] -= (xh[c] - xl[c] + gh[c] - gl[c]) * gamma[k];
    }
  }
  return value;
}

}  // namespace pdb200
