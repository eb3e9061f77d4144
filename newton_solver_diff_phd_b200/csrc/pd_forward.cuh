// Phases of the forward projective-dynamics step (one persistent launch).
//
// Per iteration (reference: SolverDiffPhD._iterate, solver.py:582-659):
//   P1 local step       elements -> contributions          (kernels.py:222-272, hex.py:122-169)
//   P2 gather + rhs     particles: p, b = m/h^2 q~ + p       (kernels.py:75-91, hex.py:246-260, :275-284)
//   P3 y = S b          S rows, nnz-balanced block ranges    (sparse.py:209-227)
//   P4 x = S^T y        S^T rows + Dirichlet values + Anderson history and Gram partials
//                       (sparse.py:341-348, kernels.py:287-291, anderson.py:306-354)
//   serial              Anderson least squares in the last-arriving block (anderson.py:410-475)
//   P5 Anderson apply + convergence partials                 (anderson.py:478-503, kernels.py:354-401)
//   serial              dual convergence gate, loop decision
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

// P1 for Tet4: one thread per element. Element e belongs to block
// e % blocks: the local step is spread over every SM instead of filling the
// first ones.
template <typename TL>
__device__ void local_step_tet(const StepArgs& a, bool warm, Team team) {
  const int gthreads = team.size * blockDim.x;
  for (int e = threadIdx.x * team.size + team.rank; e < a.ne; e += gthreads) tet_element<TL>(a, e, warm, a.svd_u, a.svd_v);
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

// P1 for Hex8: eight lanes per cell, four cells per warp. Cell groups are
// interleaved over the team's blocks (group g lives in block g % blocks).
template <typename TL>
__device__ void local_step_hex(const StepArgs& a, const double* grad_smem, bool warm, Team team) {
  const int lane = threadIdx.x & 31;
  const int group_in_warp = lane >> 3;
  const int warps_total = (team.size * blockDim.x) >> 5;
  const int warp_in_block = threadIdx.x >> 5;
  for (int base = (warp_in_block * team.size + team.rank) * 4; base < a.ne; base += warps_total * 4) {
    hex_cell<TL>(a, grad_smem, base + group_in_warp, warm, a.svd_u, a.svd_v);
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
  for (int k = threadIdx.x; k < nnz; k += blockDim.x) {
    val[k] = global_values[k0 + k];
    col[k] = plan.col[k0 + k];
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

// out = M vec for this block's rows of one product. Short rows (<= 32 nnz)
// are summed sequentially by one thread, long rows by one warp when a block has
// few of them, else by eight lanes (lane-strided, fixed shuffle trees); each
// row always by the same unit, so the result is
// bitwise reproducible. Slice data comes from shared memory when resident.
template <typename TV>
__device__ void spmv_block(const SpmvPlan& plan, const TV* global_values, bool resident, const char* smem,
                           const double* vec, double* out, int rank) {
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
    if (plan.off4 != nullptr) {
      spmv_block_streamed<TV>(plan, vec, out, plan.rowlist + r0, nshort, rows);
      return;
    }
    val = global_values;
    col = plan.col;
    off = plan.off;
    rowlist = plan.rowlist + r0;
    row_shift = 0;
  }
  for (int t = threadIdx.x; t < nshort; t += blockDim.x) {
    const int r = rowlist[t];
    const int begin = off[r], end = off[r + 1];
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int k = begin; k < end; ++k) {
      const double value = static_cast<double>(val[k]);
      const int c = col[k];
      sx += value * vec[3 * c];
      sy += value * vec[3 * c + 1];
      sz += value * vec[3 * c + 2];
    }
    const int row = r + row_shift;
    out[3 * row] = sx;
    out[3 * row + 1] = sy;
    out[3 * row + 2] = sz;
  }
  const int longs = rows - nshort;
  if (longs <= 4 * kWarps) {
    // Few long rows: one warp each (lane-strided, fixed shuffle tree).
    const int lane = threadIdx.x & 31;
    for (int w = nshort + (threadIdx.x >> 5); w < rows; w += kWarps) {
      const int r = rowlist[w];
      double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll 4
      for (int k = off[r] + lane; k < off[r + 1]; k += 32) {
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
        const int row = r + row_shift;
        out[3 * row] = sx;
        out[3 * row + 1] = sy;
        out[3 * row + 2] = sz;
      }
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
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll 8
    for (int k = begin + lane; k < end; k += 8) {
      const double value = static_cast<double>(val[k]);
      const int c = col[k];
      sx += value * vec[3 * c];
      sy += value * vec[3 * c + 1];
      sz += value * vec[3 * c + 2];
    }
#pragma unroll
    for (int offset = 4; offset > 0; offset >>= 1) {
      sx += __shfl_xor_sync(0xffffffffu, sx, offset);
      sy += __shfl_xor_sync(0xffffffffu, sy, offset);
      sz += __shfl_xor_sync(0xffffffffu, sz, offset);
    }
    if (valid && lane == 0) {
      const int row = r + row_shift;
      out[3 * row] = sx;
      out[3 * row + 1] = sy;
      out[3 * row + 2] = sz;
    }
  }
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

// Block partial of the Gram entries over this block's particle rows [r0, r1).
inline __device__ void gram_partials(const StepArgs& a, int r0, int r1, int count, int start, double* block_out,
                              double* scratch, int blocks) {
  const int entries = gram_entries(count);
  const int capacity = a.window + 1;
  const int groups = entries > 0 ? kBlock / entries : 0;
  const int t = threadIdx.x;
  double sum = 0.0;
  if (entries > 0 && t < groups * entries) {
    const int entry = t % entries;
    const int group = t / entries;
    const int pairs = count * (count + 1) / 2;
    const size_t stride = static_cast<size_t>(3) * a.n;
    if (entry < pairs) {
      int ea, eb;
      gram_entry_pair(entry, count, ea, eb);
      const double* ga1 = a.hist_g + ((start + ea + 1) % capacity) * stride;
      const double* ga0 = a.hist_g + ((start + ea) % capacity) * stride;
      const double* gb1 = a.hist_g + ((start + eb + 1) % capacity) * stride;
      const double* gb0 = a.hist_g + ((start + eb) % capacity) * stride;
      for (int i = r0 + group; i < r1; i += groups) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double da = ga1[3 * i + c] - ga0[3 * i + c];
          const double db = gb1[3 * i + c] - gb0[3 * i + c];
          sum += da * db;
        }
      }
    } else {
      const int ea = entry - pairs;
      const double* ga1 = a.hist_g + ((start + ea + 1) % capacity) * stride;
      const double* ga0 = a.hist_g + ((start + ea) % capacity) * stride;
      const double* gn = a.hist_g + ((start + count) % capacity) * stride;
      for (int i = r0 + group; i < r1; i += groups) {
#pragma unroll
        for (int c = 0; c < 3; ++c) sum += (ga1[3 * i + c] - ga0[3 * i + c]) * gn[3 * i + c];
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

// Eigen-style pivoted LDL^T solve of the leading n x n block (anderson.py:357-407).
// m, y and perm live in shared memory (work): dynamic indexing of local arrays
// would put them in local memory, a global-latency round trip per access.
inline __device__ void aa_ldlt_solve(double (*m)[kMaxWindow], const double* b, int n, double* x, double* work) {
  double* y = work;
  int* perm = reinterpret_cast<int*>(work + kMaxWindow);
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int k = 0; k < n; ++k) {
    int biggest = k;
    for (int i = k + 1; i < n; ++i)
      if (fabs(m[i][i]) > fabs(m[biggest][biggest])) biggest = i;
    if (biggest != k) {
      for (int j = 0; j < n; ++j) {
        const double t = m[k][j];
        m[k][j] = m[biggest][j];
        m[biggest][j] = t;
      }
      for (int i = 0; i < n; ++i) {
        const double t = m[i][k];
        m[i][k] = m[i][biggest];
        m[i][biggest] = t;
      }
      const int t = perm[k];
      perm[k] = perm[biggest];
      perm[biggest] = t;
    }
    for (int j = 0; j < k; ++j) m[k][k] = m[k][k] - m[k][j] * m[k][j] * m[j][j];
    for (int i = k + 1; i < n; ++i) {
      for (int j = 0; j < k; ++j) m[i][k] = m[i][k] - m[i][j] * m[j][j] * m[k][j];
      if (m[k][k] != 0.0) m[i][k] = m[i][k] / m[k][k];
    }
  }
  for (int i = 0; i < n; ++i) y[i] = b[perm[i]];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) y[i] = y[i] - m[i][j] * y[j];
  for (int i = 0; i < n; ++i) y[i] = fabs(m[i][i]) > DBL_MIN ? y[i] / m[i][i] : 0.0;
  for (int r = 0; r < n; ++r) {
    const int i = n - 1 - r;
    for (int j = i + 1; j < n; ++j) y[i] = y[i] - m[j][i] * y[j];
  }
  for (int i = 0; i < n; ++i) x[perm[i]] = y[i];
}

// Serial Anderson step (one thread) from the reduced Gram entries (anderson.py:424-475).
// work: shared memory of at least 2 * kMaxWindow * kMaxWindow doubles.
inline __device__ void aa_solve(int* state, double* gamma, int* accept, const double* reduced, int window,
                                double* work) {
  int count = state[0];
  int start = state[1];
  const int capacity = window + 1;
  state[2] = count;
  state[3] = start;
  *accept = 0;
  if (count >= 1) {
    double (*gram)[kMaxWindow] = reinterpret_cast<double (*)[kMaxWindow]>(work);
    double* rhs = work + kMaxWindow * kMaxWindow;
    double* coefficients = rhs + kMaxWindow;
    const int pairs = count * (count + 1) / 2;
    int entry = 0;
    for (int i = 0; i < count; ++i)
      for (int j = i; j < count; ++j) gram[i][j] = reduced[entry++];
    for (int i = 0; i < count; ++i) rhs[i] = reduced[pairs + i];
    double trace = 0.0;
    for (int i = 0; i < count; ++i) {
      trace += gram[i][i];
      for (int j = i + 1; j < count; ++j) gram[j][i] = gram[i][j];
    }
    const double regularization = fmax(1.0e-6 * trace / static_cast<double>(count), 1.0e-12);
    for (int i = 0; i < count; ++i) gram[i][i] = gram[i][i] + regularization;
    aa_ldlt_solve(gram, rhs, count, coefficients, coefficients + kMaxWindow);
    double norm = 0.0;
    for (int i = 0; i < count; ++i) {
      gamma[i] = coefficients[i];
      norm += coefficients[i] * coefficients[i];
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
__device__ __forceinline__ V3<double> aa_apply_row(const StepArgs& a, int i, int count, int start,
                                                   const double* gamma) {
  const int capacity = a.window + 1;
  const size_t stride = static_cast<size_t>(3) * a.n;
  const int slot = (start + count) % capacity;
  const double* hx = a.hist_x + 3 * static_cast<size_t>(i);
  const double* hg = a.hist_g + 3 * static_cast<size_t>(i);
  V3<double> value;
#pragma unroll
  for (int c = 0; c < 3; ++c) value[c] = hx[slot * stride + c] + hg[slot * stride + c];
  // Fully unrolled and predicated so every history load is issued up front.
#pragma unroll
  for (int k = 0; k < kMaxWindow; ++k) {
    if (k < count) {
      const int low = (start + k) % capacity;
      const int high = (start + k + 1) % capacity;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t h = high * stride + c;
        const size_t l = low * stride + c;
        value[c] -= (hx[h] - hx[l] + hg[h] - hg[l]) * gamma[k];
      }
    }
  }
  return value;
}

}  // namespace pdb200
