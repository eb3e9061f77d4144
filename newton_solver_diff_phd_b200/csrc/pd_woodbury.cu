// Contact projection of the parameter gradients (Adjoint._woodbury,
// adjoint.py:1272-1354): with the frictional boundary of the recorded step,
// the material and activation gradients use z = mu - W_T G^{-1} (J mu)
// instead of mu, where J holds the rows omega n (and, with friction, the two
// tangents) of the active contacts (lambda > 0, omega >= 0.5), rows with
// |J mu| below max(1e-12, 1e-3 max |J mu|) are dropped, every column of
// W_T = (A - K)^{-1} J^T is the adjoint fixed point from a zero start capped
// at min(max_iterations, 120) iterations, and G = J W_T. State gradients keep
// mu, as in the reference.
//
// Passes: the adjoint kernel for mu and the state gradients; one block
// selects the rows; one adjoint fixed point per selected row (each column
// stops on its own rule, as in the reference's batched columns); one block
// forms G, solves it with the pivoted LDL^T and writes the clipped z; the
// adjoint kernel computes the parameter gradients of z.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>

#include "../../include/pd_b200.h"
#include "pd_friction.cuh"
#include "pd_kernels.h"
#include "solver_state.h"

namespace pdb200 {
namespace {

constexpr int kWoodburyMaxIterations = 120;
constexpr double kWoodburyClip = 1.0e6;

// _backward_tangents (adjoint.py:322-344).
__device__ void backward_tangents(V3<double> n, V3<double>& t1, V3<double>& t2) {
  int axis = 0;
  for (int d = 1; d < 3; ++d)
    if (fabs(n[d]) < fabs(n[axis])) axis = d;
  V3<double> unit = v3<double>(0.0, 0.0, 0.0);
  unit[axis] = 1.0;
  t1 = unit - dot(n, unit) * n;
  double norm = sqrt(dot(t1, t1));
  t1 = norm > 1.0e-12 ? v3<double>(t1.x / norm, t1.y / norm, t1.z / norm) : v3<double>(1.0, 0.0, 0.0);
  t2 = cross(n, t1);
  norm = sqrt(dot(t2, t2));
  t2 = norm > 1.0e-12 ? v3<double>(t2.x / norm, t2.y / norm, t2.z / norm) : v3<double>(0.0, 1.0, 0.0);
}

// _basis, _project_rows, _select_rows, _compact_rows (adjoint.py:347-415) in one block.
__global__ void woodbury_rows_kernel(const int* nodes, const double* multiplier, const double* omega,
                                     const double* normal, int count, int tangents, const int* diverged,
                                     const double* mu, int* row_node, double* row_vector, double* value,
                                     int* selected, int* order, int* selected_count) {
  __shared__ double s_largest[kWarps];
  const int rows = count * (tangents ? 3 : 1);
  const bool ok = *diverged == 0;
  double largest = 0.0;
  for (int c = threadIdx.x; c < count; c += blockDim.x) {
    const int node = nodes[c];
    const V3<double> n = load3d(normal, c);
    const bool active = ok && multiplier[c] > 0.0 && omega[c] >= 0.5;
    const V3<double> vector = omega[c] * n;
    row_node[c] = node;
    store3(row_vector, c, vector);
    const V3<double> z = load3d(mu, node);
    value[c] = active ? dot(vector, z) : 0.0;
    selected[c] = active ? 1 : 0;  // valid; the gate below refines it
    if (active) largest = fmax(largest, fabs(value[c]));
    if (tangents) {
      V3<double> t1, t2;
      backward_tangents(n, t1, t2);
      const bool valid = active && multiplier[c] > 1.0e-8;
      for (int r = 0; r < 2; ++r) {
        const int row = count + 2 * c + r;
        const V3<double> t = r == 0 ? t1 : t2;
        row_node[row] = node;
        store3(row_vector, row, t);
        value[row] = valid ? dot(t, z) : 0.0;
        selected[row] = valid ? 1 : 0;
        if (valid) largest = fmax(largest, fabs(value[row]));
      }
    }
  }
  for (int offset = 16; offset > 0; offset >>= 1) largest = fmax(largest, __shfl_xor_sync(0xffffffffu, largest, offset));
  if ((threadIdx.x & 31) == 0) s_largest[threadIdx.x >> 5] = largest;
  __syncthreads();
  double total = 0.0;
  for (int w = 0; w < kWarps; ++w) total = fmax(total, s_largest[w]);
  const double gate = fmax(1.0e-12, 1.0e-3 * total);
  __syncthreads();
  for (int r = threadIdx.x; r < rows; r += blockDim.x) selected[r] = selected[r] != 0 && fabs(value[r]) >= gate;
  __syncthreads();
  if (threadIdx.x == 0) {
    int k = 0;
    for (int r = 0; r < rows; ++r)
      if (selected[r]) order[k++] = r;
    *selected_count = k;
  }
}

// Right-hand side of column k: the row vector at its particle (_batch_setup, adjoint.py:667-689).
__global__ void woodbury_seed_kernel(int n, const int* order, int k, const int* row_node, const double* row_vector,
                                     double* seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int row = order[k];
  const V3<double> value = i == row_node[row] ? load3d(row_vector, row) : v3<double>(0.0, 0.0, 0.0);
  store3(seed, i, value);
}

// _gram, ldlt_solve, _scatter_alpha, _project_adjoint and _safe_clip of z
// (adjoint.py:418-471, :184-223) in one block. columns[k] is the column of
// the k-th selected row.
__global__ void woodbury_project_kernel(int n, const int* free_, const double* mu, const double* columns,
                                        const int* order, const int* selected_count, const int* row_node,
                                        const double* row_vector, const double* value, double* gram,
                                        double* coefficients, int* permutation, double* work, double* z,
                                        int* status) {
  __shared__ double s_scratch[kBlock];
  __shared__ double s_scale;
  const int count = *selected_count;
  const size_t stride = static_cast<size_t>(3) * n;
  for (long long t = threadIdx.x; t < static_cast<long long>(count) * count; t += blockDim.x) {
    const int i = static_cast<int>(t / count), j = static_cast<int>(t % count);
    // The lower triangle in original row order: G(l, k) = J_l . W_T[k] at l's particle.
    const int high = order[max(i, j)];
    const int low = min(i, j);
    const double* column = columns + low * stride;
    gram[t] = dot(load3d(row_vector, high), load3d(column, row_node[high]));
    if (j == 0) coefficients[i] = value[order[i]];
  }
  __syncthreads();
  if (count > 0) fb_ldlt_solve(gram, count, count, coefficients, permutation, work);
  double norm2 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    V3<double> v = load3d(mu, i);
    for (int k = 0; k < count; ++k) v = v - coefficients[k] * load3d(columns + k * stride, i);
    if (free_[i] == 0) v = v3<double>(0.0, 0.0, 0.0);
    for (int c = 0; c < 3; ++c) {
      if (!isfinite(v[c])) {
        v[c] = 0.0;
        atomicOr(status, kStatusAdjointSafeguard);
      }
    }
    store3(z, i, v);
    norm2 += dot(v, v);
  }
  norm2 = block_sum(norm2, s_scratch);
  if (threadIdx.x == 0) {
    const double length = sqrt(norm2);
    s_scale = 1.0;
    if (isfinite(length) && length > kWoodburyClip) {
      s_scale = kWoodburyClip / length;
      atomicOr(status, kStatusAdjointSafeguard);
    }
  }
  __syncthreads();
  if (s_scale != 1.0) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) store3(z, i, s_scale * load3d(z, i));
  }
}

}  // namespace
}  // namespace pdb200

// Buffers of the projection, sized by the registered contacts.
static int ensure_woodbury_buffers(PdSolver* s, int rows) {
  if (s->w_rows >= rows && s->w_seed.ptr != nullptr) return PD_OK;
  const size_t r = static_cast<size_t>(std::max(rows, 1));
  const size_t vec = static_cast<size_t>(3) * s->n * sizeof(double);
  PD_CUDA(s->w_row_node.allocate(r * sizeof(int)));
  PD_CUDA(s->w_row_vector.allocate(3 * r * sizeof(double)));
  PD_CUDA(s->w_value.allocate(r * sizeof(double)));
  PD_CUDA(s->w_selected.allocate(r * sizeof(int)));
  PD_CUDA(s->w_order.allocate(r * sizeof(int)));
  PD_CUDA(s->w_control.allocate(4 * sizeof(int)));
  PD_CUDA(s->w_columns.allocate(r * vec));
  PD_CUDA(s->w_gram.allocate(r * r * sizeof(double)));
  PD_CUDA(s->w_coefficients.allocate(r * sizeof(double)));
  PD_CUDA(s->w_permutation.allocate(r * sizeof(int)));
  PD_CUDA(s->w_work.allocate(r * sizeof(double)));
  PD_CUDA(s->w_seed.allocate(vec));
  PD_CUDA(s->w_mu.allocate(vec));
  s->w_rows = rows;
  return PD_OK;
}

int pd_woodbury_gradients(PdSolver* s, const pdb200::AdjointArgs& full, const double* multiplier, const double* omega,
                          const double* normal, cudaStream_t st) {
  const int count = s->fc.count;
  const int tangents = s->fc.friction > 0.0 ? 1 : 0;
  const int rows = count * (tangents ? 3 : 1);
  if (int status = ensure_woodbury_buffers(s, rows)) return status;
  const int n = s->n;
  const size_t vec = static_cast<size_t>(3) * n * sizeof(double);
  PD_CUDA(cudaMemcpyAsync(s->w_mu.ptr, s->b_solution.ptr, vec, cudaMemcpyDeviceToDevice, st));
  int* control = s->w_control.as<int>();  // [0] selected rows, [1] iteration, [2] active
  pdb200::woodbury_rows_kernel<<<1, pdb200::kBlock, 0, st>>>(
      s->fc_nodes.as<int>(), multiplier, omega, normal, count, tangents, s->b_control_i.as<int>(),
      s->w_mu.as<double>(), s->w_row_node.as<int>(), s->w_row_vector.as<double>(), s->w_value.as<double>(),
      s->w_selected.as<int>(), s->w_order.as<int>(), control);
  PD_CUDA(cudaGetLastError());
  // One read per backward step: only the selected rows need columns (adjoint.py:1300-1307).
  int selected = 0;
  PD_CUDA(cudaMemcpyAsync(&selected, control, sizeof(int), cudaMemcpyDeviceToHost, st));
  PD_CUDA(cudaStreamSynchronize(st));
  pdb200::AdjointArgs column = full;
  column.mode = 1;
  column.seed = s->w_seed.as<double>();
  column.reuse_jacobian = 1;
  column.max_iterations = std::min(s->options.max_iterations, pdb200::kWoodburyMaxIterations);
  column.iteration = control + 1;
  column.active = control + 2;
  for (int k = 0; k < selected; ++k) {
    pdb200::woodbury_seed_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, s->w_order.as<int>(), k, s->w_row_node.as<int>(),
                                                                  s->w_row_vector.as<double>(), s->w_seed.as<double>());
    PD_CUDA(cudaMemsetAsync(s->d_barrier.ptr, 0, sizeof(pdb200::GridBarrier), st));
    PD_CUDA(pdb200::launch_adjoint_step(column, s->blocks, s->options.precision, s->smem, st));
    PD_CUDA(cudaMemcpyAsync(s->w_columns.as<double>() + static_cast<size_t>(k) * 3 * n, s->b_solution.ptr, vec,
                            cudaMemcpyDeviceToDevice, st));
  }
  pdb200::woodbury_project_kernel<<<1, pdb200::kBlock, 0, st>>>(
      n, s->d_free.as<int>(), s->w_mu.as<double>(), s->w_columns.as<double>(), s->w_order.as<int>(), control,
      s->w_row_node.as<int>(), s->w_row_vector.as<double>(), s->w_value.as<double>(), s->w_gram.as<double>(),
      s->w_coefficients.as<double>(), s->w_permutation.as<int>(), s->w_work.as<double>(), s->b_solution.as<double>(),
      s->d_status.as<int>());
  PD_CUDA(cudaGetLastError());
  pdb200::AdjointArgs parameters = full;
  parameters.mode = 2;
  parameters.reuse_jacobian = 1;
  parameters.iteration = control + 1;
  parameters.active = control + 2;
  PD_CUDA(cudaMemsetAsync(s->d_barrier.ptr, 0, sizeof(pdb200::GridBarrier), st));
  PD_CUDA(pdb200::launch_adjoint_step(parameters, s->blocks, s->options.precision, s->smem, st));
  return PD_OK;
}
