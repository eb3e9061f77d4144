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

// Right-hand sides of columns first .. first + count - 1, one [n][3] vector
// each, `pitch` doubles apart.
__global__ void woodbury_seeds_kernel(int n, const int* order, int first, int count, const int* row_node,
                                      const double* row_vector, size_t pitch, double* seeds) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<long long>(count) * n) return;
  const int k = static_cast<int>(t / n), i = static_cast<int>(t % n);
  const int row = order[first + k];
  const V3<double> value = i == row_node[row] ? load3d(row_vector, row) : v3<double>(0.0, 0.0, 0.0);
  store3(seeds + static_cast<size_t>(k) * pitch, i, value);
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

// The selected columns side by side: the solver is planned for a team of T
// blocks (T set by pd_set_woodbury_team, else from the factor's nnz, the
// element samples and the column count; the solver's own plan is set aside
// and put back), and every lane of one launch solves one column with
// its own vectors: as many lanes as the co-resident grid holds (and 8 GB of
// per-column vectors), the columns split evenly over the launches. Each
// column keeps its own stop rule, as in the sequential path.
static int woodbury_columns_team(PdSolver* s, const pdb200::AdjointArgs& column, int selected, cudaStream_t st) {
  const int n = s->n;
  int sms = 0, optin = 0, smem_per_sm = 0, per_sm = 0;
  PD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
  PD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
  PD_CUDA(cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, s->device));
  PD_CUDA(pdb200::team_columns_max_blocks(s->options.precision, 0, &per_sm));
  const int occupancy = std::max(1, std::min(per_sm, 2));
  const int grid_cap = occupancy * sms;
  const int budget = std::min(optin, smem_per_sm / occupancy) - 10 * 1024;
  const double nnz = static_cast<double>(s->factor.s.columns.size());
  const double samples = static_cast<double>(s->ne) * (s->hex ? 8 : 1);
  const double want = std::max(1.0, std::max(nnz / 65536.0, samples / 512.0));
  int team = 1;
  if (s->woodbury_team > 0) {
    team = std::min(s->woodbury_team, grid_cap);
  } else {
    // A batch's team for this instance (from nnz(S) and the samples), then
    // halved while the columns do not all fit one launch, down to an eighth
    // of it: with more columns than lanes, smaller teams finish more columns
    // per launch (measured on a 2,205-particle block with 1,323 columns:
    // teams of 2 blocks 758 ms, of 16 blocks 1,019 ms).
    while (team < 64 && team * 2 <= grid_cap && team * 1.5 < want) team *= 2;
    const int floor_team = std::max(1, team / 8);
    while (team > floor_team && static_cast<long long>(selected) * team > grid_cap) team /= 2;
  }
  // Per-column buffers. Every vector starts on a 256-byte boundary (pitch: 3n
  // rounded up to 32 doubles), as a vector of its own allocation does: the
  // products stage their input vector into shared memory with 16-byte loads.
  const size_t vec = static_cast<size_t>(3) * n;
  const size_t pitch = (vec + 31) & ~static_cast<size_t>(31);
  const size_t window = static_cast<size_t>(s->options.anderson_window) + 1;
  const size_t contrib = (static_cast<size_t>(s->ne) * s->corners * 3 + 31) & ~static_cast<size_t>(31);
  const size_t partials = static_cast<size_t>(team) * pdb200::kPartialStride;
  const size_t column_bytes = (8 * pitch + 2 * window * pitch + contrib + partials + 48) * sizeof(double);
  const size_t memory_lanes = std::max<size_t>(1, (static_cast<size_t>(8) << 30) / column_bytes);
  const int lanes_cap = static_cast<int>(std::min<size_t>(std::max(1, grid_cap / team), memory_lanes));
  const int launches = (selected + lanes_cap - 1) / lanes_cap;
  const int capacity = (selected + launches - 1) / launches;
  // Plan for the team, keep that plan's buffers for the launches, put the
  // solver's own plan back (the mode-2 pass after the columns uses it).
  SavedPlan saved;
  saved.save(s);
  TeamPlanBuffers team_plan;
  pdb200::AdjointArgs planned{};
  size_t smem = 0;
  {
    const int status = pd_plan_launch(s, team, budget);
    if (status == PD_OK) {
      fill_adjoint_args(s, &planned);
      smem = s->smem;
      team_plan.take(s);
    }
    saved.restore(s);
    if (status != PD_OK) return status;
  }
  int blocks_per_sm = 0;
  PD_CUDA(pdb200::team_columns_max_blocks(s->options.precision, smem, &blocks_per_sm));
  if (blocks_per_sm < 1 || capacity * team > blocks_per_sm * sms)
    return pd_set_error(PD_ERR_CUDA, "the column lanes do not fit the co-resident grid");
  // The column's arguments with the team plan's product layout.
  pdb200::AdjointArgs base = column;
  base.s_part = planned.s_part;
  base.st_part = planned.st_part;
  base.plan_s = planned.plan_s;
  base.plan_st = planned.plan_st;
  base.resident = planned.resident;
  base.stage_vector = planned.stage_vector;
  base.vector_smem_offset = planned.vector_smem_offset;
  // Per-column buffers for `capacity` columns.
  const auto ensure = [](DeviceBuffer& buffer, size_t bytes) -> cudaError_t {
    return buffer.bytes >= bytes ? cudaSuccess : buffer.allocate(bytes);
  };
  const size_t slots = static_cast<size_t>(capacity);
  PD_CUDA(ensure(s->w_team_args, slots * sizeof(pdb200::AdjointArgs)));
  PD_CUDA(ensure(s->w_team_lane_start, (slots + 1) * sizeof(int)));
  PD_CUDA(ensure(s->w_team_lane_class, slots * sizeof(int)));
  PD_CUDA(ensure(s->w_team_class_begin, 2 * sizeof(int)));
  PD_CUDA(ensure(s->w_team_class_order, slots * sizeof(int)));
  PD_CUDA(ensure(s->w_team_class_head, sizeof(unsigned)));
  PD_CUDA(ensure(s->w_team_lane_slot, slots * sizeof(int)));
  PD_CUDA(ensure(s->w_team_barriers, slots * sizeof(pdb200::GridBarrier)));
  PD_CUDA(ensure(s->w_team_vectors, slots * 7 * pitch * sizeof(double)));
  PD_CUDA(ensure(s->w_team_hist, slots * 2 * window * pitch * sizeof(double)));
  PD_CUDA(ensure(s->w_team_contrib, slots * contrib * sizeof(double)));
  PD_CUDA(ensure(s->w_team_ints, slots * 32 * sizeof(int)));
  PD_CUDA(ensure(s->w_team_doubles, slots * 16 * sizeof(double)));
  PD_CUDA(ensure(s->w_team_partials, slots * partials * sizeof(double)));
  PD_CUDA(ensure(s->w_team_seeds, slots * pitch * sizeof(double)));
  std::vector<int> lane_start(capacity + 1), lane_class(capacity, 0), order(capacity);
  for (int k = 0; k <= capacity; ++k) lane_start[k] = k * team;
  for (int k = 0; k < capacity; ++k) order[k] = k;
  PD_CUDA(cudaMemcpy(s->w_team_lane_start.ptr, lane_start.data(), lane_start.size() * sizeof(int),
                     cudaMemcpyHostToDevice));
  PD_CUDA(cudaMemcpy(s->w_team_lane_class.ptr, lane_class.data(), lane_class.size() * sizeof(int),
                     cudaMemcpyHostToDevice));
  PD_CUDA(cudaMemcpy(s->w_team_class_order.ptr, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
  double* vectors = s->w_team_vectors.as<double>();
  double* hist = s->w_team_hist.as<double>();
  int* ints = s->w_team_ints.as<int>();
  double* doubles = s->w_team_doubles.as<double>();
  std::vector<pdb200::AdjointArgs> args(capacity);
  for (int first = 0; first < selected; first += capacity) {
    const int count = std::min(capacity, selected - first);
    const long long entries = static_cast<long long>(count) * n;
    pdb200::woodbury_seeds_kernel<<<static_cast<unsigned>((entries + 255) / 256), 256, 0, st>>>(
        n, s->w_order.as<int>(), first, count, s->w_row_node.as<int>(), s->w_row_vector.as<double>(), pitch,
        s->w_team_seeds.as<double>());
    PD_CUDA(cudaGetLastError());
    for (int k = 0; k < count; ++k) {
      pdb200::AdjointArgs& a = args[k];
      a = base;
      double* v = vectors + static_cast<size_t>(k) * 7 * pitch;
      a.rhs = v;
      a.base = v + pitch;
      a.prev = v + 2 * pitch;
      a.work = v + 3 * pitch;
      a.y = v + 4 * pitch;
      a.raw = v + 5 * pitch;
      a.solution = v + 6 * pitch;
      a.seed = s->w_team_seeds.as<double>() + static_cast<size_t>(k) * pitch;
      a.hist_x = hist + static_cast<size_t>(k) * 2 * window * pitch;
      a.hist_g = a.hist_x + window * pitch;
      a.contrib = s->w_team_contrib.as<double>() + static_cast<size_t>(k) * contrib;
      // 32 ints a column: Anderson state [8], accept, iteration, active, control [8] at 16.
      a.aa_state = ints + 32 * k;
      a.aa_accept = ints + 32 * k + 8;
      a.iteration = ints + 32 * k + 9;
      a.active = ints + 32 * k + 10;
      a.control_i = ints + 32 * k + 16;
      // 16 doubles a column: Anderson coefficients [kMaxWindow = 8], control [8].
      a.aa_gamma = doubles + 16 * k;
      a.control_d = doubles + 16 * k + pdb200::kMaxWindow;
      a.partials = s->w_team_partials.as<double>() + static_cast<size_t>(k) * partials;
    }
    const int class_begin[2] = {0, count};
    PD_CUDA(cudaMemcpyAsync(s->w_team_args.ptr, args.data(), count * sizeof(pdb200::AdjointArgs),
                            cudaMemcpyHostToDevice, st));
    PD_CUDA(cudaMemcpyAsync(s->w_team_class_begin.ptr, class_begin, sizeof(class_begin), cudaMemcpyHostToDevice, st));
    PD_CUDA(cudaMemsetAsync(s->w_team_class_head.ptr, 0, sizeof(unsigned), st));
    PD_CUDA(cudaMemsetAsync(s->w_team_barriers.ptr, 0, count * sizeof(pdb200::GridBarrier), st));
    pdb200::TeamLaunch launch{};
    launch.adjoint = s->w_team_args.as<pdb200::AdjointArgs>();
    launch.lane_start = s->w_team_lane_start.as<int>();
    launch.lane_class = s->w_team_lane_class.as<int>();
    launch.class_begin = s->w_team_class_begin.as<int>();
    launch.class_order = s->w_team_class_order.as<int>();
    launch.count = count;
    launch.lanes = count;
    launch.solo_class = -1;
    launch.class_head = s->w_team_class_head.as<unsigned>();
    launch.lane_slot = s->w_team_lane_slot.as<int>();
    launch.lane_barrier = s->w_team_barriers.as<pdb200::GridBarrier>();
    launch.status = s->d_status.as<int>();
    PD_CUDA(pdb200::launch_team_columns(launch, count * team, s->options.precision, smem, st));
    // The solutions into the [selected][n][3] columns the projection reads.
    PD_CUDA(cudaMemcpy2DAsync(s->w_columns.as<double>() + static_cast<size_t>(first) * vec, vec * sizeof(double),
                              vectors + 6 * pitch, 7 * pitch * sizeof(double), vec * sizeof(double), count,
                              cudaMemcpyDeviceToDevice, st));
    // The host argument blocks and class range are reused by the next chunk.
    PD_CUDA(cudaStreamSynchronize(st));
  }
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
  if (selected >= 2 && s->woodbury_lanes) {
    // Side by side on lanes of one launch, as the reference's column batches.
    if (int status = woodbury_columns_team(s, column, selected, st)) return status;
  } else {
    for (int k = 0; k < selected; ++k) {
      pdb200::woodbury_seed_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, s->w_order.as<int>(), k,
                                                                    s->w_row_node.as<int>(),
                                                                    s->w_row_vector.as<double>(),
                                                                    s->w_seed.as<double>());
      PD_CUDA(cudaMemsetAsync(s->d_barrier.ptr, 0, sizeof(pdb200::GridBarrier), st));
      PD_CUDA(pdb200::launch_adjoint_step(column, s->blocks, s->options.precision, s->smem, st));
      PD_CUDA(cudaMemcpyAsync(s->w_columns.as<double>() + static_cast<size_t>(k) * 3 * n, s->b_solution.ptr, vec,
                              cudaMemcpyDeviceToDevice, st));
    }
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
