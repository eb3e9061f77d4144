// Host side of the frictional boundary (contact.py FrictionalContact:
// constructor validation :684-770, build :775-795): registered vertices,
// boundary description, per-contact device buffers, and the panel
// A^{-1}[:, nodes] formed from the built factor three columns per product.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/pd_b200.h"
#include "pd_kernels.h"
#include "solver_state.h"

namespace pdb200 {
namespace {

// rhs[3 nodes[first + c] + c] = 1 for c = 0, 1, 2: three unit columns in the three coordinates.
__global__ void unit_columns_kernel(const int* nodes, int count, int first, double* rhs) {
  const int c = threadIdx.x;
  if (c < 3 && first + c < count) rhs[3 * nodes[first + c] + c] = 1.0;
}

// panel[i][first + c] = out[3 i + c].
__global__ void scatter_panel_kernel(const double* out, int n, int count, int first, double* panel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 3 && first + c < count; ++c) panel[static_cast<long long>(i) * count + first + c] = out[3 * i + c];
}

// block[i][j] = panel[nodes[i]][j] (_gather_block, contact.py:159-162).
__global__ void gather_block_kernel(const double* panel, const int* nodes, int count, double* block) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<long long>(count) * count) return;
  const int i = static_cast<int>(t / count), j = static_cast<int>(t % count);
  block[t] = panel[static_cast<long long>(nodes[i]) * count + j];
}

}  // namespace
}  // namespace pdb200

int pd_build_frictional_panel(PdSolver* s) {
  const int k = s->fc.count;
  if (k == 0) return PD_OK;
  const int n = s->n;
  const size_t vector_bytes = static_cast<size_t>(3) * n * sizeof(double);
  double* rhs = s->d_rhs.as<double>();
  double* out = s->d_prev.as<double>();
  double* panel = s->fc_panel.as<double>();
  for (int first = 0; first < k; first += 3) {
    PD_CUDA(cudaMemset(rhs, 0, vector_bytes));
    pdb200::unit_columns_kernel<<<1, 32>>>(s->fc_nodes.as<int>(), k, first, rhs);
    PD_CUDA(pdb200::launch_apply_inverse(s->d_s_off.as<int>(), s->d_s_col.as<int>(), s->d_s_val.as<double>(),
                                         s->d_st_off.as<int>(), s->d_st_col.as<int>(), s->d_st_val.as<double>(), n,
                                         rhs, s->d_y.as<double>(), out, nullptr));
    pdb200::scatter_panel_kernel<<<(n + 255) / 256, 256>>>(out, n, k, first, panel);
  }
  const long long entries = static_cast<long long>(k) * k;
  pdb200::gather_block_kernel<<<static_cast<unsigned>((entries + 255) / 256), 256>>>(panel, s->fc_nodes.as<int>(), k,
                                                                                    s->fc_block.as<double>());
  PD_CUDA(cudaGetLastError());
  // A factor change starts the multipliers afresh (contact.py:794-795).
  PD_CUDA(cudaMemset(s->fc_multiplier.ptr, 0, static_cast<size_t>(k) * sizeof(double)));
  PD_CUDA(cudaDeviceSynchronize());
  return PD_OK;
}

extern "C" {

int pd_set_frictional_boundary(PdSolver* s, int32_t kind, const double parameters[4], int32_t count,
                               const int32_t* nodes, double friction, double restitution, int32_t split,
                               int32_t n_left, const int32_t* faces_left, int32_t n_right,
                               const int32_t* faces_right) {
  if (s == nullptr || parameters == nullptr) return pd_set_error(PD_ERR_INVALID, "null argument");
  if (kind != PD_BOUNDARY_PLANAR && kind != PD_BOUNDARY_SPHERICAL && kind != PD_BOUNDARY_MESH)
    return pd_set_error(PD_ERR_INVALID, "frictional boundary must be 'planar', 'spherical' or 'mesh'");
  if (s->hex)
    return pd_set_error(PD_ERR_UNSUPPORTED, "Hex8 currently supports planar_energies, not frictional or mesh contact");
  if (s->has_friction) return pd_set_error(PD_ERR_STATE, "the solver already has a frictional boundary");
  double params[4] = {parameters[0], parameters[1], parameters[2], parameters[3]};
  std::vector<int32_t> faces;
  if (kind == PD_BOUNDARY_MESH) {
    if (!std::isfinite(params[0]) || params[0] < 0.0)
      return pd_set_error(PD_ERR_INVALID, "contact_radius must be finite and nonnegative");
    if (n_left < 0 || n_right < 0 || (n_left > 0 && faces_left == nullptr) || (n_right > 0 && faces_right == nullptr))
      return pd_set_error(PD_ERR_INVALID, "mesh boundary faces are (F, 3) particle indices");
    faces.assign(faces_left, faces_left + 3 * static_cast<size_t>(n_left));
    faces.insert(faces.end(), faces_right, faces_right + 3 * static_cast<size_t>(n_right));
    for (int32_t node : faces) {
      if (node < 0 || node >= s->n)
        return pd_set_error(PD_ERR_INVALID, "mesh boundary faces must reference existing particles");
    }
    params[1] = params[2] = params[3] = 0.0;
  }
  for (double value : params) {
    if (!std::isfinite(value)) return pd_set_error(PD_ERR_INVALID, "frictional boundary parameters must be four finite values");
  }
  if (kind == PD_BOUNDARY_PLANAR &&
      std::sqrt(params[0] * params[0] + params[1] * params[1] + params[2] * params[2]) <= DBL_EPSILON)
    return pd_set_error(PD_ERR_INVALID, "planar boundary needs a nonzero normal");
  if (count < 0 || (count > 0 && nodes == nullptr))
    return pd_set_error(PD_ERR_INVALID, "frictional vertices must be unique particle indices");
  std::vector<int32_t> registered(nodes, nodes + count);
  std::vector<char> seen(s->n, 0);
  for (int32_t node : registered) {
    if (node < 0 || node >= s->n) return pd_set_error(PD_ERR_INVALID, "frictional vertices must reference existing particles");
    if (seen[node]) return pd_set_error(PD_ERR_INVALID, "frictional vertices must be unique particle indices");
    seen[node] = 1;
  }
  if (!std::isfinite(friction) || friction < 0.0) return pd_set_error(PD_ERR_INVALID, "friction must be finite and nonnegative");
  if (!std::isfinite(restitution) || restitution < 0.0)
    return pd_set_error(PD_ERR_INVALID, "restitution must be finite and nonnegative");
  PD_CUDA(cudaSetDevice(s->device));
  const size_t k = static_cast<size_t>(std::max(count, 1));
  const size_t d = sizeof(double), i32 = sizeof(int32_t);
  std::vector<double> host_params(params, params + 4);
  PD_CUDA(s->fc_params.upload(host_params));
  PD_CUDA(s->fc_nodes.upload(registered));
  PD_CUDA(s->fc_faces.upload(faces));
  PD_CUDA(s->fc_panel.allocate(static_cast<size_t>(s->n) * k * d));
  PD_CUDA(s->fc_block.allocate(k * k * d));
  PD_CUDA(s->fc_normal.allocate(3 * k * d));
  PD_CUDA(s->fc_tangent1.allocate(3 * k * d));
  PD_CUDA(s->fc_tangent2.allocate(3 * k * d));
  PD_CUDA(s->fc_delassus.allocate(k * k * d));
  PD_CUDA(s->fc_regularization.allocate(k * d));
  std::vector<int32_t> candidate(k, 1);
  PD_CUDA(s->fc_candidate.upload(candidate));
  PD_CUDA(s->fc_multiplier.allocate(k * d));
  PD_CUDA(s->fc_lambda_t.allocate(2 * k * d));
  PD_CUDA(s->fc_omega.allocate(k * d));
  PD_CUDA(s->fc_diagonal.allocate(k * d));
  PD_CUDA(s->fc_residual.allocate(k * d));
  PD_CUDA(s->fc_rhs.allocate(k * d));
  PD_CUDA(s->fc_force.allocate(3 * k * d));
  PD_CUDA(s->fc_response.allocate(3 * k * d));
  PD_CUDA(s->fc_order.allocate(k * i32));
  PD_CUDA(s->fc_slot.allocate(k * i32));
  PD_CUDA(s->fc_active.allocate(i32));
  PD_CUDA(s->fc_matrix.allocate(k * k * d));
  PD_CUDA(s->fc_compact.allocate(k * d));
  PD_CUDA(s->fc_permutation.allocate(k * i32));
  PD_CUDA(s->fc_work.allocate(k * d));
  PD_CUDA(s->fc_surface.allocate(kind == PD_BOUNDARY_MESH ? static_cast<size_t>(3) * s->n * d : d));
  pdb200::FrictionArgs& f = s->fc;
  f = pdb200::FrictionArgs{};
  f.count = count;
  f.kind = kind;
  f.params = s->fc_params.as<double>();
  f.nodes = s->fc_nodes.as<int>();
  f.friction = friction;
  f.restitution = restitution;
  f.faces = s->fc_faces.as<int>();
  f.face_count = n_left + n_right;
  f.left_count = n_left;
  f.split = split;
  f.radius = kind == PD_BOUNDARY_MESH ? params[0] : 0.0;
  f.panel = s->fc_panel.as<double>();
  f.block = s->fc_block.as<double>();
  f.normal = s->fc_normal.as<double>();
  f.tangent1 = s->fc_tangent1.as<double>();
  f.tangent2 = s->fc_tangent2.as<double>();
  f.delassus = s->fc_delassus.as<double>();
  f.regularization = s->fc_regularization.as<double>();
  f.candidate = s->fc_candidate.as<int>();
  f.multiplier = s->fc_multiplier.as<double>();
  f.lambda_t = s->fc_lambda_t.as<double>();
  f.omega = s->fc_omega.as<double>();
  f.diagonal = s->fc_diagonal.as<double>();
  f.residual = s->fc_residual.as<double>();
  f.rhs = s->fc_rhs.as<double>();
  f.force = s->fc_force.as<double>();
  f.response = s->fc_response.as<double>();
  f.order = s->fc_order.as<int>();
  f.slot = s->fc_slot.as<int>();
  f.active = s->fc_active.as<int>();
  f.matrix = s->fc_matrix.as<double>();
  f.compact = s->fc_compact.as<double>();
  f.permutation = s->fc_permutation.as<int>();
  f.work = s->fc_work.as<double>();
  f.surface = s->fc_surface.as<double>();
  s->has_friction = true;
  if (s->built) {
    if (int status = pd_build_frictional_panel(s)) return status;
  }
  return PD_OK;
}

int pd_frictional_buffers(PdSolver* s, double** parameters, double** multipliers, int32_t* count) {
  if (s == nullptr) return pd_set_error(PD_ERR_INVALID, "null solver");
  if (!s->has_friction) return pd_set_error(PD_ERR_STATE, "the solver has no frictional boundary");
  if (parameters != nullptr) *parameters = s->fc_params.as<double>();
  if (multipliers != nullptr) *multipliers = s->fc_multiplier.as<double>();
  if (count != nullptr) *count = s->fc.count;
  return PD_OK;
}

int pd_frictional_state(PdSolver* s, double* multiplier, double* omega, double* normal, int32_t* candidate,
                        void* stream) {
  if (s == nullptr) return pd_set_error(PD_ERR_INVALID, "null solver");
  if (!s->has_friction) return pd_set_error(PD_ERR_STATE, "the solver has no frictional boundary");
  PD_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t k = static_cast<size_t>(s->fc.count);
  if (k == 0) return PD_OK;
  if (multiplier != nullptr) PD_CUDA(cudaMemcpyAsync(multiplier, s->fc_multiplier.ptr, k * sizeof(double), cudaMemcpyDefault, st));
  if (omega != nullptr) PD_CUDA(cudaMemcpyAsync(omega, s->fc_omega.ptr, k * sizeof(double), cudaMemcpyDefault, st));
  if (normal != nullptr) PD_CUDA(cudaMemcpyAsync(normal, s->fc_normal.ptr, 3 * k * sizeof(double), cudaMemcpyDefault, st));
  if (candidate != nullptr)
    PD_CUDA(cudaMemcpyAsync(candidate, s->fc_candidate.ptr, k * sizeof(int32_t), cudaMemcpyDefault, st));
  return PD_OK;
}

int pd_set_woodbury_lanes(PdSolver* s, int32_t enabled) {
  if (s == nullptr) return pd_set_error(PD_ERR_INVALID, "null solver");
  s->woodbury_lanes = enabled != 0;
  return PD_OK;
}

int pd_set_woodbury_team(PdSolver* s, int32_t blocks) {
  if (s == nullptr) return pd_set_error(PD_ERR_INVALID, "null solver");
  if (blocks < 0 || blocks > 64 || (blocks & (blocks - 1)) != 0)
    return pd_set_error(PD_ERR_INVALID, "the Woodbury team must be 0 (automatic) or a power of two up to 64");
  s->woodbury_team = blocks;
  return PD_OK;
}

}  // extern "C"
