// Internal state of a solver instance, shared by the translation units of
// the library (the single-instance path and the batched path).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pd_b200.h"
#include "factor.h"
#include "pd_device.cuh"

using pdb200::InverseFactor;

// Records the message returned by pd_last_error() and returns code.
int pd_set_error(int code, const std::string& message);

struct PdSolver;
namespace pdb200 {
struct StepArgs;
struct AdjointArgs;
}  // namespace pdb200

extern "C" {
// Launch plan of a built solver for a team of `blocks` blocks with `budget`
// bytes of dynamic shared memory (pd_solver.cu).
int pd_plan_launch(PdSolver* s, int blocks, int budget);
// The single-instance plan of the last build, planned again if a batch took it.
int pd_ensure_plan(PdSolver* s);
// The fields of the step / adjoint arguments that do not change between
// calls (pd_solver.cu); the adjoint buffers must exist (pd_ensure_adjoint_buffers).
void fill_step_args(const PdSolver* s, pdb200::StepArgs* a);
void fill_adjoint_args(const PdSolver* s, pdb200::AdjointArgs* b);
int pd_ensure_adjoint_buffers(PdSolver* s);
// The mesh contact force of the state (q, v) into s->mc_force (pd_contact.cu).
int pd_evaluate_mesh_contact(PdSolver* s, const void* q, const void* v, int f64, cudaStream_t stream);
// Panel A^{-1}[:, nodes] and block of the frictional boundary from the built
// factor; zeroes the multipliers (pd_friction.cu).
int pd_build_frictional_panel(PdSolver* s);
}
// After the full adjoint pass `full` (run without parameter gradients): the
// Woodbury columns of the recorded contact state and the parameter gradients
// of z (pd_woodbury.cu).
int pd_woodbury_gradients(PdSolver* s, const pdb200::AdjointArgs& full, const double* multiplier, const double* omega,
                          const double* normal, cudaStream_t st);
extern "C" {
}

#define PD_CUDA(call)                                                                                 \
  do {                                                                                                \
    cudaError_t pd_status_ = (call);                                                                  \
    if (pd_status_ != cudaSuccess) {                                                                  \
      return pd_set_error(PD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(pd_status_));   \
    }                                                                                                 \
  } while (0)

// Owned device allocation.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { release(); }
  void release() {
    if (ptr != nullptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  cudaError_t allocate(size_t size) {
    release();
    if (size == 0) size = 16;
    bytes = size;
    cudaError_t status = cudaMalloc(&ptr, size);
    if (status != cudaSuccess) {
      ptr = nullptr;
      bytes = 0;
      return status;
    }
    return cudaMemset(ptr, 0, size);
  }
  template <typename T>
  cudaError_t upload(const std::vector<T>& host) {
    cudaError_t status = allocate(host.size() * sizeof(T));
    if (status != cudaSuccess || host.empty()) return status;
    return cudaMemcpy(ptr, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice);
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
  // Exchanges the allocations of two buffers (ownership moves, pointers stay valid).
  void swap(DeviceBuffer& other) {
    std::swap(ptr, other.ptr);
    std::swap(bytes, other.bytes);
  }
};

struct PdSolver {
  int device = 0;
  int n = 0, ne = 0, corners = 0, hex = 0;
  double mean_volume = 0.0;
  PdOptions options{};
  std::vector<int32_t> indices;
  std::vector<double> gradients;
  std::vector<int32_t> free_;
  bool has_dirichlet = false;
  // Materials and energies (host copies).
  std::vector<double> mu, lame;
  bool materials_set = false;
  std::vector<double> muscle_dir, muscle_stiffness;
  bool has_muscles = false;
  std::vector<double> muscle_targets;
  const float* activations = nullptr;
  std::vector<int32_t> plane_vertices;
  std::vector<double> plane_stiffness;
  double plane[4] = {0, 0, 0, 0};
  // Build state.
  bool built = false;
  bool stale = true;
  double built_dt = 0.0;
  double inertia = 0.0, mass = 0.0;
  double nh_mu = 0.0, nh_lame = 0.0, nh_penalty = 0.0;
  int blocks = 0;
  int max_blocks = 0;
  // The single-instance launch plan of the last build; a batch that plans the
  // solver for a team takes that plan's buffers and leaves plan_valid false,
  // so the next single-instance call plans again.
  int default_blocks = 0, default_budget = 0;
  bool plan_valid = false;
  // Bumped whenever a build or a window change reallocates buffers that a
  // batch's argument blocks point to; a batch refuses to run after a change.
  uint64_t generation = 0;
  // Launch plan of the sparse products.
  pdb200::SpmvPlan plan_s{}, plan_st{};
  int resident = 0, stage_vector = 0, vector_smem_offset = 0;
  // Own-row Anderson history in dynamic shared memory (offset -1: global),
  // planned for hist_slots history slots.
  int hist_smem_offset = -1, hist_slots = 0;
  size_t smem = 0;
  DeviceBuffer d_s_rowlist, d_s_nshort, d_st_rowlist, d_st_nshort, d_svd_u, d_svd_v;
  // Subset staging of the product vectors (resident, staged plans): per block
  // the columns its slice reads, and the slice columns renumbered into them.
  DeviceBuffer d_s_stage_off, d_s_stage_cols, d_s_col_local, d_st_stage_off, d_st_stage_cols, d_st_col_local;
  unsigned long long* timers = nullptr;  // phase timers of PD_PHASE_TIMERS builds
  InverseFactor factor;
  // Device mesh data.
  DeviceBuffer d_indices, d_gradients, d_free, d_inc_offsets, d_inc_entries, d_plane_weight;
  // Mesh contact state force between two bodies (mesh_contact.py): parameters
  // (radius, kn_left, kn_right, kf, mu), surface vertices and faces of A and
  // B, per-particle slots and (face, corner) incidence, pair buffers.
  bool has_mesh_contact = false;
  double mc_params[5] = {0, 0, 0, 0, 0};
  int mc_va = 0, mc_vb = 0, mc_fa = 0, mc_fb = 0;
  DeviceBuffer mc_vertices_a, mc_vertices_b, mc_faces_a, mc_faces_b, mc_slot_a, mc_slot_b;
  DeviceBuffer mc_inc_a_off, mc_inc_a, mc_inc_b_off, mc_inc_b;
  DeviceBuffer mc_force_ab, mc_bary_ab, mc_force_ba, mc_bary_ba, mc_force, mc_pairs;
  // Frictional boundary (contact.py FrictionalContact): the device argument
  // block with pointers into the buffers below; fc.count == 0 when absent.
  bool has_friction = false;
  pdb200::FrictionArgs fc{};
  DeviceBuffer fc_params, fc_nodes, fc_faces, fc_panel, fc_block, fc_normal, fc_tangent1, fc_tangent2, fc_delassus,
      fc_regularization, fc_candidate, fc_multiplier, fc_lambda_t, fc_omega, fc_diagonal, fc_residual, fc_rhs,
      fc_force, fc_response, fc_order, fc_slot, fc_active, fc_matrix, fc_compact, fc_permutation, fc_work,
      fc_surface;
  // Contact projection of the parameter gradients (pd_woodbury.cu), sized for w_rows rows.
  int w_rows = 0;
  bool woodbury_lanes = true;  // columns side by side on lanes (false: one launch per column)
  unsigned spin_limit = 0;     // poll budget of the step and backward barriers (0: the built-in budget)
  int factor_device = 0;       // 1: the inverse rows of the factor build run on the device
  // DiffPD forward (pd_diffpd.cu): vectors, L-BFGS history for dp_history
  // pairs, element energies, packed state forces and counters.
  DeviceBuffer dp_vectors, dp_hist, dp_energy, dp_kinds, dp_params, dp_counters;
  int dp_history = 0;
  int dp_force_count = 0;
  int woodbury_team = 0;       // blocks per lane (0: from nnz(S) and the element samples)
  DeviceBuffer w_row_node, w_row_vector, w_value, w_selected, w_order, w_control, w_columns, w_gram, w_coefficients,
      w_permutation, w_work, w_seed, w_mu;
  // Columns solved side by side on lanes of one launch: argument blocks,
  // lanes and each column's own vectors.
  DeviceBuffer w_team_args, w_team_lane_start, w_team_lane_class, w_team_class_begin, w_team_class_order,
      w_team_class_head, w_team_lane_slot, w_team_barriers, w_team_vectors, w_team_hist, w_team_contrib,
      w_team_ints, w_team_doubles, w_team_partials, w_team_seeds;
  DeviceBuffer d_wc, d_wv, d_wn, d_wm, d_mdir, d_mtarget;
  DeviceBuffer d_s_off, d_s_col, d_s_val, d_s_val32, d_st_off, d_st_col, d_st_val, d_st_val32, d_s_part, d_st_part;
  DeviceBuffer d_a_off, d_a_col, d_a_val;
  // Padded streaming layouts of S and S^T (plans that are not resident).
  DeviceBuffer d_s_off4, d_s_col4, d_s_val4, d_st_off4, d_st_col4, d_st_val4;
  // Step vectors.
  DeviceBuffer d_position, d_velocity, d_target, d_boundary, d_x, d_prev, d_proj, d_prev_proj, d_rhs, d_y, d_contrib;
  DeviceBuffer d_hist_x, d_hist_g, d_aa_state, d_aa_gamma, d_aa_accept, d_partials;
  DeviceBuffer d_iteration, d_active, d_status, d_barrier;
  // Adjoint vectors.
  DeviceBuffer b_rhs, b_base, b_solution, b_prev, b_work, b_y, b_raw, b_contrib, b_jac, b_hist_x, b_hist_g, b_aa_state,
      b_aa_gamma, b_aa_accept, b_partials, b_iteration, b_active, b_control_d, b_control_i, b_material_scratch,
      b_activation_scratch, b_zero_gq, b_zero_gqd, b_scratch_gq, b_scratch_gqd, b_scratch_gf;
};

// Buffers of a launch plan planned for a team size (row partitions, row
// lists, streaming layouts, partial sums), taken out of the solver: the
// argument blocks filled from that plan stay valid while this object lives,
// whatever the solver plans next.
struct TeamPlanBuffers {
  DeviceBuffer s_part, st_part, s_rowlist, s_nshort, st_rowlist, st_nshort, s_off4, s_col4, s_val4, st_off4, st_col4,
      st_val4, partials, b_partials, s_stage_off, s_stage_cols, s_col_local, st_stage_off, st_stage_cols, st_col_local;
  void take(PdSolver* s) {
    s_part.swap(s->d_s_part);
    st_part.swap(s->d_st_part);
    s_rowlist.swap(s->d_s_rowlist);
    s_nshort.swap(s->d_s_nshort);
    st_rowlist.swap(s->d_st_rowlist);
    st_nshort.swap(s->d_st_nshort);
    s_off4.swap(s->d_s_off4);
    s_col4.swap(s->d_s_col4);
    s_val4.swap(s->d_s_val4);
    st_off4.swap(s->d_st_off4);
    st_col4.swap(s->d_st_col4);
    st_val4.swap(s->d_st_val4);
    partials.swap(s->d_partials);
    b_partials.swap(s->b_partials);
    s_stage_off.swap(s->d_s_stage_off);
    s_stage_cols.swap(s->d_s_stage_cols);
    s_col_local.swap(s->d_s_col_local);
    st_stage_off.swap(s->d_st_stage_off);
    st_stage_cols.swap(s->d_st_stage_cols);
    st_col_local.swap(s->d_st_col_local);
    s->plan_valid = false;
  }
};

// The whole single-instance launch plan of a solver, set aside while the
// solver is planned for another team size and put back afterwards (pointers
// taken from the saved plan stay valid throughout).
struct SavedPlan {
  TeamPlanBuffers buffers;
  int blocks = 0, resident = 0, stage_vector = 0, vector_smem_offset = 0, hist_smem_offset = -1, hist_slots = 0;
  size_t smem = 0;
  pdb200::SpmvPlan plan_s{}, plan_st{};
  bool valid = false;
  void save(PdSolver* s) {
    blocks = s->blocks;
    resident = s->resident;
    stage_vector = s->stage_vector;
    vector_smem_offset = s->vector_smem_offset;
    hist_smem_offset = s->hist_smem_offset;
    hist_slots = s->hist_slots;
    smem = s->smem;
    plan_s = s->plan_s;
    plan_st = s->plan_st;
    valid = s->plan_valid;
    buffers.take(s);
  }
  void restore(PdSolver* s) {
    TeamPlanBuffers other;
    other.take(s);    // releases whatever plan the solver holds now when `other` goes out of scope
    buffers.take(s);  // swaps the saved buffers back in
    s->blocks = blocks;
    s->resident = resident;
    s->stage_vector = stage_vector;
    s->vector_smem_offset = vector_smem_offset;
    s->hist_smem_offset = hist_smem_offset;
    s->hist_slots = hist_slots;
    s->smem = smem;
    s->plan_s = plan_s;
    s->plan_st = plan_st;
    s->plan_valid = valid;
  }
};
