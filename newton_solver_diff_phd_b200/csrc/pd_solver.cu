// Host side of the B200 DiffPhD solver: the C ABI declared in include/pd_b200.h.
//
// The solver object owns every device buffer of one instance. pd_build mirrors
// SolverDiffPhD._build (src/newton_solver_diff_phd/_src/solvers/diff_phd/solver.py:491-552):
// element weights, assembly of the constant matrix in the reference's
// accumulation order, the host inverse factor, then the upload. pd_step and
// pd_backward fill the argument blocks and launch one cooperative kernel each.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/pd_b200.h"
#include "factor.h"
#include "runs.h"
#include "pd_kernels.h"
#include "solver_state.h"

using pdb200::AdjointArgs;
using pdb200::StepArgs;

// pd_noalloc.cu: resolves the device address of pd_apply_inverse_static's
// scratch array on `device` (the current device).
int pd_internal_resolve_static_scratch(int device);

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& message) { return pd_set_error(code, message); }

// Contiguous row ranges with balanced cost (nnz + per-row overhead) per block.
std::vector<int32_t> partition_rows(const std::vector<int32_t>& offsets, int blocks) {
  const int rows = static_cast<int>(offsets.size()) - 1;
  std::vector<int32_t> bounds(blocks + 1, rows);
  bounds[0] = 0;
  const double overhead = 16.0;
  const double total = static_cast<double>(offsets[rows]) + overhead * rows;
  int b = 1;
  double cumulative = 0.0;
  for (int r = 0; r < rows && b < blocks; ++r) {
    cumulative += static_cast<double>(offsets[r + 1] - offsets[r]) + overhead;
    while (b < blocks && cumulative >= total * b / blocks) {
      bounds[b] = r + 1;
      ++b;
    }
  }
  for (; b < blocks; ++b) bounds[b] = rows;
  return bounds;
}

// Per-block row order for the SpMV: rows with at most kShortRow entries first
// (one thread each), then the longer rows by decreasing length (one warp each).
constexpr int kShortRow = 32;

void plan_rows(const std::vector<int32_t>& offsets, const std::vector<int32_t>& part, std::vector<int32_t>& rowlist,
               std::vector<int32_t>& nshort, int& max_nnz, int& max_rows) {
  const int blocks = static_cast<int>(part.size()) - 1;
  rowlist.assign(offsets.size() - 1, 0);
  nshort.assign(blocks, 0);
  max_nnz = 0;
  max_rows = 0;
  std::vector<int32_t> longs;
  for (int b = 0; b < blocks; ++b) {
    const int r0 = part[b], r1 = part[b + 1];
    int cursor = r0;
    longs.clear();
    for (int r = r0; r < r1; ++r) {
      if (offsets[r + 1] - offsets[r] <= kShortRow) {
        rowlist[cursor++] = r;
      } else {
        longs.push_back(r);
      }
    }
    nshort[b] = cursor - r0;
    std::stable_sort(longs.begin(), longs.end(), [&](int x, int y) {
      return offsets[x + 1] - offsets[x] > offsets[y + 1] - offsets[y];
    });
    for (int r : longs) rowlist[cursor++] = r;
    max_nnz = std::max(max_nnz, offsets[r1] - offsets[r0]);
    max_rows = std::max(max_rows, r1 - r0);
  }
}

}  // namespace

int pd_set_error(int code, const std::string& message) {
  g_last_error = message;
  return code;
}



namespace {

int validate_options(const PdOptions& o) {
  if (o.material != PD_MATERIAL_PD && o.material != PD_MATERIAL_NEO_HOOKEAN)
    return fail(PD_ERR_INVALID, "material must be 'pd' or 'neo_hookean'");
  if (!(o.density > 0.0) || !std::isfinite(o.density)) return fail(PD_ERR_INVALID, "density must be finite and positive");
  if (!(o.abs_tol >= 0.0) || !std::isfinite(o.abs_tol)) return fail(PD_ERR_INVALID, "abs_tol must be finite and nonnegative");
  if (!(o.rel_tol >= 0.0) || !std::isfinite(o.rel_tol)) return fail(PD_ERR_INVALID, "rel_tol must be finite and nonnegative");
  if (o.max_iterations < 1) return fail(PD_ERR_INVALID, "max_iterations must be a positive integer");
  if (o.anderson_window < 0 || o.anderson_window > pdb200::kMaxWindow)
    return fail(PD_ERR_INVALID, "anderson_window must be an integer in [0, 8]");
  if (o.precision != PD_PRECISION_FP64 && o.precision != PD_PRECISION_FP32_REFINE && o.precision != PD_PRECISION_FP32)
    return fail(PD_ERR_INVALID, "precision must be fp64, fp32+refine or fp32");
  if (o.adjoint_mode != PD_ADJOINT_REFERENCE && o.adjoint_mode != PD_ADJOINT_EXACT)
    return fail(PD_ERR_INVALID, "adjoint mode must be reference or exact");
  if (o.blocks < 0) return fail(PD_ERR_INVALID, "blocks must be nonnegative");
  if (o.state_precision != 0 && o.state_precision != 1) return fail(PD_ERR_INVALID, "state precision must be 0 or 1");
  if (o.adjoint_solver < PD_ADJOINT_SOLVER_AUTO || o.adjoint_solver > PD_ADJOINT_SOLVER_CG)
    return fail(PD_ERR_INVALID, "adjoint solver must be auto, fixed point or CG");
  return PD_OK;
}

int samples_of(const PdSolver* s) { return s->hex ? 8 : 1; }
double sample_volume_of(const PdSolver* s) { return s->mean_volume / static_cast<double>(samples_of(s)); }

// Per-sample gradient rows of element e, sample q.
const double* sample_rows(const PdSolver* s, int e, int q) {
  return s->hex ? s->gradients.data() + 8 * 3 * q : s->gradients.data() + 12 * e;
}

int ensure_adjoint_buffers(PdSolver* s) {
  const size_t vec = static_cast<size_t>(3) * s->n * sizeof(double);
  if (s->b_rhs.ptr != nullptr) return PD_OK;
  for (DeviceBuffer* buffer : {&s->b_rhs, &s->b_base, &s->b_solution, &s->b_prev, &s->b_work, &s->b_y, &s->b_raw})
    PD_CUDA(buffer->allocate(vec));
  PD_CUDA(s->b_contrib.allocate(static_cast<size_t>(s->ne) * s->corners * 3 * sizeof(double)));
  const size_t jac_entries = static_cast<size_t>(s->ne) * samples_of(s) * 81;
  PD_CUDA(s->b_jac.allocate(jac_entries * (s->options.precision == PD_PRECISION_FP32 ? sizeof(float) : sizeof(double))));
  const size_t window = static_cast<size_t>(s->options.anderson_window);
  PD_CUDA(s->b_hist_x.allocate((window + 1) * vec));
  PD_CUDA(s->b_hist_g.allocate((window + 1) * vec));
  PD_CUDA(s->b_aa_state.allocate(8 * sizeof(int)));
  PD_CUDA(s->b_aa_gamma.allocate(pdb200::kMaxWindow * sizeof(double)));
  PD_CUDA(s->b_aa_accept.allocate(sizeof(int)));
  PD_CUDA(s->b_iteration.allocate(sizeof(int)));
  PD_CUDA(s->b_active.allocate(sizeof(int)));
  PD_CUDA(s->b_control_d.allocate(8 * sizeof(double)));
  PD_CUDA(s->b_control_i.allocate(8 * sizeof(int)));
  PD_CUDA(s->b_material_scratch.allocate(static_cast<size_t>(s->ne) * 2 * sizeof(double)));
  PD_CUDA(s->b_activation_scratch.allocate(static_cast<size_t>(s->ne) * sizeof(double)));
  const size_t fvec = static_cast<size_t>(3) * s->n * sizeof(double);  // fits float32 and float64 states
  for (DeviceBuffer* buffer : {&s->b_zero_gq, &s->b_zero_gqd, &s->b_scratch_gq, &s->b_scratch_gqd, &s->b_scratch_gf})
    PD_CUDA(buffer->allocate(fvec));
  return PD_OK;
}

}  // namespace

extern "C" {

const char* pd_version(void) { return "newton-solver-diff-phd-b200 0.1 (sm_100a)"; }

const char* pd_last_error(void) { return g_last_error.c_str(); }

int pd_create(const PdMeshDesc* mesh, const PdOptions* options, int device, PdSolver** out) {
  if (mesh == nullptr || options == nullptr || out == nullptr) return fail(PD_ERR_INVALID, "null argument");
  *out = nullptr;
  if (int status = validate_options(*options)) return status;
  if (mesh->corners != 4 && mesh->corners != 8) return fail(PD_ERR_INVALID, "corners must be 4 (Tet4) or 8 (Hex8)");
  if (mesh->n_vertices <= 0 || mesh->n_elements <= 0)
    return fail(PD_ERR_INVALID, "SolverDiffPhD requires tetrahedral soft bodies or an explicit hex_mesh");
  if (mesh->indices == nullptr || mesh->gradients == nullptr || mesh->free == nullptr)
    return fail(PD_ERR_INVALID, "mesh arrays must not be null");
  if (!(mesh->mean_volume > 0.0) || !std::isfinite(mesh->mean_volume))
    return fail(PD_ERR_INVALID, "mean element volume must be finite and positive");
  auto solver = new PdSolver();
  solver->device = device;
  solver->n = mesh->n_vertices;
  solver->ne = mesh->n_elements;
  solver->corners = mesh->corners;
  solver->hex = mesh->corners == 8 ? 1 : 0;
  solver->mean_volume = mesh->mean_volume;
  solver->options = *options;
  const size_t index_count = static_cast<size_t>(solver->ne) * solver->corners;
  solver->indices.assign(mesh->indices, mesh->indices + index_count);
  for (int32_t v : solver->indices) {
    if (v < 0 || v >= solver->n) {
      delete solver;
      return fail(PD_ERR_INVALID, "element indices must reference existing particles");
    }
  }
  const size_t gradient_count = solver->hex ? 8 * 8 * 3 : static_cast<size_t>(solver->ne) * 12;
  solver->gradients.assign(mesh->gradients, mesh->gradients + gradient_count);
  solver->free_.resize(solver->n);
  bool any_free = false;
  for (int i = 0; i < solver->n; ++i) {
    solver->free_[i] = mesh->free[i] != 0 ? 1 : 0;
    any_free = any_free || solver->free_[i];
    solver->has_dirichlet = solver->has_dirichlet || !solver->free_[i];
  }
  if (!any_free) {
    delete solver;
    return fail(PD_ERR_INVALID, "SolverDiffPhD needs at least one dynamic particle");
  }
  solver->muscle_targets.assign(solver->ne, 1.0);
  cudaError_t status = cudaSetDevice(device);
  if (status != cudaSuccess) {
    delete solver;
    return fail(PD_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(status));
  }
  // Incidence lists sorted by element (kernels.py:61-72, hex.py:83-92). Hex8
  // contributions are pre-summed over the eight samples of a cell.
  std::vector<int32_t> counts(solver->n + 1, 0);
  for (int32_t v : solver->indices) counts[v + 1] += 1;
  for (int i = 0; i < solver->n; ++i) counts[i + 1] += counts[i];
  std::vector<int32_t> entries(index_count);
  {
    std::vector<int32_t> cursor(counts.begin(), counts.end() - 1);
    for (size_t k = 0; k < index_count; ++k) entries[cursor[solver->indices[k]]++] = static_cast<int32_t>(k);
  }
  int rc = PD_OK;
  auto check = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == PD_OK) rc = fail(PD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  check(solver->d_indices.upload(solver->indices), "indices");
  check(solver->d_gradients.upload(solver->gradients), "gradients");
  check(solver->d_free.upload(solver->free_), "free");
  check(solver->d_inc_offsets.upload(counts), "incidence");
  check(solver->d_inc_entries.upload(entries), "incidence");
  const size_t vec = static_cast<size_t>(3) * solver->n * sizeof(double);
  for (DeviceBuffer* buffer : {&solver->d_position, &solver->d_velocity, &solver->d_target, &solver->d_boundary,
                               &solver->d_x, &solver->d_prev, &solver->d_proj, &solver->d_prev_proj, &solver->d_rhs,
                               &solver->d_y})
    check(buffer->allocate(vec), "vectors");
  check(solver->d_contrib.allocate(index_count * 3 * sizeof(double)), "contributions");
  const size_t window = static_cast<size_t>(options->anderson_window);
  check(solver->d_hist_x.allocate((window + 1) * vec), "history");
  check(solver->d_hist_g.allocate((window + 1) * vec), "history");
  check(solver->d_aa_state.allocate(8 * sizeof(int)), "anderson");
  check(solver->d_aa_gamma.allocate(pdb200::kMaxWindow * sizeof(double)), "anderson");
  check(solver->d_aa_accept.allocate(sizeof(int)), "anderson");
  check(solver->d_iteration.allocate(sizeof(int)), "iteration");
  check(solver->d_active.allocate(sizeof(int)), "active");
  check(solver->d_status.allocate(sizeof(int)), "status");
  check(solver->d_barrier.allocate(sizeof(pdb200::GridBarrier)), "barrier");
  check(solver->d_mtarget.upload(solver->muscle_targets), "muscle targets");
  std::vector<double> zeros(solver->ne, 0.0);
  check(solver->d_wm.upload(zeros), "muscles");
  std::vector<double> zeros3(static_cast<size_t>(solver->ne) * 3, 0.0);
  check(solver->d_mdir.upload(zeros3), "muscles");
  if (rc != PD_OK) {
    delete solver;
    return rc;
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  check(solver->d_svd_u.allocate(index_count / solver->corners * (solver->hex ? 8 : 1) * 9 * sizeof(double)), "svd");
  check(solver->d_svd_v.allocate(index_count / solver->corners * (solver->hex ? 8 : 1) * 9 * sizeof(double)), "svd");
  if (rc != PD_OK) {
    delete solver;
    return rc;
  }
  int per_sm_forward = 0, per_sm_adjoint = 0;
  pdb200::forward_step_max_blocks(options->precision, 0, &per_sm_forward);
  pdb200::adjoint_step_max_blocks(options->precision, 0, &per_sm_adjoint);
  solver->max_blocks = sms * std::max(1, std::min(per_sm_forward, per_sm_adjoint));
  *out = solver;
  return PD_OK;
}

int pd_destroy(PdSolver* solver) {
  if (solver == nullptr) return PD_OK;
  cudaSetDevice(solver->device);
  delete solver;
  return PD_OK;
}

int pd_set_tolerances(PdSolver* solver, int32_t max_iterations, double abs_tol, double rel_tol) {
  if (solver == nullptr) return fail(PD_ERR_INVALID, "null solver");
  PdOptions o = solver->options;
  o.max_iterations = max_iterations;
  o.abs_tol = abs_tol;
  o.rel_tol = rel_tol;
  if (int status = validate_options(o)) return status;
  solver->options = o;
  return PD_OK;
}

int pd_set_anderson_window(PdSolver* solver, int32_t window) {
  if (solver == nullptr) return fail(PD_ERR_INVALID, "null solver");
  PdOptions o = solver->options;
  o.anderson_window = window;
  if (int status = validate_options(o)) return status;
  PD_CUDA(cudaSetDevice(solver->device));
  const size_t vec = static_cast<size_t>(3) * solver->n * sizeof(double);
  const size_t need = (static_cast<size_t>(window) + 1) * vec;
  if (solver->d_hist_x.bytes < need) {
    PD_CUDA(solver->d_hist_x.allocate(need));
    PD_CUDA(solver->d_hist_g.allocate(need));
    solver->generation += 1;
  }
  if (solver->b_hist_x.ptr != nullptr && solver->b_hist_x.bytes < need) {
    PD_CUDA(solver->b_hist_x.allocate(need));
    PD_CUDA(solver->b_hist_g.allocate(need));
    solver->generation += 1;
  }
  solver->options = o;
  return PD_OK;
}

int pd_set_materials(PdSolver* solver, const double* mu_lambda) {
  if (solver == nullptr || mu_lambda == nullptr) return fail(PD_ERR_INVALID, "null argument");
  solver->mu.resize(solver->ne);
  solver->lame.resize(solver->ne);
  for (int e = 0; e < solver->ne; ++e) {
    solver->mu[e] = mu_lambda[2 * e];
    solver->lame[e] = mu_lambda[2 * e + 1];
  }
  solver->materials_set = true;
  solver->stale = true;
  return PD_OK;
}

int pd_set_muscles(PdSolver* solver, const double* directions, const double* stiffness) {
  if (solver == nullptr) return fail(PD_ERR_INVALID, "null solver");
  if ((directions == nullptr) != (stiffness == nullptr))
    return fail(PD_ERR_INVALID, "muscle_directions and muscle_stiffness must be supplied together");
  solver->has_muscles = false;
  solver->muscle_dir.assign(static_cast<size_t>(solver->ne) * 3, 0.0);
  solver->muscle_stiffness.assign(solver->ne, 0.0);
  if (directions != nullptr) {
    for (int e = 0; e < solver->ne; ++e) {
      const double s = stiffness[e];
      if (!std::isfinite(s) || s < 0.0) return fail(PD_ERR_INVALID, "Muscle directions and stiffness must be finite, with nonnegative stiffness");
      solver->muscle_stiffness[e] = s;
      for (int c = 0; c < 3; ++c) solver->muscle_dir[3 * e + c] = s > 0.0 ? directions[3 * e + c] : 0.0;
      solver->has_muscles = solver->has_muscles || s > 0.0;
    }
  }
  std::vector<double> weight(solver->ne);
  const double volume = sample_volume_of(solver);
  for (int e = 0; e < solver->ne; ++e) weight[e] = solver->muscle_stiffness[e] * volume;
  PD_CUDA(solver->d_wm.upload(weight));
  PD_CUDA(solver->d_mdir.upload(solver->muscle_dir));
  solver->stale = true;
  return PD_OK;
}

int pd_set_muscle_targets(PdSolver* solver, const double* targets) {
  if (solver == nullptr || targets == nullptr) return fail(PD_ERR_INVALID, "null argument");
  for (int e = 0; e < solver->ne; ++e) {
    if (!std::isfinite(targets[e]) || targets[e] < 0.0)
      return fail(PD_ERR_INVALID, "muscle_targets must be finite nonnegative native target lengths");
  }
  solver->muscle_targets.assign(targets, targets + solver->ne);
  PD_CUDA(solver->d_mtarget.upload(solver->muscle_targets));
  return PD_OK;
}

int pd_set_activations(PdSolver* solver, const float* device_contractions) {
  if (solver == nullptr) return fail(PD_ERR_INVALID, "null solver");
  if (solver->hex && device_contractions != nullptr)
    return fail(PD_ERR_INVALID, "Hex8 uses solver.muscle_targets; tet_activations cannot control Hex8 fibres");
  solver->activations = device_contractions;
  return PD_OK;
}

int pd_set_planar_energies(PdSolver* solver, int32_t count, const int32_t* vertices, const double* stiffness,
                           const double plane[4]) {
  if (solver == nullptr) return fail(PD_ERR_INVALID, "null solver");
  solver->plane_vertices.clear();
  solver->plane_stiffness.clear();
  if (count > 0) {
    if (vertices == nullptr || stiffness == nullptr || plane == nullptr) return fail(PD_ERR_INVALID, "null argument");
    for (int k = 0; k < count; ++k) {
      if (vertices[k] < 0 || vertices[k] >= solver->n) return fail(PD_ERR_INVALID, "planar_energies needs distinct valid particle indices");
      if (!std::isfinite(stiffness[k]) || stiffness[k] < 0.0)
        return fail(PD_ERR_INVALID, "planar_energies stiffness must be finite and nonnegative");
    }
    solver->plane_vertices.assign(vertices, vertices + count);
    solver->plane_stiffness.assign(stiffness, stiffness + count);
    for (int c = 0; c < 4; ++c) solver->plane[c] = plane[c];
  }
  std::vector<double> weight(solver->n, 0.0);
  for (size_t k = 0; k < solver->plane_vertices.size(); ++k) weight[solver->plane_vertices[k]] = solver->plane_stiffness[k];
  PD_CUDA(solver->d_plane_weight.upload(weight));
  solver->stale = true;
  return PD_OK;
}

// Splits both factor products into `blocks` nnz-balanced row ranges (the
// blocks of one cooperative team), orders each range's rows for the SpMV, and
// decides what stays in `budget` bytes of dynamic shared memory: the factor
// slices for the whole launch when they fit, the SpMV input vector when it
// fits as well. The factor arrays must be uploaded.
int pd_plan_launch(PdSolver* s, int blocks, int budget) {
  s->blocks = blocks;
  const std::vector<int32_t> s_part = partition_rows(s->factor.s.offsets, blocks);
  const std::vector<int32_t> st_part = partition_rows(s->factor.st.offsets, blocks);
  PD_CUDA(s->d_s_part.upload(s_part));
  PD_CUDA(s->d_st_part.upload(st_part));
  {
    std::vector<int32_t> rowlist, nshort;
    int max_nnz = 0, max_rows = 0;
    plan_rows(s->factor.s.offsets, s_part, rowlist, nshort, max_nnz, max_rows);
    PD_CUDA(s->d_s_rowlist.upload(rowlist));
    PD_CUDA(s->d_s_nshort.upload(nshort));
    s->plan_s.max_nnz = max_nnz;
    s->plan_s.max_rows = max_rows;
    plan_rows(s->factor.st.offsets, st_part, rowlist, nshort, max_nnz, max_rows);
    PD_CUDA(s->d_st_rowlist.upload(rowlist));
    PD_CUDA(s->d_st_nshort.upload(nshort));
    s->plan_st.max_nnz = max_nnz;
    s->plan_st.max_rows = max_rows;
  }
  const int value_bytes = s->options.precision == PD_PRECISION_FP64 ? 8 : 4;
  const int slice_s = pdb200::slice_bytes(s->plan_s.max_nnz, s->plan_s.max_rows, value_bytes);
  const int slice_st = pdb200::slice_bytes(s->plan_st.max_nnz, s->plan_st.max_rows, value_bytes);
  const int vector_bytes = pdb200::align16(3 * s->n * 8);
  s->resident = s->options.resident != 0 && slice_s + slice_st <= budget ? 1 : 0;
  const int slices = s->resident ? slice_s + slice_st : 0;
  s->stage_vector = s->options.resident != 0 && slices + vector_bytes <= budget ? 1 : 0;
  s->plan_s.smem_offset = 0;
  s->plan_st.smem_offset = slice_s;
  s->vector_smem_offset = slices;
  s->smem = static_cast<size_t>(slices + (s->stage_vector ? vector_bytes : 0));
  // The Anderson history of a block's own particle rows, x and g, for the
  // current window, when it fits beside resident slices. A streamed factor
  // keeps the shared memory as L1 cache for the gathers of the product
  // vectors instead (on the 35,721-particle Hex8 beam the history in shared
  // memory made every iteration 29 % slower).
  {
    const int slots = s->options.anderson_window + 1;
    const size_t history_bytes = 2 * static_cast<size_t>(slots) * s->plan_st.max_rows * 3 * sizeof(double);
    const size_t offset = static_cast<size_t>(pdb200::align16(static_cast<int>(s->smem)));
    if (s->resident && s->options.anderson_window > 0 && offset + history_bytes <= static_cast<size_t>(budget)) {
      s->hist_smem_offset = static_cast<int>(offset);
      s->hist_slots = slots;
      s->smem = offset + history_bytes;
    } else {
      s->hist_smem_offset = -1;
      s->hist_slots = 0;
    }
  }
  auto fill_plan = [&](pdb200::SpmvPlan& plan, const DeviceBuffer& off, const DeviceBuffer& col, const DeviceBuffer& val,
                       const DeviceBuffer& val32, const DeviceBuffer& part, const DeviceBuffer& rowlist,
                       const DeviceBuffer& nshort) {
    plan.off = off.as<int>();
    plan.col = col.as<int>();
    plan.val64 = val.as<double>();
    plan.val32 = val32.as<float>();
    plan.part = part.as<int>();
    plan.rowlist = rowlist.as<int>();
    plan.nshort = nshort.as<int>();
  };
  fill_plan(s->plan_s, s->d_s_off, s->d_s_col, s->d_s_val, s->d_s_val32, s->d_s_part, s->d_s_rowlist, s->d_s_nshort);
  fill_plan(s->plan_st, s->d_st_off, s->d_st_col, s->d_st_val, s->d_st_val32, s->d_st_part, s->d_st_rowlist,
            s->d_st_nshort);
  // Subset staging: with resident slices and a staged vector, each block
  // stages only the vector entries its rows read (a block of S^T rows reads
  // the elimination rows above its particles, a fraction of the vector), and
  // its slice columns are renumbered into that list.
  auto subset = [&](const pdb200::Csr& csr, const std::vector<int32_t>& part, pdb200::SpmvPlan& plan,
                    DeviceBuffer& stage_off, DeviceBuffer& stage_cols, DeviceBuffer& col_local) -> int {
    if (!(s->resident && s->stage_vector)) {
      stage_off.release();
      stage_cols.release();
      col_local.release();
      plan.stage_off = nullptr;
      plan.stage_cols = nullptr;
      plan.col_local = nullptr;
      return PD_OK;
    }
    std::vector<int32_t> offsets(blocks + 1, 0), columns, local(csr.columns.size());
    std::vector<int32_t> position(s->n, -1);
    for (int b = 0; b < blocks; ++b) {
      const int k0 = csr.offsets[part[b]], k1 = csr.offsets[part[b + 1]];
      std::vector<int32_t> used(csr.columns.begin() + k0, csr.columns.begin() + k1);
      std::sort(used.begin(), used.end());
      used.erase(std::unique(used.begin(), used.end()), used.end());
      for (size_t j = 0; j < used.size(); ++j) position[used[j]] = static_cast<int32_t>(j);
      for (int k = k0; k < k1; ++k) local[k] = position[csr.columns[k]];
      columns.insert(columns.end(), used.begin(), used.end());
      offsets[b + 1] = static_cast<int32_t>(columns.size());
    }
    if (columns.empty()) columns.push_back(0);
    PD_CUDA(stage_off.upload(offsets));
    PD_CUDA(stage_cols.upload(columns));
    PD_CUDA(col_local.upload(local));
    plan.stage_off = stage_off.as<int>();
    plan.stage_cols = stage_cols.as<int>();
    plan.col_local = col_local.as<int>();
    return PD_OK;
  };
  if (int status = subset(s->factor.s, s_part, s->plan_s, s->d_s_stage_off, s->d_s_stage_cols, s->d_s_col_local))
    return status;
  if (int status = subset(s->factor.st, st_part, s->plan_st, s->d_st_stage_off, s->d_st_stage_cols, s->d_st_col_local))
    return status;
  // Streaming layouts for a factor that stays in global memory.
  auto pad = [&](const pdb200::Csr& csr, pdb200::SpmvPlan& plan, DeviceBuffer& off4, DeviceBuffer& col4,
                 DeviceBuffer& val4) -> int {
    if (s->resident) {
      off4.release();
      col4.release();
      val4.release();
      plan.off4 = nullptr;
      plan.col4 = nullptr;
      plan.val4 = nullptr;
      return PD_OK;
    }
    const int rows = static_cast<int>(csr.offsets.size()) - 1;
    std::vector<int32_t> offsets(rows + 1, 0);
    for (int r = 0; r < rows; ++r) offsets[r + 1] = offsets[r] + (csr.offsets[r + 1] - csr.offsets[r] + 3) / 4;
    const size_t groups = static_cast<size_t>(offsets[rows]);
    std::vector<int32_t> columns(4 * groups, 0);
    std::vector<double> values(4 * groups, 0.0);
    for (int r = 0; r < rows; ++r) {
      size_t slot = 4 * static_cast<size_t>(offsets[r]);
      for (int k = csr.offsets[r]; k < csr.offsets[r + 1]; ++k, ++slot) {
        columns[slot] = csr.columns[k];
        values[slot] = csr.values[k];
      }
      // Padding entries repeat the row's last column with a zero value.
      const int32_t last = csr.offsets[r + 1] > csr.offsets[r] ? csr.columns[csr.offsets[r + 1] - 1] : 0;
      for (; slot < 4 * static_cast<size_t>(offsets[r + 1]); ++slot) columns[slot] = last;
    }
    PD_CUDA(off4.upload(offsets));
    PD_CUDA(col4.upload(columns));
    if (s->options.precision == PD_PRECISION_FP64) {
      PD_CUDA(val4.upload(values));
    } else {
      std::vector<float> narrow(values.begin(), values.end());
      PD_CUDA(val4.upload(narrow));
    }
    plan.off4 = off4.as<int>();
    plan.col4 = col4.as<int4>();
    plan.val4 = val4.ptr;
    return PD_OK;
  };
  if (int status = pad(s->factor.s, s->plan_s, s->d_s_off4, s->d_s_col4, s->d_s_val4)) return status;
  if (int status = pad(s->factor.st, s->plan_st, s->d_st_off4, s->d_st_col4, s->d_st_val4)) return status;
  PD_CUDA(s->d_partials.allocate(static_cast<size_t>(blocks) * pdb200::kPartialStride * sizeof(double)));
  PD_CUDA(s->b_partials.allocate(static_cast<size_t>(blocks) * pdb200::kPartialStride * sizeof(double)));
  return PD_OK;
}

int pd_ensure_plan(PdSolver* s) {
  if (s->plan_valid) return PD_OK;
  if (int status = pd_plan_launch(s, s->default_blocks, s->default_budget)) return status;
  s->plan_valid = true;
  return PD_OK;
}

int pd_build(PdSolver* s, double dt) {
  if (s == nullptr) return fail(PD_ERR_INVALID, "null solver");
  if (!std::isfinite(dt) || dt <= 0.0) return fail(PD_ERR_INVALID, "dt must be finite and positive");
  if (!s->materials_set) return fail(PD_ERR_STATE, "materials must be set before the build");
  PD_CUDA(cudaSetDevice(s->device));
  for (int e = 0; e < s->ne; ++e) {
    if (!std::isfinite(s->mu[e]) || !std::isfinite(s->lame[e]) || s->mu[e] <= 0.0 || s->lame[e] < 0.0)
      return fail(PD_ERR_INVALID, "DiffPhD requires positive shear modulus and nonnegative Lame lambda");
  }
  const int samples = samples_of(s);
  const double volume = sample_volume_of(s);
  // Element weights (kernels.py:112-133, hex.py:95-112).
  std::vector<double> wc(s->ne, 0.0), wv(s->ne, 0.0), wn(s->ne, 0.0);
  for (int e = 0; e < s->ne; ++e) {
    if (s->options.material == PD_MATERIAL_PD) {
      wc[e] = 2.0 * s->mu[e] * volume;
      wv[e] = s->lame[e] * volume;
    } else {
      wn[e] = 2.0 * s->mu[e] * volume;
    }
  }
  // Mean Lame parameters of the Neo-Hookean projection (solver.py:514-518).
  // The reference takes NumPy means; the same pairwise summation order
  // (blocks of 8 below 128 entries, halving above) is used here.
  auto pairwise = [](const std::vector<double>& v) {
    // numpy.add.reduce pairwise summation with blocks of 8 (n < 8 sequential).
    std::function<double(const double*, size_t)> sum = [&](const double* a, size_t n) -> double {
      if (n < 8) {
        double r = 0.0;
        for (size_t i = 0; i < n; ++i) r += a[i];
        return r;
      }
      if (n <= 128) {
        double r[8];
        for (int j = 0; j < 8; ++j) r[j] = a[j];
        size_t i = 8;
        for (; i + 8 <= n; i += 8)
          for (int j = 0; j < 8; ++j) r[j] += a[i + j];
        double result = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) result += a[i];
        return result;
      }
      size_t half = n / 2;
      half -= half % 8;
      return sum(a, half) + sum(a + half, n - half);
    };
    return sum(v.data(), v.size()) / static_cast<double>(v.size());
  };
  s->nh_mu = pairwise(s->mu);
  s->nh_lame = pairwise(s->lame);
  s->nh_penalty = 2.0 * s->nh_mu;
  s->mass = s->options.density * s->mean_volume;
  s->inertia = s->mass / (dt * dt);
  // Constant matrix rows in the reference's accumulation order
  // (solver.py:521-545). A fixed sparsity pattern (particle adjacency) holds the
  // running sums; each entry receives the same additions in the same order.
  std::vector<std::vector<int32_t>> adjacency(s->n);
  for (int e = 0; e < s->ne; ++e) {
    const int32_t* nodes = s->indices.data() + s->corners * e;
    for (int a = 0; a < s->corners; ++a)
      for (int b = 0; b < s->corners; ++b)
        if (s->free_[nodes[a]] && s->free_[nodes[b]]) adjacency[nodes[a]].push_back(nodes[b]);
  }
  std::vector<int32_t> row_offsets(s->n + 1, 0);
  for (int i = 0; i < s->n; ++i) {
    adjacency[i].push_back(i);
    std::sort(adjacency[i].begin(), adjacency[i].end());
    adjacency[i].erase(std::unique(adjacency[i].begin(), adjacency[i].end()), adjacency[i].end());
    row_offsets[i + 1] = row_offsets[i] + static_cast<int32_t>(adjacency[i].size());
  }
  std::vector<int32_t> row_columns(row_offsets[s->n]);
  std::vector<double> row_values(row_offsets[s->n], 0.0);
  for (int i = 0; i < s->n; ++i) {
    std::copy(adjacency[i].begin(), adjacency[i].end(), row_columns.begin() + row_offsets[i]);
    const auto at = std::lower_bound(adjacency[i].begin(), adjacency[i].end(), i) - adjacency[i].begin();
    row_values[row_offsets[i] + at] = s->free_[i] ? s->inertia : 1.0;
  }
  auto add = [&](int i, int j, double value) {
    const int32_t* first = row_columns.data() + row_offsets[i];
    const int32_t* last = row_columns.data() + row_offsets[i + 1];
    row_values[row_offsets[i] + (std::lower_bound(first, last, j) - first)] += value;
  };
  const int k = s->corners;
  std::vector<double> block(static_cast<size_t>(k) * k);
  std::vector<double> fibre(k);
  for (int e = 0; e < s->ne; ++e) {
    const int32_t* nodes = s->indices.data() + k * e;
    const double weight = (wc[e] + wv[e]) + wn[e];
    const double muscle = s->muscle_stiffness.empty() ? 0.0 : s->muscle_stiffness[e] * volume;
    for (int q = 0; q < samples; ++q) {
      const double* g = sample_rows(s, e, q);
      for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) {
          const double dot = (g[3 * a] * g[3 * b] + g[3 * a + 1] * g[3 * b + 1]) + g[3 * a + 2] * g[3 * b + 2];
          block[a * k + b] = weight * dot;
        }
      if (s->has_muscles && muscle > 0.0) {
        const double* m = s->muscle_dir.data() + 3 * e;
        for (int a = 0; a < k; ++a) fibre[a] = (g[3 * a] * m[0] + g[3 * a + 1] * m[1]) + g[3 * a + 2] * m[2];
        for (int a = 0; a < k; ++a)
          for (int b = 0; b < k; ++b) block[a * k + b] += muscle * (fibre[a] * fibre[b]);
      }
      for (int a = 0; a < k; ++a) {
        const int i = nodes[a];
        if (!s->free_[i]) continue;
        for (int b = a; b < k; ++b) {
          const int j = nodes[b];
          if (!s->free_[j]) continue;
          const double value = block[a * k + b];
          add(i, j, value);
          if (i != j) add(j, i, value);
        }
      }
    }
  }
  for (size_t p = 0; p < s->plane_vertices.size(); ++p) {
    const int i = s->plane_vertices[p];
    if (s->free_[i]) add(i, i, s->plane_stiffness[p]);
  }
  InverseFactor factor;
  pdb200::InverseRowsProvider provider;
  pdb200::LdltProvider ldlt_provider;
  if (s->factor_device) {
    PD_CUDA(cudaSetDevice(s->device));
    provider = [](const pdb200::LowerFactorView& lower, pdb200::InverseRows* rows) {
      return pdb200::device_inverse_rows(lower, rows);
    };
    ldlt_provider = [](const pdb200::SymbolicView& symbolic, double* values, double* diagonal) {
      return pdb200::device_ldlt(symbolic, values, diagonal);
    };
  }
  const std::string error = pdb200::build_inverse_factor(s->n, row_offsets.data(), row_columns.data(),
                                                         row_values.data(), &factor, provider, ldlt_provider);
  if (!error.empty()) return fail(error.find("positive definite") != std::string::npos ? PD_ERR_NOT_SPD : PD_ERR_INVALID, error);
  s->factor = std::move(factor);
  // Grid size: all SMs for large factors, fewer blocks for small meshes.
  int blocks = s->options.blocks;
  if (blocks <= 0) {
    const int64_t work = std::max<int64_t>(static_cast<int64_t>(s->factor.s.columns.size()) / 2048,
                                           static_cast<int64_t>(s->ne) * samples / 256);
    blocks = static_cast<int>(std::max<int64_t>(8, std::min<int64_t>(work, s->max_blocks)));
  }
  // Fixed-order reductions handle up to 256 blocks (8 chunks of 32).
  blocks = std::min(std::min(blocks, s->max_blocks), 256);
  if (int status = pd_internal_resolve_static_scratch(s->device)) return status;
  PD_CUDA(s->d_s_off.upload(s->factor.s.offsets));
  PD_CUDA(s->d_s_col.upload(s->factor.s.columns));
  PD_CUDA(s->d_s_val.upload(s->factor.s.values));
  PD_CUDA(s->d_st_off.upload(s->factor.st.offsets));
  PD_CUDA(s->d_st_col.upload(s->factor.st.columns));
  PD_CUDA(s->d_st_val.upload(s->factor.st.values));
  if (s->options.precision != PD_PRECISION_FP64) {
    std::vector<float> s32(s->factor.s.values.begin(), s->factor.s.values.end());
    std::vector<float> st32(s->factor.st.values.begin(), s->factor.st.values.end());
    PD_CUDA(s->d_s_val32.upload(s32));
    PD_CUDA(s->d_st_val32.upload(st32));
  }
  {
    int optin = 0;
    PD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
    // 16 KB: static shared memory of the step kernels (the contact section's
    // 32 x 33 Cholesky tile included).
    if (int status = pd_plan_launch(s, blocks, optin - 16 * 1024)) return status;
    s->default_blocks = blocks;
    s->default_budget = optin - 16 * 1024;
    s->plan_valid = true;
    int per_sm_forward = 0, per_sm_adjoint = 0;
    PD_CUDA(pdb200::forward_step_max_blocks(s->options.precision, s->smem, &per_sm_forward));
    PD_CUDA(pdb200::adjoint_step_max_blocks(s->options.precision, s->smem, &per_sm_adjoint));
    int sms = 0;
    PD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    if (std::min(per_sm_forward, per_sm_adjoint) * sms < blocks) {
      return fail(PD_ERR_CUDA, "the persistent step kernels cannot keep the requested grid co-resident");
    }
  }
  PD_CUDA(s->d_a_off.upload(row_offsets));
  PD_CUDA(s->d_a_col.upload(row_columns));
  PD_CUDA(s->d_a_val.upload(row_values));
  PD_CUDA(s->d_wc.upload(wc));
  PD_CUDA(s->d_wv.upload(wv));
  PD_CUDA(s->d_wn.upload(wn));
  if (s->d_plane_weight.ptr == nullptr) {
    std::vector<double> none(s->n, 0.0);
    PD_CUDA(s->d_plane_weight.upload(none));
  }
  s->built = true;
  s->stale = false;
  s->built_dt = dt;
  s->generation += 1;
  if (s->has_friction) {
    if (int status = pd_build_frictional_panel(s)) return status;
  }
  return PD_OK;
}


int pd_factor_stats(const PdSolver* s, int64_t* rows, int64_t* nnz_s, int64_t* nnz_l) {
  if (s == nullptr) return fail(PD_ERR_INVALID, "null solver");
  if (!s->built) return fail(PD_ERR_STATE, "the factor has not been built");
  if (rows) *rows = s->factor.size;
  if (nnz_s) *nnz_s = static_cast<int64_t>(s->factor.s.columns.size());
  if (nnz_l) *nnz_l = s->factor.factorization_nnz;
  return PD_OK;
}

// Every field of the step arguments that does not change between steps.
void fill_step_args(const PdSolver* s, StepArgs* a) {
  a->n = s->n;
  a->ne = s->ne;
  a->corners = s->corners;
  a->hex = s->hex;
  a->indices = s->d_indices.as<int>();
  a->gradients = s->d_gradients.as<double>();
  a->free_ = s->d_free.as<int>();
  a->inc_offsets = s->d_inc_offsets.as<int>();
  a->inc_entries = s->d_inc_entries.as<int>();
  a->plane_weight = s->plane_vertices.empty() ? nullptr : s->d_plane_weight.as<double>();
  {
    const double* p = s->plane;
    for (int c = 0; c < 4; ++c) a->plane[c] = p[c];
  }
  a->wc = s->d_wc.as<double>();
  a->wv = s->d_wv.as<double>();
  a->wn = s->d_wn.as<double>();
  a->wm = s->d_wm.as<double>();
  a->mdir = s->d_mdir.as<double>();
  a->mtarget = s->d_mtarget.as<double>();
  a->activations = s->hex ? nullptr : s->activations;
  a->has_muscles = s->has_muscles ? 1 : 0;
  a->material = s->options.material;
  a->nh_mu = s->nh_mu;
  a->nh_lame = s->nh_lame;
  a->nh_penalty = s->nh_penalty;
  a->s_off = s->d_s_off.as<int>();
  a->s_col = s->d_s_col.as<int>();
  a->s_val = s->d_s_val.as<double>();
  a->s_val32 = s->d_s_val32.as<float>();
  a->st_off = s->d_st_off.as<int>();
  a->st_col = s->d_st_col.as<int>();
  a->st_val = s->d_st_val.as<double>();
  a->st_val32 = s->d_st_val32.as<float>();
  a->s_part = s->d_s_part.as<int>();
  a->st_part = s->d_st_part.as<int>();
  a->a_off = s->d_a_off.as<int>();
  a->a_col = s->d_a_col.as<int>();
  a->a_val = s->d_a_val.as<double>();
  a->refine = s->options.precision != PD_PRECISION_FP64 ? 1 : 0;
  a->position = s->d_position.as<double>();
  a->velocity = s->d_velocity.as<double>();
  a->target = s->d_target.as<double>();
  a->boundary = s->d_boundary.as<double>();
  a->x = s->d_x.as<double>();
  a->prev = s->d_prev.as<double>();
  a->proj = s->d_proj.as<double>();
  a->prev_proj = s->d_prev_proj.as<double>();
  a->rhs = s->d_rhs.as<double>();
  a->y = s->d_y.as<double>();
  a->contrib = s->d_contrib.as<double>();
  a->window = s->options.anderson_window;
  a->hist_x = s->d_hist_x.as<double>();
  a->hist_g = s->d_hist_g.as<double>();
  a->hist_smem_offset =
      (s->hist_smem_offset >= 0 && s->options.anderson_window + 1 <= s->hist_slots) ? s->hist_smem_offset : -1;
  a->hist_rows = s->plan_st.max_rows;
  a->aa_state = s->d_aa_state.as<int>();
  a->aa_gamma = s->d_aa_gamma.as<double>();
  a->aa_accept = s->d_aa_accept.as<int>();
  a->partials = s->d_partials.as<double>();
  a->iteration = s->d_iteration.as<int>();
  a->active = s->d_active.as<int>();
  a->status = s->d_status.as<int>();
  a->max_iterations = s->options.max_iterations;
  a->abs_tol = s->options.abs_tol;
  a->rel_tol = s->options.rel_tol;
  a->barrier = s->d_barrier.as<pdb200::GridBarrier>();
  a->mass = s->mass;
  a->inertia = s->inertia;
  a->integrate_pinned = s->options.integrate_pinned_velocities;
  a->state_f64 = s->options.state_precision;
  a->timers = s->timers;
  a->plan_s = s->plan_s;
  a->plan_st = s->plan_st;
  a->resident = s->resident;
  a->stage_vector = s->stage_vector;
  a->vector_smem_offset = s->vector_smem_offset;
  // Float32 residual products, except with a frictional boundary: its Newton
  // step on the multipliers combines the product with the float64 panel,
  // and the float32 sums keep the coupled iteration from its tight tolerances.
  a->f32_vectors =
      (s->options.precision != PD_PRECISION_FP64 && s->resident && s->stage_vector && !s->has_friction) ? 1 : 0;
  a->svd_u = s->options.svd_warm_start ? s->d_svd_u.as<double>() : nullptr;
  a->svd_v = s->options.svd_warm_start ? s->d_svd_v.as<double>() : nullptr;
  a->fc = s->fc;
}

int pd_step(PdSolver* s, const void* q, const void* qd, const void* f, const void* dirichlet,
            const double gravity[3], double dt, void* q_out, void* qd_out, double* x_record, void* stream) {
  if (s == nullptr || q == nullptr || qd == nullptr || f == nullptr || gravity == nullptr || q_out == nullptr ||
      qd_out == nullptr)
    return fail(PD_ERR_INVALID, "null argument");
  if (!std::isfinite(dt) || dt <= 0.0) return fail(PD_ERR_INVALID, "dt must be finite and positive");
  if (q == q_out || qd == qd_out || q == qd_out || qd == q_out)
    return fail(PD_ERR_INVALID, "DiffPhD requires distinct input and output states");
  if (dirichlet != nullptr && (dirichlet == q_out || dirichlet == qd_out))
    return fail(PD_ERR_INVALID, "dirichlet_positions must not alias an output state");
  if (!s->built || s->stale || s->built_dt != dt)
    return fail(PD_ERR_STATE, "SolverDiffPhD must rebuild its factor (pd_build) for this dt and model");
  PD_CUDA(cudaSetDevice(s->device));
  if (int status = pd_ensure_plan(s)) return status;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  StepArgs a{};
  fill_step_args(s, &a);
  a.q_in = q;
  a.qd_in = qd;
  a.f_in = f;
  a.dirichlet = dirichlet;
  a.q_out = q_out;
  a.qd_out = qd_out;
  a.x_record = x_record;
  a.dt = dt;
  for (int c = 0; c < 3; ++c) a.gravity[c] = gravity[c];
  if (s->has_mesh_contact) {
    // Evaluated once on the start-of-step state (mesh_contact.py, solver.py:762-770).
    if (int status = pd_evaluate_mesh_contact(s, q, qd, s->options.state_precision, st)) return status;
    a.extra_force = s->mc_force.as<double>();
  }
  PD_CUDA(cudaMemsetAsync(s->d_barrier.ptr, 0, sizeof(pdb200::GridBarrier), st));
  if (s->spin_limit != 0u) PD_CUDA(pdb200::launch_set_spin_limit(a.barrier, s->spin_limit, st));
  PD_CUDA(pdb200::launch_forward_step(a, s->blocks, s->options.precision, s->smem, st));
  return PD_OK;
}

// Every field of the adjoint arguments that does not change between calls.
void fill_adjoint_args(const PdSolver* s, AdjointArgs* b) {
  b->n = s->n;
  b->ne = s->ne;
  b->corners = s->corners;
  b->hex = s->hex;
  b->indices = s->d_indices.as<int>();
  b->gradients = s->d_gradients.as<double>();
  b->free_ = s->d_free.as<int>();
  b->inc_offsets = s->d_inc_offsets.as<int>();
  b->inc_entries = s->d_inc_entries.as<int>();
  b->wc = s->d_wc.as<double>();
  b->wv = s->d_wv.as<double>();
  b->wn = s->d_wn.as<double>();
  b->wm = s->d_wm.as<double>();
  b->mdir = s->d_mdir.as<double>();
  b->mtarget = s->d_mtarget.as<double>();
  b->has_muscles = s->has_muscles ? 1 : 0;
  b->material = s->options.material;
  b->exact = s->options.adjoint_mode == PD_ADJOINT_EXACT ? 1 : 0;
  b->pcg = s->options.adjoint_solver == PD_ADJOINT_SOLVER_CG ||
                  (s->options.adjoint_solver == PD_ADJOINT_SOLVER_AUTO && b->exact)
              ? 1
              : 0;
  b->nh_mu = s->nh_mu;
  b->nh_lame = s->nh_lame;
  b->nh_penalty = s->nh_penalty;
  const double volume = sample_volume_of(s);
  // StepRecord.jacobian_weights (adjoint.py:828-832): the mean weight per energy.
  b->jwc = s->options.material == PD_MATERIAL_PD ? 2.0 * s->nh_mu * volume : 0.0;
  b->jwv = s->options.material == PD_MATERIAL_PD ? s->nh_lame * volume : 0.0;
  b->jwn = s->options.material == PD_MATERIAL_NEO_HOOKEAN ? 2.0 * s->nh_mu * volume : 0.0;
  b->sample_volume = volume;
  b->s_off = s->d_s_off.as<int>();
  b->s_col = s->d_s_col.as<int>();
  b->s_val = s->d_s_val.as<double>();
  b->s_val32 = s->d_s_val32.as<float>();
  b->st_off = s->d_st_off.as<int>();
  b->st_col = s->d_st_col.as<int>();
  b->st_val = s->d_st_val.as<double>();
  b->st_val32 = s->d_st_val32.as<float>();
  b->s_part = s->d_s_part.as<int>();
  b->st_part = s->d_st_part.as<int>();
  b->a_off = s->d_a_off.as<int>();
  b->a_col = s->d_a_col.as<int>();
  b->a_val = s->d_a_val.as<double>();
  b->refine = s->options.precision != PD_PRECISION_FP64 ? 1 : 0;
  b->rhs = s->b_rhs.as<double>();
  b->base = s->b_base.as<double>();
  b->solution = s->b_solution.as<double>();
  b->prev = s->b_prev.as<double>();
  b->work = s->b_work.as<double>();
  b->y = s->b_y.as<double>();
  b->raw = s->b_raw.as<double>();
  b->contrib = s->b_contrib.as<double>();
  b->jac64 = s->b_jac.as<double>();
  b->jac32 = s->b_jac.as<float>();
  b->window = s->options.anderson_window;
  b->hist_x = s->b_hist_x.as<double>();
  b->hist_g = s->b_hist_g.as<double>();
  b->aa_state = s->b_aa_state.as<int>();
  b->aa_gamma = s->b_aa_gamma.as<double>();
  b->aa_accept = s->b_aa_accept.as<int>();
  b->partials = s->b_partials.as<double>();
  b->iteration = s->b_iteration.as<int>();
  b->active = s->b_active.as<int>();
  b->status = s->d_status.as<int>();
  b->max_iterations = s->options.max_iterations;
  b->abs_tol = s->options.abs_tol;
  b->rel_tol = s->options.rel_tol;
  b->barrier = s->d_barrier.as<pdb200::GridBarrier>();
  b->control_d = s->b_control_d.as<double>();
  b->control_i = s->b_control_i.as<int>();
  b->state_f64 = s->options.state_precision;
  b->material_scratch = s->b_material_scratch.as<double>();
  b->activation_scratch = s->b_activation_scratch.as<double>();
  b->has_dirichlet = s->has_dirichlet ? 1 : 0;
  b->integrate_pinned = s->options.integrate_pinned_velocities;
  b->inertia = s->inertia;
  b->plan_s = s->plan_s;
  b->plan_st = s->plan_st;
  b->resident = s->resident;
  b->stage_vector = s->stage_vector;
  b->vector_smem_offset = s->vector_smem_offset;
}

int pd_ensure_adjoint_buffers(PdSolver* s) { return ensure_adjoint_buffers(s); }

int pd_backward(PdSolver* s, const double* x_record, const float* activations, double dt, const void* gq_out,
                const void* gqd_out, void* gq, void* gqd, void* gf, void* gdirichlet, double* gmaterials,
                float* gactivations, void* stream) {
  return pd_backward_contact(s, x_record, activations, dt, gq_out, gqd_out, gq, gqd, gf, gdirichlet, gmaterials,
                             gactivations, nullptr, nullptr, nullptr, stream);
}

int pd_backward_contact(PdSolver* s, const double* x_record, const float* activations, double dt, const void* gq_out,
                        const void* gqd_out, void* gq, void* gqd, void* gf, void* gdirichlet, double* gmaterials,
                        float* gactivations, const double* multiplier, const double* omega, const double* normal,
                        void* stream) {
  if (s == nullptr || x_record == nullptr) return fail(PD_ERR_INVALID, "null argument");
  if ((multiplier != nullptr || omega != nullptr || normal != nullptr) &&
      (multiplier == nullptr || omega == nullptr || normal == nullptr || !s->has_friction))
    return fail(PD_ERR_INVALID, "a contact snapshot needs multipliers, omega and normals of a frictional boundary");
  if (!s->built || s->stale || s->built_dt != dt)
    return fail(PD_ERR_STATE, "the backward pass needs the factor of its recorded step (same dt and model)");
  PD_CUDA(cudaSetDevice(s->device));
  if (int status = pd_ensure_plan(s)) return status;
  if (int status = ensure_adjoint_buffers(s)) return status;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t fvec = static_cast<size_t>(3) * s->n * (s->options.state_precision ? sizeof(double) : sizeof(float));
  // Missing output gradients read as zero; missing input accumulators go to scratch.
  if (gq_out == nullptr || gqd_out == nullptr) {
    PD_CUDA(cudaMemsetAsync(s->b_zero_gq.ptr, 0, fvec, st));
    PD_CUDA(cudaMemsetAsync(s->b_zero_gqd.ptr, 0, fvec, st));
  }
  AdjointArgs b{};
  fill_adjoint_args(s, &b);
  b.x = x_record;
  b.gq_out = gq_out != nullptr ? gq_out : s->b_zero_gq.ptr;
  b.gqd_out = gqd_out != nullptr ? gqd_out : s->b_zero_gqd.ptr;
  b.gq = gq != nullptr ? gq : s->b_scratch_gq.ptr;
  b.gqd = gqd != nullptr ? gqd : s->b_scratch_gqd.ptr;
  b.gf = gf != nullptr ? gf : s->b_scratch_gf.ptr;
  b.gdirichlet = gdirichlet;
  b.gmaterials = gmaterials;
  b.gactivations = s->hex ? nullptr : gactivations;
  b.zero_energy_weight =
      (gmaterials != nullptr && s->options.material == PD_MATERIAL_PD && s->nh_lame == 0.0) ? 1 : 0;
  b.dt = dt;
  // A Tet4 step's fibre targets are 1 - u of the activations it used.
  b.activations = (!s->hex && s->has_muscles) ? activations : nullptr;
  // Parameter gradients with recorded contact rows use z = mu - W_T G^{-1} J mu
  // (adjoint.py:1141-1145): the full pass leaves them to the projection.
  const bool woodbury = multiplier != nullptr && s->fc.count > 0 && (b.gmaterials != nullptr || b.gactivations != nullptr);
  pdb200::AdjointArgs full = b;
  if (woodbury) {
    full.gmaterials = nullptr;
    full.gactivations = nullptr;
  }
  PD_CUDA(cudaMemsetAsync(s->d_barrier.ptr, 0, sizeof(pdb200::GridBarrier), st));
  if (s->spin_limit != 0u) PD_CUDA(pdb200::launch_set_spin_limit(full.barrier, s->spin_limit, st));
  PD_CUDA(pdb200::launch_adjoint_step(full, s->blocks, s->options.precision, s->smem, st));
  if (woodbury) return pd_woodbury_gradients(s, b, multiplier, omega, normal, st);
  return PD_OK;
}

int pd_set_factor_device(PdSolver* s, int32_t enabled) {
  if (s == nullptr) return fail(PD_ERR_INVALID, "null solver");
  if (enabled != 0 && enabled != 1) return fail(PD_ERR_INVALID, "enabled must be 0 or 1");
  s->factor_device = enabled;
  return PD_OK;
}

int pd_set_spin_limit(PdSolver* s, uint32_t polls) {
  if (s == nullptr) return fail(PD_ERR_INVALID, "null solver");
  s->spin_limit = polls;
  return PD_OK;
}

int pd_barrier_probe(int device, int32_t blocks, int32_t missing, int32_t mode, uint32_t polls, int32_t* status,
                     int32_t* returned) {
  if (status == nullptr || returned == nullptr) return fail(PD_ERR_INVALID, "null argument");
  if (blocks < 1 || missing < 1 || (mode != 0 && mode != 1) || polls == 0u || polls > (1u << 20) ||
      blocks + missing > static_cast<int>(pdb200::kCountMask))
    return fail(PD_ERR_INVALID, "blocks and missing must be positive, mode 0 or 1, polls in [1, 2^20]");
  int previous = 0;
  PD_CUDA(cudaGetDevice(&previous));
  PD_CUDA(cudaSetDevice(device));
  int sms = 0;
  cudaError_t error = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  void* memory = nullptr;
  if (error == cudaSuccess && blocks > sms) error = cudaErrorInvalidValue;  // one block per SM is co-resident
  if (error == cudaSuccess) error = cudaMalloc(&memory, sizeof(pdb200::GridBarrier) + 2 * sizeof(int));
  if (error == cudaSuccess) error = cudaMemset(memory, 0, sizeof(pdb200::GridBarrier) + 2 * sizeof(int));
  auto* barrier = static_cast<pdb200::GridBarrier*>(memory);
  int* words = reinterpret_cast<int*>(barrier + 1);
  if (error == cudaSuccess) error = pdb200::launch_set_spin_limit(barrier, polls, nullptr);
  if (error == cudaSuccess) error = pdb200::launch_barrier_probe(barrier, words, words + 1, blocks, missing, mode, nullptr);
  if (error == cudaSuccess) error = cudaDeviceSynchronize();
  int host[2] = {0, 0};
  if (error == cudaSuccess) error = cudaMemcpy(host, words, sizeof(host), cudaMemcpyDeviceToHost);
  if (memory != nullptr) cudaFree(memory);
  cudaSetDevice(previous);
  if (error != cudaSuccess) return fail(PD_ERR_CUDA, cudaGetErrorString(error));
  *status = host[0];
  *returned = host[1];
  return PD_OK;
}

int pd_set_phase_timers(PdSolver* s, unsigned long long* device_timers) {
  if (s == nullptr) return fail(PD_ERR_INVALID, "null solver");
  s->timers = device_timers;
  return PD_OK;
}

int pd_read_status(PdSolver* s, int32_t* bits, void* stream) {
  if (s == nullptr || bits == nullptr) return fail(PD_ERR_INVALID, "null argument");
  PD_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int value = 0;
  PD_CUDA(cudaMemcpyAsync(&value, s->d_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  PD_CUDA(cudaStreamSynchronize(st));
  PD_CUDA(cudaMemsetAsync(s->d_status.ptr, 0, sizeof(int), st));
  PD_CUDA(cudaStreamSynchronize(st));
  *bits = value;
  return PD_OK;
}

int pd_iterations(PdSolver* s, int32_t* forward, int32_t* backward, void* stream) {
  if (s == nullptr) return fail(PD_ERR_INVALID, "null solver");
  PD_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int f = 0, b = 0;
  PD_CUDA(cudaMemcpyAsync(&f, s->d_iteration.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (s->b_iteration.ptr != nullptr)
    PD_CUDA(cudaMemcpyAsync(&b, s->b_iteration.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  PD_CUDA(cudaStreamSynchronize(st));
  if (forward) *forward = f;
  if (backward) *backward = b;
  return PD_OK;
}

int pd_deformation_determinants(PdSolver* s, const float* q, double* out, void* stream) {
  if (s == nullptr || q == nullptr || out == nullptr) return fail(PD_ERR_INVALID, "null argument");
  if (!s->hex) return fail(PD_ERR_UNSUPPORTED, "deformation_determinants currently requires hex_mesh");
  PD_CUDA(cudaSetDevice(s->device));
  PD_CUDA(pdb200::launch_hex_determinants(q, s->d_indices.as<int>(), s->d_gradients.as<double>(), s->ne, out,
                                          static_cast<cudaStream_t>(stream)));
  return PD_OK;
}

int pd_apply_inverse(PdSolver* s, const double* rhs, double* out, void* stream) {
  if (s == nullptr || rhs == nullptr || out == nullptr) return fail(PD_ERR_INVALID, "null argument");
  if (!s->built) return fail(PD_ERR_STATE, "the factor has not been built");
  PD_CUDA(cudaSetDevice(s->device));
  PD_CUDA(pdb200::launch_apply_inverse(s->d_s_off.as<int>(), s->d_s_col.as<int>(), s->d_s_val.as<double>(),
                                       s->d_st_off.as<int>(), s->d_st_col.as<int>(), s->d_st_val.as<double>(), s->n,
                                       rhs, s->d_y.as<double>(), out, static_cast<cudaStream_t>(stream)));
  return PD_OK;
}

}  // extern "C"

// Internal hooks for pd_noalloc.cu (C++ linkage, not part of the ABI).
int pd_internal_fail(int code, const char* message) { return fail(code, message); }

int pd_internal_particles(const PdSolver* s) { return s->n; }

int pd_internal_factor(PdSolver* s, int* device, int* rows, const int** s_off, const int** s_col, const double** s_val,
                       const int** st_off, const int** st_col, const double** st_val) {
  if (!s->built) return fail(PD_ERR_STATE, "the factor has not been built");
  *device = s->device;
  *rows = s->n;
  *s_off = s->d_s_off.as<int>();
  *s_col = s->d_s_col.as<int>();
  *s_val = s->d_s_val.as<double>();
  *st_off = s->d_st_off.as<int>();
  *st_col = s->d_st_col.as<int>();
  *st_val = s->d_st_val.as<double>();
  return PD_OK;
}

extern "C" {

struct PdInverseFactor {
  InverseFactor factor;
};

int pd_inverse_parallel_work(int64_t work) {
  pdb200::g_parallel_row_work.store(std::max<int64_t>(work, 0));
  return PD_OK;
}

int pd_inverse_parallel_levels(int64_t entries) {
  pdb200::g_parallel_level_entries.store(std::max<int64_t>(entries, 0));
  return PD_OK;
}

int pd_factor_device_rows(int32_t mode) {
  if (mode != 0 && mode != 1) return fail(PD_ERR_INVALID, "mode must be 0 (chunked rows) or 1 (grouped dense rows)");
  pdb200::g_device_rows_grouped.store(mode);
  return PD_OK;
}

int pd_inverse_build(int32_t size, const int32_t* row_offsets, const int32_t* columns, const double* values,
                     PdInverseFactor** out) {
  return pd_inverse_build_on(-1, size, row_offsets, columns, values, out);
}

int pd_inverse_build_on(int32_t device, int32_t size, const int32_t* row_offsets, const int32_t* columns,
                        const double* values, PdInverseFactor** out) {
  if (out == nullptr || row_offsets == nullptr || (size > 0 && (columns == nullptr || values == nullptr)))
    return fail(PD_ERR_INVALID, "null argument");
  pdb200::InverseRowsProvider provider;
  pdb200::LdltProvider ldlt_provider;
  int previous = -1;
  if (device >= 0) {
    int count = 0;
    PD_CUDA(cudaGetDeviceCount(&count));
    if (device >= count) return fail(PD_ERR_INVALID, "no such CUDA device");
    PD_CUDA(cudaGetDevice(&previous));
    PD_CUDA(cudaSetDevice(device));
    provider = [](const pdb200::LowerFactorView& lower, pdb200::InverseRows* rows) {
      return pdb200::device_inverse_rows(lower, rows);
    };
    ldlt_provider = [](const pdb200::SymbolicView& symbolic, double* values, double* diagonal) {
      return pdb200::device_ldlt(symbolic, values, diagonal);
    };
  }
  auto result = new PdInverseFactor();
  const std::string error =
      pdb200::build_inverse_factor(size, row_offsets, columns, values, &result->factor, provider, ldlt_provider);
  if (previous >= 0) cudaSetDevice(previous);
  if (!error.empty()) {
    delete result;
    *out = nullptr;
    return fail(error.find("positive definite") != std::string::npos ? PD_ERR_NOT_SPD : PD_ERR_INVALID, error);
  }
  *out = result;
  return PD_OK;
}

int pd_inverse_sizes(const PdInverseFactor* f, int32_t* size, int64_t* nnz, int64_t* factorization_nnz) {
  if (f == nullptr) return fail(PD_ERR_INVALID, "null factor");
  if (size) *size = f->factor.size;
  if (nnz) *nnz = static_cast<int64_t>(f->factor.s.columns.size());
  if (factorization_nnz) *factorization_nnz = f->factor.factorization_nnz;
  return PD_OK;
}

int pd_inverse_export(const PdInverseFactor* f, int32_t* permutation, int32_t* s_offsets, int32_t* s_columns,
                      double* s_values, int32_t* st_offsets, int32_t* st_columns, double* st_values) {
  if (f == nullptr) return fail(PD_ERR_INVALID, "null factor");
  const InverseFactor& x = f->factor;
  auto copy = [](auto* dst, const auto& src) {
    if (dst != nullptr && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
  };
  copy(permutation, x.permutation);
  copy(s_offsets, x.s.offsets);
  copy(s_columns, x.s.columns);
  copy(s_values, x.s.values);
  copy(st_offsets, x.st.offsets);
  copy(st_columns, x.st.columns);
  copy(st_values, x.st.values);
  return PD_OK;
}

int pd_inverse_free(PdInverseFactor* f) {
  delete f;
  return PD_OK;
}

int pd_inverse_run_sizes(const PdInverseFactor* f, int32_t max_gap, int64_t* s_runs, int64_t* s_values,
                         int64_t* st_runs, int64_t* st_values) {
  if (f == nullptr || max_gap < 0) return fail(PD_ERR_INVALID, "null factor or negative gap");
  const pdb200::RunFactor runs = pdb200::build_run_factor(f->factor, max_gap);
  if (s_runs) *s_runs = static_cast<int64_t>(runs.s.run_col.size());
  if (s_values) *s_values = static_cast<int64_t>(runs.s.values.size());
  if (st_runs) *st_runs = static_cast<int64_t>(runs.st.run_col.size());
  if (st_values) *st_values = static_cast<int64_t>(runs.st.values.size());
  return PD_OK;
}

int pd_inverse_run_export(const PdInverseFactor* f, int32_t max_gap, int32_t* label_of, int32_t* s_row_runs,
                          int32_t* s_run_col, int32_t* s_run_off, double* s_values, int32_t* st_row_runs,
                          int32_t* st_run_col, int32_t* st_run_off, double* st_values) {
  if (f == nullptr || max_gap < 0) return fail(PD_ERR_INVALID, "null factor or negative gap");
  const pdb200::RunFactor runs = pdb200::build_run_factor(f->factor, max_gap);
  auto copy = [](auto* dst, const auto& src) {
    if (dst != nullptr && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
  };
  copy(label_of, runs.label_of);
  copy(s_row_runs, runs.s.row_runs);
  copy(s_run_col, runs.s.run_col);
  copy(s_run_off, runs.s.run_off);
  copy(s_values, runs.s.values);
  copy(st_row_runs, runs.st.row_runs);
  copy(st_run_col, runs.st.run_col);
  copy(st_run_off, runs.st.run_off);
  copy(st_values, runs.st.values);
  return PD_OK;
}

}  // extern "C"
