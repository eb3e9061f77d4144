// Launchers of the persistent step kernels and the adjoint argument block.
#pragma once

#include <cuda_runtime.h>

#include "pd_device.cuh"

namespace pdb200 {

// Everything one backward launch needs (see pd_adjoint.cu).
struct AdjointArgs {
  int n, ne, corners, hex;
  const int* indices;
  const double* gradients;
  const int* free_;
  const int* inc_offsets;
  const int* inc_entries;
  const double* wc;
  const double* wv;
  const double* wn;
  const double* wm;
  const double* mdir;
  const double* mtarget;
  const float* activations;  // Tet4 contractions of the recorded step (target 1 - u), or nullptr
  int has_muscles;
  int material;
  int exact;               // K with per-element weights instead of the mean weights
  int pcg;                 // solve (A - K) mu = g by CG preconditioned with A^{-1} instead of the fixed point
  double nh_mu, nh_lame, nh_penalty;
  double jwc, jwv, jwn;    // mean weights of K (reference mode), per sample
  double sample_volume;    // Vbar (Tet4) or Vbar/8 (Hex8)
  const int* s_off;
  const int* s_col;
  const double* s_val;
  const float* s_val32;
  const int* st_off;
  const int* st_col;
  const double* st_val;
  const float* st_val32;
  const int* s_part;
  const int* st_part;
  SpmvPlan plan_s;
  SpmvPlan plan_st;
  int resident;
  int stage_vector;
  int vector_smem_offset;
  const int* a_off;
  const int* a_col;
  const double* a_val;
  int refine;
  const double* x;         // recorded converged positions of the step
  double* rhs;
  double* base;
  double* solution;
  double* prev;
  double* work;
  double* y;
  double* raw;
  double* contrib;
  double* jac64;           // [ne*samples][81]
  float* jac32;
  int window;
  double* hist_x;
  double* hist_g;
  int* aa_state;
  double* aa_gamma;
  int* aa_accept;
  double* partials;
  int* iteration;
  int* active;
  int* status;
  int max_iterations;
  double abs_tol, rel_tol;
  GridBarrier* barrier;
  double* control_d;       // [8]
  int* control_i;          // [8]
  const void* gq_out;    // float32, or float64 when state_f64
  const void* gqd_out;
  void* gq;
  void* gqd;
  void* gf;
  void* gdirichlet;
  int state_f64;
  double* gmaterials;
  float* gactivations;
  double* material_scratch;    // [ne][2]
  double* activation_scratch;  // [ne]
  int has_dirichlet;
  int integrate_pinned;
  int zero_energy_weight;
  double dt, inertia;
};

cudaError_t launch_forward_step(const StepArgs& args, int blocks, int precision, size_t smem, cudaStream_t stream);
cudaError_t forward_step_max_blocks(int precision, size_t smem, int* blocks_per_sm);
cudaError_t launch_adjoint_step(const AdjointArgs& args, int blocks, int precision, size_t smem, cudaStream_t stream);
cudaError_t adjoint_step_max_blocks(int precision, size_t smem, int* blocks_per_sm);
cudaError_t launch_apply_inverse(const int* s_off, const int* s_col, const double* s_val, const int* st_off,
                                 const int* st_col, const double* st_val, int rows, const double* rhs, double* work,
                                 double* out, cudaStream_t stream);
cudaError_t launch_hex_determinants(const float* q, const int* indices, const double* gradients, int ne, double* out,
                                    cudaStream_t stream);

}  // namespace pdb200
