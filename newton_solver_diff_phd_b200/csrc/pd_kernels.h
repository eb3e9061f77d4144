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
  // Passes of the contact (Woodbury) projection of the parameter gradients:
  // 0 the whole step; 1 only the fixed point (A - K) w = seed from zero,
  // capped at max_iterations without a status bit (one column of
  // W_T = (A - K)^{-1} J^T); 2 only the parameter gradients of the solution
  // already in `solution` (z), with the divergence flag of the last pass 0.
  int mode;
  const double* seed;   // [n][3] right-hand side of mode 1
  int reuse_jacobian;   // the local Jacobians of x are already in jac64/jac32
};

// One persistent launch that runs whole rollouts of many instances. The grid
// is cut into lanes: fixed ranges of blocks that form one team each. Every
// lane belongs to a size class and pulls instances of its class from the
// class queue; a team runs all steps of its instance with the
// single-instance step body and its lane's barrier, then pulls again.
struct TeamLaunch {
  const StepArgs* forward;          // [count] per-instance step arguments (class plans; per-step fields unset)
  const AdjointArgs* adjoint;       // [count] per-instance adjoint arguments (per-call fields unset)
  const int* lane_start;            // [lanes + 1] first block of each lane
  const int* lane_class;            // [lanes]
  const int* class_begin;           // [classes + 1] range of each class in class_order
  const int* class_order;           // instance ids, grouped by class
  const long long* particle_offset; // [count] first particle in the concatenated arrays
  const long long* element_offset;  // [count] first element in the concatenated arrays
  int count;
  int lanes;
  int solo_class;                   // class of one-block teams (-1: none); idle lanes' blocks drain it
  int steps;
  double dt;
  double gravity[3];
  int state_f64;
  unsigned* class_head;             // [classes] next position of each class queue
  int* lane_slot;                   // [lanes] instance the lane works on (broadcast to its blocks)
  GridBarrier* lane_barrier;        // [lanes]
  int* status;                      // launch-wide status (a lane barrier that gave up)
  int* iteration_log;               // [steps][count]
  unsigned long long* timeline;     // [count][2] global-timer start and end of each instance's rollout, or nullptr
  unsigned long long* timers;       // phase timers of one instance (builds with PD_PHASE_TIMERS), or nullptr
  int timer_instance;
  // Forward rollout: concatenated [P][3] states.
  const void* q0;
  const void* qd0;
  const void* forces;               // step t at forces + t * force_stride elements
  long long force_stride;
  void* q_traj;                     // [steps][P][3]
  void* qd_traj;
  double* x_record;                 // [steps][P][3] float64 (required by the adjoint)
  // Adjoint rollout: gradients of the loss w.r.t. the final state in, w.r.t.
  // the initial state, every step's forces and the per-element Lame
  // parameters out.
  const void* grad_q_final;         // [P][3]
  const void* grad_qd_final;
  void* grad_q;                     // [2][P][3] ping-pong; the last written holds dL/dq0
  void* grad_qd;
  void* grad_forces;                // [steps][P][3], accumulated
  double* grad_materials;           // [E][2] concatenated, accumulated
  long long particles;              // P
};

cudaError_t launch_team_forward(const TeamLaunch& launch, int blocks, int precision, size_t smem, cudaStream_t stream);
cudaError_t team_forward_max_blocks(int precision, size_t smem, int* blocks_per_sm);
cudaError_t launch_team_adjoint(const TeamLaunch& launch, int blocks, int precision, size_t smem, cudaStream_t stream);
cudaError_t team_adjoint_max_blocks(int precision, size_t smem, int* blocks_per_sm);
// Woodbury columns on lanes: one mode-1 adjoint fixed point per work item.
cudaError_t launch_team_columns(const TeamLaunch& launch, int blocks, int precision, size_t smem, cudaStream_t stream);
cudaError_t team_columns_max_blocks(int precision, size_t smem, int* blocks_per_sm);

cudaError_t launch_forward_step(const StepArgs& args, int blocks, int precision, size_t smem, cudaStream_t stream);
cudaError_t forward_step_max_blocks(int precision, size_t smem, int* blocks_per_sm);
cudaError_t launch_adjoint_step(const AdjointArgs& args, int blocks, int precision, size_t smem, cudaStream_t stream);
cudaError_t adjoint_step_max_blocks(int precision, size_t smem, int* blocks_per_sm);
cudaError_t launch_apply_inverse(const int* s_off, const int* s_col, const double* s_val, const int* st_off,
                                 const int* st_col, const double* st_val, int rows, const double* rhs, double* work,
                                 double* out, cudaStream_t stream);
// Writes a barrier's poll budget (after the launch's barrier was cleared).
cudaError_t launch_set_spin_limit(GridBarrier* barrier, unsigned limit, cudaStream_t stream);
// Cooperative probe of the bounded waits: `blocks` blocks wait at a barrier
// that expects blocks + missing arrivals (mode 0: grid_sync; mode 1: the
// serial-section barrier). Every block counts itself in `returned` once its
// wait has given up.
cudaError_t launch_barrier_probe(GridBarrier* barrier, int* status, int* returned, int blocks, int missing, int mode,
                                 cudaStream_t stream);
cudaError_t launch_hex_determinants(const float* q, const int* indices, const double* gradients, int ne, double* out,
                                    cudaStream_t stream);

}  // namespace pdb200
