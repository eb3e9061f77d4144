// Device-side description of a batch of independent projective-dynamics
// instances advanced together.
//
// The batched step runs each phase of the local/global iteration as its own
// kernel over the work of every instance that is still iterating: the local
// step over all element samples, the gather over all particles, the two
// factor products over all factor rows, and the Anderson/convergence phase
// with one block per instance. The iterations of a step repeat inside a CUDA
// graph WHILE node whose condition the Anderson kernel sets on the device, so
// a whole rollout is one graph launch with no host round trip.
//
// The factor of each instance is stored as run matrices in postorder labels
// (runs.h): particle vectors entering and leaving the products are permuted
// by label_of / particle_of, everything else stays in particle order.
#pragma once

#include "pd_device.cuh"

namespace pdb200 {

// A factor in run format: row u has runs [row_runs[u], row_runs[u+1]); run k
// covers columns run_col[k] .. run_col[k] + (run_off[k+1] - run_off[k]) - 1
// with its values at values[run_off[k] ...].
struct RunView {
  const int* row_runs;
  const int* run_col;
  const int* run_off;
  const void* values;  // TV
};

struct BatchInstance {
  // Mesh (device arrays of the instance's solver)
  int n, ne, corners, hex;
  const int* indices;
  const double* gradients;
  const int* free_;
  const int* inc_offsets;
  const int* inc_entries;
  const double* plane_weight;
  double plane[4];
  // Materials and energies
  const double* wc;
  const double* wv;
  const double* wn;
  const double* wm;
  const double* mdir;
  double* mtarget;
  int has_muscles;
  int material;
  double nh_mu, nh_lame, nh_penalty;
  int* status;
  // Factor in labels and the constant matrix (particle order) for refinement
  RunView s, st;
  const int* label_of;
  const int* particle_of;
  const int* a_off;
  const int* a_col;
  const double* a_val;
  int refine;
  // Warm-start singular vectors [samples][9] in the local-step precision
  void* svd_u;
  void* svd_v;
  // Step vectors [n][3] float64, particle order
  double* position;
  double* velocity;
  double* target;
  double* boundary;
  double* x;
  double* prev;
  double* proj;
  double* prev_proj;
  double* contrib;
  // Product vectors [n][3] in labels, factor precision
  void* rhs;
  void* y;
  // Anderson: history ring, Gram cache by ring slot pair, state
  int window;
  double* hist_x;
  double* hist_g;
  double* gram;   // [(kMaxWindow+1)^2]
  int* aa_state;  // count, start, count used, start used
  int* step;      // the instance's current step of the rollout
  // Loop control
  int* iteration;
  int* active;
  int max_iterations;
  double abs_tol, rel_tol;
  double mass, inertia;
  int integrate_pinned;
  int state_f64;
  // Offsets into the batch's concatenated particle and element arrays
  long long particle_offset;
  long long element_offset;
};

// Pointers of one step: concatenated [P][3] states of all instances. A
// rollout holds one entry per step in device memory.
struct BatchStepIo {
  const void* q_in;
  const void* qd_in;
  const void* f_in;
  void* q_out;
  void* qd_out;
  double* x_record;  // [P][3] float64, or nullptr
};

// Work items of the task-parallel kernels.
struct RangeTask {
  int inst;
  int begin;
  int end;
};

struct RowTask {
  int inst;
  int r0, r1;  // rows (labels)
  int c0, c1;  // columns their runs touch (labels): the staged vector window
};

// Task kinds of the work-list kernels.
constexpr int kTaskLocal = 0;
constexpr int kTaskGather = 1;
constexpr int kTaskS = 2;
constexpr int kTaskSt = 3;
constexpr int kTaskKinds = 4;

// Work list of one pass: the instances still iterating and, per task kind,
// the prefix sums of their task counts. The kernels of a pass run a fixed
// grid that strides over the listed tasks, so a pass with few instances left
// costs little more than its launches. Rebuilt by the last Anderson block.
struct ScheduleView {
  int count;              // instances in the batch
  int* n_active;          // [1]
  int* active;            // [count]: instance ids, ascending
  int* prefix;            // [kTaskKinds][count + 1]
  const int* task_begin;  // [kTaskKinds][count + 1]: first task of each instance (static)
};

// Iteration control shared by the blocks of the Anderson kernel.
struct BatchControl {
  unsigned arrived;
  unsigned active;
  unsigned passes;       // passes of the current rollout
  unsigned last_active;  // instances still iterating after the last pass
};

}  // namespace pdb200
