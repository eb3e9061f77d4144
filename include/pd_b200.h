/*
 * C ABI of the B200 DiffPhD projective-dynamics step and its adjoint.
 *
 * This library replaces the device path of the reference's Newton solver
 * plugin `SolverDiffPhD` (src/newton_solver_diff_phd/_src/solvers/diff_phd/
 * solver.py). The reference is Python over NVIDIA Warp and exposes no C
 * interface of its own; each entry point below names the reference call it
 * stands in for. Host code (the Python package newton_solver_diff_phd_b200)
 * validates the model exactly like the reference and hands plain arrays here.
 *
 * Conventions
 *  - Every function returns PD_OK (0) or a PD_ERR_* code; pd_last_error()
 *    returns a thread-local message for the last failure.
 *  - Device pointers are marked "device"; everything else is host memory.
 *    Vectors of particles are float32 xyz triples (Newton's wp.vec3) unless
 *    stated as double.
 *  - Steps and backward passes are asynchronous on the caller's stream. Solver
 *    failures never interrupt the device: they set bits of a device status
 *    word that pd_read_status() returns (the reference's status contract,
 *    kernels.py:28-31, adjoint.py:64-65).
 *  - A solver instance serialises its own launches: use one stream per
 *    instance at a time (the reference's single-stream rule, sparse.py:280-282).
 */
#ifndef PD_B200_H
#define PD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PD_OK 0
#define PD_ERR_INVALID 1   /* invalid argument; the reference raises ValueError */
#define PD_ERR_CUDA 2      /* a CUDA runtime call failed */
#define PD_ERR_NOT_SPD 3   /* the constant matrix is not positive definite (sparse.py:139-140) */
#define PD_ERR_STATE 4     /* wrong call order, e.g. step before build; RuntimeError in the reference */
#define PD_ERR_UNSUPPORTED 5 /* NotImplementedError in the reference */

/* Device status bits (solver.py:380-387, kernels.py:28-31, adjoint.py:64-65). */
#define PD_STATUS_NOT_CONVERGED 1
#define PD_STATUS_SINGULAR 2
#define PD_STATUS_ACTIVATION 4
#define PD_STATUS_ADJOINT_NOT_CONVERGED 8
#define PD_STATUS_ADJOINT_SAFEGUARD 16
/* A device barrier gave up waiting (bounded spin); the step result is invalid. */
#define PD_STATUS_BARRIER_TIMEOUT 1024

#define PD_MATERIAL_PD 0          /* corotated 2 mu + volume lambda */
#define PD_MATERIAL_NEO_HOOKEAN 1 /* proximal Neo-Hookean, weight 2 mu */

#define PD_PRECISION_FP64 0        /* every solver operation in float64, as the reference */
#define PD_PRECISION_FP32_REFINE 1 /* fp32 factor products with fp64 residual refinement; fp64 local step:
                                      the converged positions are the fp64 solver's */
#define PD_PRECISION_FP32 2        /* fp32+refine with fp32 local projections and adjoint Jacobians: fastest;
                                      the fixed point moves by about cond(A) * 6e-8 relative */

#define PD_ADJOINT_REFERENCE 0 /* K with the mean weight per energy (adjoint.py:17-18) */
#define PD_ADJOINT_EXACT 1     /* K with per-element weights: the derivative of the forward map */

#define PD_ADJOINT_SOLVER_AUTO 0        /* fixed point for the reference mode, CG for the exact mode */
#define PD_ADJOINT_SOLVER_FIXED_POINT 1 /* mu <- A^{-1}(g + K mu) with Anderson and safeguards (adjoint.py:927-1086) */
#define PD_ADJOINT_SOLVER_CG 2          /* CG on (A - K) mu = g preconditioned by A^{-1} = S^T S */

typedef struct PdSolver PdSolver;

typedef struct PdMeshDesc {
  int32_t n_vertices;
  int32_t n_elements;
  int32_t corners;         /* 4: Tet4, 8: Hex8 (eight Gauss samples per cell) */
  const int32_t* indices;  /* [n_elements][corners] */
  /* Tet4: [n_elements][4][3] rest shape gradients G (solver.py:218-219).
     Hex8: [8 samples][8 corners][3] shared Gauss gradients (hex.py:64-79). */
  const double* gradients;
  double mean_volume;      /* Vbar: every element's volume and the mass basis */
  const uint8_t* free;     /* [n_vertices]; 0 marks a Dirichlet (zero inverse mass) particle */
} PdMeshDesc;

typedef struct PdOptions {
  int32_t material;          /* PD_MATERIAL_* */
  int32_t max_iterations;    /* >= 1 */
  double abs_tol;            /* >= 0 */
  double rel_tol;            /* >= 0 */
  int32_t anderson_window;   /* 0..8 */
  double density;            /* > 0 */
  int32_t integrate_pinned_velocities;
  int32_t precision;         /* PD_PRECISION_* */
  int32_t adjoint_mode;      /* PD_ADJOINT_* */
  int32_t blocks;            /* persistent grid size; 0 = automatic */
  int32_t resident;          /* 1: keep factor slices in shared memory when they fit (default) */
  int32_t svd_warm_start;    /* 1: warm-start each sample's SVD from the previous iteration (default) */
  int32_t adjoint_solver;    /* PD_ADJOINT_SOLVER_* */
  int32_t state_precision;   /* 0: float32 particle states (Newton's), 1: float64 states and gradients */
} PdOptions;

/* Library identity and the message of the last failure on this thread. */
const char* pd_version(void);
const char* pd_last_error(void);

/* SolverDiffPhD.__init__ (solver.py:157-333): copies the mesh to the device.
   `device` is the CUDA ordinal. */
int pd_create(const PdMeshDesc* mesh, const PdOptions* options, int device, PdSolver** out);
/* Releases all device memory of the instance. */
int pd_destroy(PdSolver* solver);

/* Mutable convergence settings (solver.max_iterations / abs_tol / rel_tol). */
int pd_set_tolerances(PdSolver* solver, int32_t max_iterations, double abs_tol, double rel_tol);

/* Anderson window (0..8) of the following steps and backward passes; the
   history grows when needed. The reference fixes it at construction
   (anderson_window keyword); changing it lets a driver tune it. */
int pd_set_anderson_window(PdSolver* solver, int32_t window);

/* Lame parameters [mu, lambda] per element (model.tet_materials columns 0-1,
   or hex_materials), float64 host array [n_elements][2]. Marks the factor
   stale (notify_model_changed, solver.py:419-427). */
int pd_set_materials(PdSolver* solver, const double* mu_lambda);

/* Fibres (solver.py:429-462): unit directions [n_elements][3] (zero rows for
   disabled fibres) and stiffness [n_elements] in Pa. Pass NULLs to disable. */
int pd_set_muscles(PdSolver* solver, const double* directions, const double* stiffness);

/* Hex8 native fibre target lengths [n_elements] (solver.muscle_targets).
   `targets` is a host float64 array. */
int pd_set_muscle_targets(PdSolver* solver, const double* targets);

/* Tet4 fibre contractions u (target length 1 - u) for the following steps,
   a device float32 array [n_elements] read at every step
   (read_activations, kernels.py:136-152). NULL keeps zero contraction. */
int pd_set_activations(PdSolver* solver, const float* device_contractions);

/* Hex8 vertex-plane energies (hex.py:204-260): vertex indices, stiffness per
   vertex and the normalised plane (nx, ny, nz, offset). count 0 disables. */
int pd_set_planar_energies(PdSolver* solver, int32_t count, const int32_t* vertices, const double* stiffness,
                           const double plane[4]);

/* The reference's mesh_contact state force between two bodies
   (mesh_contact.py:185-272, wired in solver.py:321-325 and :762-770): radius
   [m], normal stiffness of A's vertices against B's faces (kn_left) and of B's
   against A's (kn_right) [N/m], friction bound kf [N s/m], Coulomb mu, and the
   surface triangles [n][3] (particle indices, host arrays) of A and B. Every
   following step evaluates it on its start-of-step state and adds h^2/m f to
   the inertial target; it has no gradient, as in the reference. Tet4 only. */
int pd_set_mesh_contact(PdSolver* solver, double radius, double kn_left, double kn_right, double kf, double mu,
                        int32_t n_faces_a, const int32_t* faces_a, int32_t n_faces_b, const int32_t* faces_b);
/* MeshContact.evaluate (mesh_contact.py:253-272) on given float64 device
   positions and velocities [n][3]: force (device float64 [n][3], or NULL)
   and the number of vertex-face pairs within the radius (host, or NULL;
   synchronises). */
int pd_mesh_contact_force(PdSolver* solver, const double* q, const double* v, double* force, int32_t* pairs,
                          void* stream);
/* Pairs within the radius at the last step (solver.mesh_contact_pairs, solver.py:351-353). Synchronises. */
int pd_mesh_contact_pairs(PdSolver* solver, int32_t* pairs, void* stream);

#define PD_BOUNDARY_PLANAR 0    /* parameters (nx, ny, nz, offset): gap (n.x + offset) / |n| */
#define PD_BOUNDARY_SPHERICAL 1 /* parameters (cx, cy, cz, radius): gap |x - c| - radius */
#define PD_BOUNDARY_MESH 2      /* parameters[0] = contact radius; faces_left / faces_right, split index */
/* The reference's frictional boundary (FrictionalContact, contact.py:684-1015;
   SolverDiffPhD(frictional_boundary=..., frictional_vertices=..., friction=...,
   restitution=...), solver.py:170-171 and :303-320): `count` registered
   particles `nodes` (host, unique). Every local/global iteration of the
   following steps takes one Fischer-Burmeister Newton step on their normal
   multipliers and a Coulomb stick/slip update, and restitution acts after
   convergence. The mesh kind tests vertices below `split` against faces_right
   and the others against faces_left (host [n][3]); the other kinds ignore
   split and faces. The multipliers start from zero at every factor build and
   warm-start the following steps. Tet4 only; one boundary per solver. */
int pd_set_frictional_boundary(PdSolver* solver, int32_t kind, const double parameters[4], int32_t count,
                               const int32_t* nodes, double friction, double restitution, int32_t split,
                               int32_t n_left, const int32_t* faces_left, int32_t n_right,
                               const int32_t* faces_right);
/* Device pointers of the boundary parameters (float64 [4]; planar and
   spherical kinds read them at every step, so edits between steps and
   between graph replays take effect: solver.boundary_parameters,
   solver.py:340-343) and of the normal multipliers (float64 [count]; the
   warm start: solver.contact_multipliers, solver.py:345-348). */
int pd_frictional_buffers(PdSolver* solver, double** parameters, double** multipliers, int32_t* count);
/* Copies of the last step's contact state (the StepRecord snapshot,
   adjoint.py:834-841): multipliers [count], omega [count], normals [count][3]
   and mesh candidate flags [count] into caller buffers (device or host,
   NULL to skip), ordered on `stream`. */
int pd_frictional_state(PdSolver* solver, double* multiplier, double* omega, double* normal, int32_t* candidate,
                        void* stream);

/* SolverDiffPhD._build (solver.py:491-552): assembles the constant matrix
   A = m/h^2 I + sum_e w_e Vbar G_e^T G_e (+ fibres, + plane diagonal) and builds
   the exact inverse factor A^{-1} = S^T S on the host (sparse.py:291-320),
   then uploads it. Synchronous; not capturable. */
int pd_build(PdSolver* solver, double dt);
/* Where pd_build runs the numeric LDL^T and the rows of L^{-1}: 1 on the
   solver's device (see pd_inverse_build_on), 0 on the host (default).
   Bit-identical either way; takes effect at the next build. Added (no
   reference counterpart). */
int pd_set_factor_device(PdSolver* solver, int32_t enabled);

/* Factor statistics of the last build: rows, nnz(S), nnz(L) incl. diagonal. */
int pd_factor_stats(const PdSolver* solver, int64_t* rows, int64_t* nnz_s, int64_t* nnz_l);

/* SolverDiffPhD.step (solver.py:689-786).
   Particle arrays are float32 (Newton's states), or float64 when the solver
   was created with state_precision 1 (the same holds for the gradient arrays
   of pd_backward).
   q, qd, f: device [n][3] inputs; dirichlet: optional device [n][3]
   prescribed positions of the pinned particles (or NULL); gravity: host [3];
   q_out, qd_out: device [n][3] float32 outputs (must not alias the inputs);
   x_record: optional device [n][3] float64 that receives the converged
   positions for pd_backward (the reference StepRecord.x, adjoint.py:809-841).
   dt must equal the dt of the last pd_build. `stream` is a cudaStream_t. */
int pd_step(PdSolver* solver, const void* q, const void* qd, const void* f, const void* dirichlet,
            const double gravity[3], double dt, void* q_out, void* qd_out, double* x_record, void* stream);

/* Adjoint.backward (adjoint.py:1088-1259) of one recorded step.
   x_record: device [n][3] float64 positions recorded by pd_step; activations:
   the device contractions used by that step (or NULL).
   gq_out, gqd_out: device float32 [n][3] gradients of the step outputs.
   gq, gqd, gf: device float32 [n][3] accumulators (+=) for the gradients of
   the step inputs q, qd, f; gdirichlet: optional device float32 [n][3]
   accumulator when the step used explicit Dirichlet targets.
   gmaterials: optional device float64 [n_elements][2] accumulator (+=) of
   dL/dmu, dL/dlambda; gactivations: optional device float32 [n_elements]
   accumulator of dL/du. Passing gmaterials/gactivations requests z, exactly
   as a requires_grad material array does in the reference. */
int pd_backward(PdSolver* solver, const double* x_record, const float* activations, double dt, const void* gq_out,
                const void* gqd_out, void* gq, void* gqd, void* gf, void* gdirichlet, double* gmaterials,
                float* gactivations, void* stream);
/* pd_backward of a step with a frictional boundary, given the contact state
   that step recorded (pd_frictional_state right after it: device float64
   multipliers [count], omega [count], normals [count][3]). When material or
   activation gradients are requested, they use the reference's contact
   projection z = mu - W_T G^{-1} (J mu) (Adjoint._woodbury, adjoint.py:1272-1354):
   one adjoint fixed point per selected contact row, capped at
   min(max_iterations, 120) iterations; the state gradients use mu as in the
   reference. Reads the selected row count back to the host once (synchronises
   `stream`). NULL snapshot pointers make it pd_backward. */
int pd_backward_contact(PdSolver* solver, const double* x_record, const float* activations, double dt,
                        const void* gq_out, const void* gqd_out, void* gq, void* gqd, void* gf, void* gdirichlet,
                        double* gmaterials, float* gactivations, const double* multiplier, const double* omega,
                        const double* normal, void* stream);
/* How pd_backward_contact solves two or more selected columns. 1 (default):
   side by side, as many per launch as the grid holds, each on its own lane
   of blocks with its own vectors (the reference solves its columns in
   batches, adjoint.py:666-806); 0: one launch per column, one after the
   other. Both give the same gradients to rounding. */
int pd_set_woodbury_lanes(PdSolver* solver, int32_t enabled);
/* Blocks per lane of those columns: 0 (default) picks it from nnz(S) and the
   element samples; 1, 2, 4, ..., 64 fixes it (a tuning knob; the reference
   has none). Fewer blocks per lane give more lanes per launch. */
int pd_set_woodbury_team(PdSolver* solver, int32_t blocks);

/* Device buffer of 8 uint64 nanosecond accumulators for the per-phase timers
   of a library built with -DPD_PHASE_TIMERS (profiling); ignored otherwise.
   NULL disables. */
int pd_set_phase_timers(PdSolver* solver, unsigned long long* device_timers);

/* Failure detection of the device barriers (the reference's status contract,
   kernels.py:28-31, has no barrier of its own: Warp launches are separate).
   Every wait of a persistent launch polls a bounded number of times, then
   sets PD_STATUS_BARRIER_TIMEOUT, raises the team's abort flag and returns.
   pd_set_spin_limit lowers that poll budget for the solver's following step
   and backward launches (0 restores the built-in budget of 2^26 polls), so a
   test can make the waits run out. pd_barrier_probe launches `blocks`
   cooperative blocks (at most one per SM) on a barrier that expects
   `missing` more arrivals than are launched, with a budget of `polls`
   (mode 0: the plain grid barrier; mode 1: the serial-section barrier), and
   returns the status bits and how many blocks gave up and returned.
   Synchronises the device. */
int pd_set_spin_limit(PdSolver* solver, uint32_t polls);
int pd_barrier_probe(int device, int32_t blocks, int32_t missing, int32_t mode, uint32_t polls, int32_t* status,
                     int32_t* returned);

/* Reads and clears the status word (read_status, solver.py:380-390). Synchronises the stream. */
int pd_read_status(PdSolver* solver, int32_t* bits, void* stream);
/* Iteration count of the last step and of the last backward fixed point. Synchronises the stream. */
int pd_iterations(PdSolver* solver, int32_t* forward, int32_t* backward, void* stream);

/* det(F) at every Hex8 Gauss sample (deformation_determinants, solver.py:360-378):
   q device float32 [n][3], out device float64 [n_elements][8]. */
int pd_deformation_determinants(PdSolver* solver, const float* q, double* out, void* stream);

/* Applies the uploaded factor: out = S^T (S rhs), device float64 [n][3] arrays
   (SparseInverse.apply, sparse.py:350-352). */
int pd_apply_inverse(PdSolver* solver, const double* rhs, double* out, void* stream);

/* out = S^T (S rhs) without any allocation; no counterpart in the reference.
   For callers that cannot allocate device memory when they solve (inside a
   stream capture, under a host-owned allocator, in a real-time loop): the
   intermediate vector lives in a file-scope device array of at most 65536
   particles (1.5 MiB, resident on each GPU that loads the library until
   exit). Rejects larger solvers with PD_ERR_INVALID, built or not. The
   first call on a device resolves the array's address and must come before
   any stream capture. All calls share the array: calls that overlap on the
   GPU race. The caller's current device is the same after the call. */
int pd_apply_inverse_static(PdSolver* solver, const double* rhs, double* out, void* stream);

/* ---- The DiffPD pd_eigen forward step (SolverDiffPD, reference
   src/newton_solver_diff_phd/_src/solvers/diff_pd/solver.py:65-591). It runs on a
   Tet4 solver created and built as usual, whose materials are mu = w_c / 2
   and lambda = w_v for every element (so its constant matrix and inverse
   factor are DiffPD's A = m/h^2 I + (w_c + w_v) Vbar sum_e G_e G_e^T). Each
   step minimises 1/2 m/h^2 |x - rhs|^2 + E_pd(x) by L-BFGS with A^{-1} as
   initial inverse Hessian and a backtracking Armijo line search, in one
   persistent launch. Status bits (pd_read_status): 1 not converged within
   max_pd_iter, 2 a singular deformation gradient met the volume projection,
   4 a line search used all max_ls_iter halvings (informational). */
typedef struct PdDiffPdOptions {
  int32_t max_pd_iter;     /* >= 1 */
  int32_t max_ls_iter;     /* >= 1 */
  int32_t history;         /* L-BFGS pairs, 2..32 */
  int32_t use_corotated;   /* 1: the corotated energy w_c/2 |F - R|^2 is on */
  int32_t use_volume;      /* 1: the volume energy w_v/2 |F - P_v(F)|^2 is on */
  double corotated_weight; /* w_c [Pa] */
  double volume_weight;    /* w_v [Pa] */
  double abs_tol;          /* [N] */
  double rel_tol;          /* relative to |m/h^2 rhs| over the free rows */
  int32_t recursion;       /* PD_DIFFPD_TWO_LOOP or PD_DIFFPD_GRAM */
} PdDiffPdOptions;
/* The L-BFGS direction. TWO_LOOP: the reference's two loops, one team sum per
   pair and loop. GRAM: the same recursion from the Gram matrix s_i . y_j of
   the stored pairs and the products s_i . g, two batched team sums per
   iteration; the dot products are rounded in another order. */
#define PD_DIFFPD_TWO_LOOP 0
#define PD_DIFFPD_GRAM 1
/* The explicit contact state forces after gravity (SolverDiffPD(state_forces=...),
   solver.py:24-56): kinds[count] (0 planar_contact, 1 arc_contact) and packed
   rows parameters[count][18] (planar: unit normal, offset / |n|, p, kn, kf, mu;
   arc: center, unit axis, unit start, axis x start, radius, angle, p, kn, kf,
   mu). Host arrays, copied. count 0 removes them. */
int pd_diffpd_set_state_forces(PdSolver* solver, int32_t count, const int32_t* kinds, const double* parameters);
/* SolverDiffPD.step (solver.py:539-591): q, qd, f device [n][3] in the state
   precision; gravity host [3] (the gravity state force); q_out, qd_out device
   outputs (distinct from the inputs). dt must equal the last pd_build's dt. */
int pd_diffpd_step(PdSolver* solver, const PdDiffPdOptions* options, const void* q, const void* qd, const void* f,
                   const double gravity[3], double dt, void* q_out, void* qd_out, void* stream);
/* Device float64 [n][3] positions and velocities of the last DiffPD step
   (solver.positions / solver.velocities, solver.py:260-268) and its L-BFGS
   iteration count (host; synchronises `stream` when requested). */
int pd_diffpd_results(PdSolver* solver, double** positions, double** velocities, int32_t* iterations, void* stream);

/* ---- Batched rollouts.
   Many independent built solvers (uneven sizes allowed) advanced together in
   one CUDA graph per rollout. Under the default TEAMS schedule the graph is
   one persistent cooperative launch: every instance runs all its steps on a
   team of blocks with the single-instance step body (PHASES, kept for
   comparison: per-phase kernels over all iterating instances in a graph WHILE
   loop, the factor in postorder run format). Each instance follows the same
   algorithm as pd_step (solver.py:582-687: local step, gather, S^T S solve,
   Anderson, dual convergence gate) with its own tolerances and iteration
   limit. The reference steps one model at a time; batching has no
   counterpart there. Instances do not wait for each other between steps.
   Every solver must be built for the same dt, on one device, with one
   precision and one state precision, without Dirichlet targets or Tet4
   activations. The solvers must outlive the batch and must not step on
   their own while a batched rollout runs (the batch uses their buffers). */
typedef struct PdBatch PdBatch;
/* Schedules of a batch.
   TEAMS: one persistent cooperative launch per rollout; every instance runs
   all its steps on a team of blocks sized to its factor and element count,
   with the single-instance step body (and adjoint body) and its own team
   barriers; teams form from a queue as blocks finish earlier instances.
   PHASES: per-phase kernels over all instances inside a graph WHILE loop,
   the factor in postorder run format (forward only). */
#define PD_BATCH_TEAMS 0
#define PD_BATCH_PHASES 1
typedef struct PdBatchOptions {
  int32_t svd_warm_start; /* phases: 1 = warm-started SVD after the first iteration */
  int32_t task_nnz;       /* phases: factor entries per product task (>= 256; default 32768) */
  int32_t run_gap;        /* phases: omitted zeros bridged inside a run (default 2) */
  int32_t local_cells;    /* phases: Hex8 cells per local-step task (>= 4; default 64) */
  int32_t schedule;       /* PD_BATCH_TEAMS (default) or PD_BATCH_PHASES */
  int32_t team_nnz;       /* teams: factor entries of S per block of a team (default 65536) */
  int32_t team_samples;   /* teams: element samples per block of a team (default 512) */
  /* teams, optional (all three or none): a previous rollout of the same
     instances measured per instance, [count] each: its duration on its lane
     [us] (pd_batch_timeline), its total local/global iterations
     (pd_batch_read) and the team size it ran with (pd_batch_team_sizes).
     Team sizes and lanes are then planned from these costs: instances whose
     estimated duration would set the makespan get larger teams, and lanes
     go to the classes with the longest estimated completion. */
  const double* measured_us;
  const int32_t* measured_iterations;
  const int32_t* measured_team;
  /* teams, optional with the three above: each instance's last adjoint
     rollout duration [us]; the adjoint launch then gets its own lane counts
     and queue order (same team sizes). NULL: the adjoint uses the forward's lanes. */
  const double* measured_adjoint_us;
} PdBatchOptions;
/* options may be NULL (defaults). */
int pd_batch_create(PdSolver* const* solvers, int32_t count, const PdBatchOptions* options, PdBatch** out);
int pd_batch_destroy(PdBatch* batch);
/* First particle / element of each instance in the concatenated arrays, [count + 1] each. */
int pd_batch_layout(const PdBatch* batch, int64_t* particle_offsets, int64_t* element_offsets);
/* Stored factor values (S and S^T), runs, and task counts [local, gather, S, S^T]. */
int pd_batch_factor_stats(const PdBatch* batch, int64_t* values, int64_t* runs, int64_t* tasks);
/* Rollout of `steps` PD steps of every instance (SolverDiffPhD.step repeated,
   solver.py:689-786). q0, qd0: device [P][3] in the state precision (P = all
   particles); forces: device [P][3] per step, step t at forces + t *
   force_step_stride elements (0: the same forces every step); q_traj,
   qd_traj: device [steps][P][3] outputs; x_record: device float64
   [steps][P][3] or NULL. The graph is rebuilt when any pointer, steps, dt or
   gravity differs from the previous call. */
int pd_batch_forward(PdBatch* batch, int32_t steps, double dt, const double gravity[3], const void* q0,
                     const void* qd0, const void* forces, int64_t force_step_stride, void* q_traj, void* qd_traj,
                     double* x_record, void* stream);
/* Adjoint of the last rollout (teams schedule), last step first (the
   reference's tape replay, adjoint.py:1088-1259, per step): x_record the
   forward's float64 [steps][P][3] record; grad_q_final / grad_qd_final the
   loss gradient w.r.t. the final state [P][3]; grad_q / grad_qd scratch of
   [2][P][3] each, where dL/dq0 and dL/dqd0 end in slot (steps - 1) & 1;
   grad_forces [steps][P][3] receives dL/df of every step; grad_materials
   float64 [E][2] (or NULL) receives dL/d(mu, lambda) per element. State
   arrays use the state precision. iterations (host [steps][count], or NULL)
   receives every adjoint step's solver iterations and synchronises. */
int pd_batch_backward(PdBatch* batch, int32_t steps, double dt, const double* x_record, const void* grad_q_final,
                      const void* grad_qd_final, void* grad_q, void* grad_qd, void* grad_forces,
                      double* grad_materials, int32_t* iterations, void* stream);
/* Global-timer nanoseconds [count][2] at which each instance's last forward
   and adjoint rollout started and ended on its lane (teams schedule). Either
   pointer may be NULL. Synchronises. */
int pd_batch_timeline(PdBatch* batch, uint64_t* forward, uint64_t* adjoint, void* stream);
/* Phase timers of one instance's forward steps in the teams schedule: device
   uint64 [8] accumulating global-timer nanoseconds per phase, written only by
   builds compiled with -DPD_PHASE_TIMERS (as pd_set_phase_timers). */
int pd_batch_set_phase_timers(PdBatch* batch, int32_t instance, unsigned long long* device_timers);
/* Team size of every instance (0 under the phases schedule) and the grid of the team launch. */
int pd_batch_team_sizes(const PdBatch* batch, int32_t* sizes, int32_t* grid);
/* The same rollout without a graph: every kernel launched on its own, the
   loop decided on the host every 16 passes (synchronises). For profilers
   that follow plain launches; results equal pd_batch_forward's. Phases
   schedule only. */
int pd_batch_forward_stepwise(PdBatch* batch, int32_t steps, double dt, const double gravity[3], const void* q0,
                              const void* qd0, const void* forces, int64_t force_step_stride, void* q_traj,
                              void* qd_traj, double* x_record, void* stream);
/* Status bits per instance accumulated since the last read, [count] (the read
   clears them, like pd_read_status), and the iteration count of every step
   of the last rollout, [steps][count]. Either pointer may be NULL.
   Synchronises the stream. */
int pd_batch_read(PdBatch* batch, int32_t* status, int32_t* iterations, void* stream);

/* Host factor build for an arbitrary SPD matrix given as full symmetric CSR
   (SparseInverse.__init__, sparse.py:291-320). Arrays are host memory; the
   result is freed with pd_inverse_free. */
typedef struct PdInverseFactor PdInverseFactor;
/* Update work (entries of earlier rows a row combines) from which a row of
   the inverse factor is computed by all host threads, each on a column range
   (default 65536; 0: every row). The factor is bit-identical either way.
   Process-wide setting. */
int pd_inverse_parallel_work(int64_t work);
/* Entries of L (its nonzeros, diagonal included) from which the numeric LDL^T
   (sparse.py:136-151) and the rows of L^{-1} (sparse.py:159-177) run over all
   host threads level by level of the elimination tree (left-looking columns;
   rows as dense segments in groups of consecutive rows and 256-label chunks)
   instead of the sequential right-looking loop and the row-by-row walk
   (default 32,768; 0: every factor). Every entry sees the same sequence of
   rounded operations either way: the factor is bit-identical. Process-wide
   setting. */
int pd_inverse_parallel_levels(int64_t entries);
/* How the device computes the rows of L^{-1} when the factor build runs on
   the device (pd_set_factor_device, pd_inverse_build_on): 0 (default) rows in
   256-label chunks, one block per (row, chunk), a block barrier per column k;
   1 the host's grouped dense segments (groups of up to 32 consecutive rows),
   one block per (group, chunk) and one thread per label holding the group's
   entries in registers, no barriers, levels launched back to back. Both are
   bit-identical to the host walk by construction; mode 1 has not yet run on
   a GPU. Process-wide setting. */
int pd_factor_device_rows(int32_t mode);
int pd_inverse_build(int32_t size, const int32_t* row_offsets, const int32_t* columns, const double* values,
                     PdInverseFactor** out);
/* pd_inverse_build with the numeric LDL^T (sparse.py:136-151) and the rows of
   L^{-1} (sparse.py:159-177), the two costly stages, computed on CUDA device
   `device`, level by level of the elimination tree; ordering, symbolic fill
   and the CSR assembly stay on the host. The factor is bit-identical to the
   host build (rows of L longer than the device stages take run on the
   host). device < 0 builds on the host. Added: the reference builds on the
   host only. */
int pd_inverse_build_on(int32_t device, int32_t size, const int32_t* row_offsets, const int32_t* columns,
                        const double* values, PdInverseFactor** out);
int pd_inverse_sizes(const PdInverseFactor* factor, int32_t* size, int64_t* nnz, int64_t* factorization_nnz);
/* Copies the arrays: permutation[size], s_offsets[size+1], s_columns[nnz], s_values[nnz],
   st_offsets[size+1], st_columns[nnz], st_values[nnz]. Any pointer may be NULL. */
int pd_inverse_export(const PdInverseFactor* factor, int32_t* permutation, int32_t* s_offsets, int32_t* s_columns,
                      double* s_values, int32_t* st_offsets, int32_t* st_columns, double* st_values);
int pd_inverse_free(PdInverseFactor* factor);
/* The factor in postorder run format (the storage of the batched path): rows
   of S and S^T as runs of consecutive labels, omitted zeros bridged inside a
   run when at most max_gap of them lie between two stored entries. Sizes
   first; then label_of[size], s_row_runs[size+1], s_run_col[s_runs],
   s_run_off[s_runs+1], s_values[s_values], and the same for S^T. No
   counterpart in the reference (sparse.py keeps CSR only). */
int pd_inverse_run_sizes(const PdInverseFactor* factor, int32_t max_gap, int64_t* s_runs, int64_t* s_values,
                         int64_t* st_runs, int64_t* st_values);
int pd_inverse_run_export(const PdInverseFactor* factor, int32_t max_gap, int32_t* label_of, int32_t* s_row_runs,
                          int32_t* s_run_col, int32_t* s_run_off, double* s_values, int32_t* st_row_runs,
                          int32_t* st_run_col, int32_t* st_run_off, double* st_values);

#ifdef __cplusplus
}
#endif

#endif /* PD_B200_H */
