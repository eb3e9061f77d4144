// Device-side building blocks of the persistent DiffPhD kernels: the bounded
// grid barrier with a last-arriver serial section, fixed-order reductions,
// and the argument block shared by the forward and adjoint kernels.
//
// One cooperative launch runs every local/global iteration of a step. The
// grid is co-resident (cudaLaunchCooperativeKernel refuses otherwise), phases
// are separated by grid barriers, and every wait gives up after a bounded
// number of polls, raising PD_STATUS_BARRIER_TIMEOUT and unwinding the
// kernel instead of hanging the device.
#pragma once

#include <cstdint>

#include "pd_math.cuh"

namespace pdb200 {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr int kPartialStride = 64;  // partial-sum slots per block
constexpr int kMaxWindow = 8;
// Poll budget of one barrier wait (~2^26 polls of >= 32 ns: seconds, far
// beyond any legitimate phase). A nonzero GridBarrier::spin_limit replaces it
// (a test knob: the host writes it after clearing the barrier).
constexpr unsigned kSpinLimit = 1u << 26;

constexpr int kStatusNotConverged = 1;
constexpr int kStatusSingular = 2;
constexpr int kStatusActivation = 4;
constexpr int kStatusAdjointNotConverged = 8;
constexpr int kStatusAdjointSafeguard = 16;
constexpr int kStatusBarrierTimeout = 1024;

// Grid barrier state: one 32-bit word, generation in the high 16 bits and the
// arrival count in the low 16 bits, so arriving is a single atomic and the
// release (generation + 1, count reset) is another.
struct GridBarrier {
  unsigned int state;  // serial-section barriers
  unsigned int abort;
  unsigned int flip;   // plain barriers: arrival count with a flipping high bit
  unsigned int spin_limit;  // polls before a wait gives up; 0: kSpinLimit
};

__device__ __forceinline__ unsigned spin_limit_of(const GridBarrier* bar) {
  const unsigned limit = *reinterpret_cast<const volatile unsigned*>(&bar->spin_limit);
  return limit != 0u ? limit : kSpinLimit;
}

constexpr unsigned kCountBits = 16;
constexpr unsigned kCountMask = (1u << kCountBits) - 1u;

__device__ __forceinline__ unsigned load_volatile(const unsigned* p) { return *reinterpret_cast<const volatile unsigned*>(p); }

__device__ __forceinline__ unsigned load_acquire(const unsigned* p) {
  unsigned value;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(value) : "l"(p) : "memory");
  return value;
}
__device__ __forceinline__ unsigned add_acq_rel(unsigned* p, unsigned value) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(value) : "memory");
  return old;
}
__device__ __forceinline__ void red_release(unsigned* p, unsigned value) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(value) : "memory");
}

// Arrive at the grid barrier. Returns true in the block that arrived last;
// that block must run its serial section and then call barrier_release().
// Every other block must call barrier_wait(). The arrival is an acq_rel
// atomic: this block's writes (ordered before it by __syncthreads and the
// cumulative release) are visible to the block that completes the count,
// which acquires them.
__device__ __forceinline__ bool barrier_arrive(GridBarrier* bar, unsigned& generation, int blocks) {
  __shared__ int s_last;
  __shared__ unsigned s_generation;
  __syncthreads();
  if (blocks == 1) {
    generation = 0;
    return true;
  }
  if (threadIdx.x == 0) {
    const unsigned old = add_acq_rel(&bar->state, 1u);
    s_generation = old >> kCountBits;
    s_last = (old & kCountMask) + 1u == static_cast<unsigned>(blocks);
  }
  __syncthreads();
  generation = s_generation;
  return s_last != 0;
}

// Last arriver: next generation and a zero count in one release atomic.
__device__ __forceinline__ void barrier_release(GridBarrier* bar, unsigned generation, int blocks) {
  __syncthreads();
  if (blocks > 1 && threadIdx.x == 0) red_release(&bar->state, (1u << kCountBits) - static_cast<unsigned>(blocks));
}

// Returns false when the wait gave up (timeout here or an abort elsewhere).
__device__ __forceinline__ bool barrier_wait(GridBarrier* bar, unsigned generation, int* status) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned spins = 0;
    const unsigned limit = spin_limit_of(bar);
    while ((load_acquire(&bar->state) >> kCountBits) == (generation & (kCountMask))) {
      if (load_volatile(&bar->abort) != 0u) {
        ok = 0;
        break;
      }
      if (++spins > limit) {
        atomicOr(status, kStatusBarrierTimeout);
        atomicExch(&bar->abort, 1u);
        ok = 0;
        break;
      }
      if (spins > 256) __nanosleep(20);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Plain barrier without a serial section: block 0 adds 2^31 - (blocks - 1),
// every other block adds 1, so the arrival that completes the count also
// flips the high bit and resets the low bits; waiters poll for the flip. One
// atomic per block and no separate release.
__device__ __forceinline__ bool grid_sync(GridBarrier* bar, int* status, int blocks, int rank) {
  __shared__ int s_ok;
  __syncthreads();
  if (blocks == 1) return true;
  if (threadIdx.x == 0) {
    const unsigned increment = rank == 0 ? 0x80000000u - static_cast<unsigned>(blocks - 1) : 1u;
    const unsigned old = add_acq_rel(&bar->flip, increment);
    int ok = 1;
    unsigned spins = 0;
    const unsigned limit = spin_limit_of(bar);
    while (((old ^ load_acquire(&bar->flip)) & 0x80000000u) == 0u) {
      if (load_volatile(&bar->abort) != 0u) {
        ok = 0;
        break;
      }
      if (++spins > limit) {
        atomicOr(status, kStatusBarrierTimeout);
        atomicExch(&bar->abort, 1u);
        ok = 0;
        break;
      }
      if (spins > 256) __nanosleep(20);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) v += __shfl_xor_sync(0xffffffffu, v, offset);
  return v;
}

// Deterministic block-wide sum of one value per thread; result valid in all threads.
__device__ __forceinline__ double block_sum(double v, double* scratch /* [kWarps] */) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double total = 0.0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) total += scratch[w];
  return total;
}


// Sums slots [offset, offset + count) over all blocks in a fixed order. The
// blocks of a slot are cut into kReduceChunks contiguous chunks; one thread
// sums a chunk (all its loads issued together), then one thread per slot adds
// the chunk sums in chunk order. Every load of the reduction is in flight at
// once, so the latency is about one L2 round trip. Uses the whole block;
// results land in out[0..count) (shared memory) for every thread.
constexpr int kReduceChunks = 8;
constexpr int kReduceChunkMax = 32;  // blocks per chunk: grids up to 256 blocks

__device__ __forceinline__ void reduce_partials(const double* partials, int offset, int count, int blocks,
                                                double* out /* shared [count] */,
                                                double* scratch /* shared [>= kBlock] */) {
  const int chunk = (blocks + kReduceChunks - 1) / kReduceChunks;
  for (int base = 0; base < count * kReduceChunks; base += blockDim.x) {
    const int t = base + threadIdx.x;
    double sum = 0.0;
    if (t < count * kReduceChunks) {
      const int slot = t / kReduceChunks;
      const int c = t % kReduceChunks;
      const double* row = partials + (offset + slot) * blocks;
      const int b0 = c * chunk;
      double values[kReduceChunkMax];
#pragma unroll
      for (int k = 0; k < kReduceChunkMax; ++k) values[k] = (k < chunk && b0 + k < blocks) ? row[b0 + k] : 0.0;
#pragma unroll
      for (int k = 0; k < kReduceChunkMax; ++k) sum += values[k];
    }
    scratch[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x * kReduceChunks < blockDim.x && base / kReduceChunks + threadIdx.x < count) {
      double total = 0.0;
#pragma unroll
      for (int c = 0; c < kReduceChunks; ++c) total += scratch[threadIdx.x * kReduceChunks + c];
      out[base / kReduceChunks + threadIdx.x] = total;
    }
    __syncthreads();
  }
}

// Particle state arrays are float32 (Newton's wp.vec3) or float64.
__device__ __forceinline__ double state_load(const void* p, int f64, int k) {
  return f64 ? static_cast<const double*>(p)[k] : static_cast<double>(static_cast<const float*>(p)[k]);
}
__device__ __forceinline__ void state_store(void* p, int f64, int k, double v) {
  if (f64) {
    static_cast<double*>(p)[k] = v;
  } else {
    static_cast<float*>(p)[k] = static_cast<float>(v);
  }
}
// Accumulate as the reference does: in the array's own precision.
__device__ __forceinline__ void state_add(void* p, int f64, int k, double v) {
  if (f64) {
    static_cast<double*>(p)[k] += v;
  } else {
    float* f = static_cast<float*>(p);
    f[k] = f[k] + static_cast<float>(v);
  }
}

template <typename T>
__device__ __forceinline__ V3<T> load3(const double* v, int i) {
  return v3<T>(static_cast<T>(v[3 * i]), static_cast<T>(v[3 * i + 1]), static_cast<T>(v[3 * i + 2]));
}
__device__ __forceinline__ V3<double> load3d(const double* v, int i) { return v3<double>(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }
__device__ __forceinline__ void store3(double* v, int i, V3<double> a) {
  v[3 * i] = a.x;
  v[3 * i + 1] = a.y;
  v[3 * i + 2] = a.z;
}

// One sparse product (S or S^T) split into per-block row ranges.
struct SpmvPlan {
  const int* off;       // CSR row offsets (global)
  const int* col;       // CSR columns
  const double* val64;  // CSR values (float64)
  const float* val32;   // CSR values (float32 copy, fp32+refine)
  const int* part;      // [blocks+1] row range of each block, balanced by nnz
  const int* rowlist;   // rows of each block's range: short rows first (one thread each), then long rows (one warp each)
  const int* nshort;    // [blocks] number of short rows of each block
  int smem_offset;      // byte offset of this product's slice in dynamic shared memory (resident plans)
  int max_nnz;          // largest per-block nnz (slice layout size)
  int max_rows;         // largest per-block row count
  // Streaming layout for plans that are not resident: every row padded to a
  // multiple of four entries (zero values), so a lane moves four entries per
  // 16-byte load of columns and of values. Row r covers groups [off4[r], off4[r+1]).
  const int* off4;      // [rows + 1]
  const int4* col4;     // [groups]
  const void* val4;     // [groups][4] values in the factor precision
  // Subset staging (resident plans whose vector is staged): block b stages
  // only the vector entries stage_cols[stage_off[b] .. stage_off[b+1]) and its
  // resident slice holds columns renumbered into that list (col_local).
  // nullptr: the whole vector is staged and the slice keeps global columns.
  const int* stage_off;
  const int* stage_cols;
  const int* col_local;
};

// Shared-memory layout of one resident slice: values, columns, relative row
// offsets, row list; every section 16-byte aligned.
__host__ __device__ __forceinline__ int align16(int bytes) { return (bytes + 15) & ~15; }
__host__ __device__ __forceinline__ int slice_bytes(int max_nnz, int max_rows, int value_bytes) {
  return align16(max_nnz * value_bytes) + align16(max_nnz * 4) + align16((max_rows + 1) * 4) + align16(max_rows * 4);
}

// The blocks that solve one instance: the whole grid in the plain launch, or
// one block per instance in the batched launch (then every barrier is a
// __syncthreads and the serial sections run in that block).
struct Team {
  int rank;
  int size;
};

// A frictional boundary of the step (the reference's FrictionalContact):
// registered vertices, boundary description, the factor's panel and the
// per-step and per-iteration contact state. count == 0 disables it.
struct FrictionArgs {
  int count;              // registered vertices K
  int kind;               // 0 planar, 1 spherical, 2 mesh
  const double* params;   // [4] plane (n, offset) or sphere (center, radius); device memory, editable
  const int* nodes;       // [K] particle of each contact
  double friction;        // Coulomb coefficient
  double restitution;     // normal restitution coefficient
  const int* faces;       // mesh: [F][3], faces_left then faces_right
  int face_count, left_count, split;
  double radius;          // mesh contact radius
  const double* panel;    // [n][K] A^{-1} e_nodes[j]
  const double* block;    // [K][K] panel rows of the registered vertices
  double* normal;         // [K][3] frames frozen at the step start
  double* tangent1;
  double* tangent2;
  double* delassus;       // [K][K]
  double* regularization; // [K]
  int* candidate;         // [K] mesh pre-filter (1 for planar and spherical)
  double* multiplier;     // [K] normal multipliers, warm start across steps
  double* lambda_t;       // [K][2] tangential multipliers
  double* omega;          // [K] per-iteration Fischer-Burmeister scalars
  double* diagonal;
  double* residual;
  double* rhs;
  double* force;          // [K][3]
  double* response;       // [K][3]
  int* order;             // [K] coupled candidates in candidate order
  int* slot;              // [K] position in order or -1
  int* active;            // [1] number of coupled candidates
  double* matrix;         // [K][K] coupled Newton block and its factor
  double* compact;        // [K]
  int* permutation;       // [K]
  double* work;           // [K]
  double* surface;        // [n][3] mesh restitution: iterate of the last contact update
};

// Everything one persistent launch needs. Passed by value as kernel argument.
struct StepArgs {
  // Mesh
  int n;         // vertices
  int ne;        // elements
  int corners;   // 4 (Tet4) or 8 (Hex8)
  int hex;       // 1 when every element has eight shared-gradient samples
  const int* indices;      // [ne][corners]
  const double* gradients; // Tet4 [ne][4][3]; Hex8 [8][8][3]
  const int* free_;        // [n]
  const int* inc_offsets;  // [n+1]
  const int* inc_entries;  // element*corners + corner, element-major order
  const double* plane_weight;  // [n] stiffness of the vertex-plane energy (0: none), or nullptr
  const double* extra_force;   // [n][3] state force added to the inertial target (mesh contact), or nullptr
  double plane[4];
  // Materials (per element; for Hex8 already multiplied by the sample volume)
  const double* wc;
  const double* wv;
  const double* wn;
  const double* wm;
  const double* mdir;      // [ne][3]
  double* mtarget;         // [ne]
  const float* activations;  // Tet4 contractions [ne] or nullptr
  int has_muscles;
  int material;
  double nh_mu, nh_lame, nh_penalty;
  // Factor (S: rows in elimination order; S^T: rows in particle order)
  const int* s_off;
  const int* s_col;
  const double* s_val;
  const float* s_val32;
  const int* st_off;
  const int* st_col;
  const double* st_val;
  const float* st_val32;
  const int* s_part;   // [blocks+1] S row partition
  const int* st_part;  // [blocks+1] S^T row partition (also owns particle rows)
  SpmvPlan plan_s;
  SpmvPlan plan_st;
  int resident;        // 1: factor slices live in dynamic shared memory for the launch
  int stage_vector;    // 1: the SpMV input vector is staged in shared memory
  int vector_smem_offset;
  int f32_vectors;     // 1: refinement products on float4 vectors with float32 sums (resident, staged)
  double* svd_u;       // warm-start singular vectors per element sample [E*S][9] (or nullptr)
  double* svd_v;
  const int* a_off;    // constant matrix A (refinement residual)
  const int* a_col;
  const double* a_val;
  int refine;          // 1: delta form x = x_prev + S^T S (b - A x_prev)
  // Step vectors [n][3] float64
  double* position;
  double* velocity;
  double* target;
  double* boundary;
  double* x;
  double* prev;
  double* proj;
  double* prev_proj;
  double* rhs;
  double* y;
  double* contrib;  // [ne][corners][3]
  // Anderson
  int window;
  double* hist_x;   // [(window+1)][3n]
  double* hist_g;
  // History of the block's own particle rows in dynamic shared memory: byte
  // offset of [window+1][hist_rows][3] x then g, or -1 to use hist_x/hist_g.
  int hist_smem_offset;
  int hist_rows;
  int* aa_state;    // count, start, count_used, start_used
  double* aa_gamma; // [kMaxWindow]
  int* aa_accept;
  double* partials; // [kPartialStride][blocks], slot-major
  unsigned long long* timers;  // optional phase timers (PD_PHASE_TIMERS builds)
  // Loop control
  int* iteration;
  int* active;
  int* status;
  int max_iterations;
  double abs_tol, rel_tol;
  GridBarrier* barrier;
  // Inputs and outputs of the step (float32, or float64 when state_f64)
  const void* q_in;
  const void* qd_in;
  const void* f_in;
  const void* dirichlet;
  void* q_out;
  void* qd_out;
  int state_f64;
  double* x_record;
  double dt, mass, inertia;
  double gravity[3];
  int integrate_pinned;
  FrictionArgs fc;
};

}  // namespace pdb200
