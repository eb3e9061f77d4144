// Batched projective-dynamics rollouts: many independent instances of
// uneven size advanced together, one CUDA graph per rollout.
//
// Per PD step the graph holds a prologue kernel, a WHILE node whose body is
// one local/global iteration of every instance that still iterates, and an
// epilogue kernel. The body kernels spread the work of all active instances
// over the whole GPU at their own occupancy (no grid barriers):
//   local     element samples -> corner contributions (solver.py:582-659 loop body, kernels.py:222-272, hex.py:122-169)
//   gather    particles: projection sum, right-hand side (refinement residual) in labels (kernels.py:75-91)
//   s         y = S b over the run-format rows of S                         (sparse.py:209-227)
//   st        x = S^T y (+ x_prev when refining), Dirichlet values          (sparse.py:341-348, kernels.py:287-291)
//   anderson  one block per instance: history push, incremental Gram, least squares, mixing, dual convergence gate
//             (anderson.py:306-503, kernels.py:354-401); the last block sets the WHILE condition
// The Anderson update and the convergence decision are the single-instance
// path's (aa_solve, the dual gate with k > 0); only the summation order of the
// reductions differs, so both paths agree to rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "pd_batch.cuh"
#include "pd_forward.cuh"
#include "pd_kernels.h"
#include "runs.h"
#include "solver_state.h"

namespace pdb200 {

constexpr int kShortRun = 32;          // rows with at most this many entries: one thread each
constexpr int kGramStride = kMaxWindow + 1;

struct Gravity {
  double g[3];
};

template <typename T>
__device__ __forceinline__ T warp_sum_t(T v) {
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) v += __shfl_xor_sync(0xffffffffu, v, offset);
  return v;
}

// Deterministic block sums of `count` values per thread (count uniform over
// the block, at most N). Results in out[0..count) (shared) for every thread.
template <int N>
__device__ __forceinline__ void block_sum_many(double (&v)[N], int count, double* scratch /* [kWarps * N] */,
                                               double* out /* [N] */) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k)
    if (k < count) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k)
      if (k < count) scratch[warp * N + k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < count) {
    double total = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) total += scratch[w * N + threadIdx.x];
    out[threadIdx.x] = total;
  }
  __syncthreads();
}

__device__ __forceinline__ const void* state_at(const void* base, int f64, long long offset) {
  return f64 ? static_cast<const void*>(static_cast<const double*>(base) + offset)
             : static_cast<const void*>(static_cast<const float*>(base) + offset);
}
__device__ __forceinline__ void* state_at(void* base, int f64, long long offset) {
  return f64 ? static_cast<void*>(static_cast<double*>(base) + offset) : static_cast<void*>(static_cast<float*>(base) + offset);
}

__device__ __forceinline__ bool instance_active(const BatchInstance& a) {
  return *reinterpret_cast<const volatile int*>(a.active) != 0;
}

// Task index of the t-th listed task of `kind` (t < listed total).
__device__ __forceinline__ int schedule_task(const ScheduleView& sch, int kind, int n_active, int t) {
  const int* prefix = sch.prefix + kind * (sch.count + 1);
  int lo = 0, hi = n_active;  // prefix[lo] <= t < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= t) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  const int inst = sch.active[lo];
  return sch.task_begin[kind * (sch.count + 1) + inst] + (t - prefix[lo]);
}

__device__ __forceinline__ int schedule_total(const ScheduleView& sch, int kind, int n_active) {
  return sch.prefix[kind * (sch.count + 1) + n_active];
}

// Exclusive block-wide prefix sum of one value per thread; `total` receives
// the sum. Uses the whole block.
__device__ __forceinline__ int block_exclusive_scan(int v, int* scratch /* [kWarps] */, int& total) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int inclusive = v;
#pragma unroll
  for (int offset = 1; offset < 32; offset <<= 1) {
    const int up = __shfl_up_sync(0xffffffffu, inclusive, offset);
    if (lane >= offset) inclusive += up;
  }
  __syncthreads();
  if (lane == 31) scratch[warp] = inclusive;
  __syncthreads();
  int before = 0;
  total = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const int value = scratch[w];
    if (w < warp) before += value;
    total += value;
  }
  return before + inclusive - v;
}

// Rebuilds the work list from the instances' active flags (one block).
__device__ void build_schedule(const BatchInstance* insts, const ScheduleView& sch) {
  __shared__ int s_scan[kWarps];
  int base_active = 0;
  int base_tasks[kTaskKinds] = {0, 0, 0, 0};
  for (int chunk = 0; chunk < sch.count; chunk += blockDim.x) {
    const int i = chunk + threadIdx.x;
    const int flag = i < sch.count ? *reinterpret_cast<const volatile int*>(insts[i].active) : 0;
    int total = 0;
    const int position = base_active + block_exclusive_scan(flag, s_scan, total);
    if (flag) sch.active[position] = i;
    const int listed = base_active;
    base_active += total;
#pragma unroll
    for (int kind = 0; kind < kTaskKinds; ++kind) {
      const int* begin = sch.task_begin + kind * (sch.count + 1);
      const int tasks = flag ? begin[i + 1] - begin[i] : 0;
      int kind_total = 0;
      const int offset = block_exclusive_scan(tasks, s_scan, kind_total);
      if (flag) sch.prefix[kind * (sch.count + 1) + position] = base_tasks[kind] + offset;
      base_tasks[kind] += kind_total;
    }
    (void)listed;
  }
  if (threadIdx.x == 0) {
    *sch.n_active = base_active;
#pragma unroll
    for (int kind = 0; kind < kTaskKinds; ++kind) sch.prefix[kind * (sch.count + 1) + base_active] = base_tasks[kind];
  }
}

// ---- Start of a PD step of one instance by one block: begin_step
// (kernels.py:155-190), explicit_boundary (:199-207), begin_solve and the
// Anderson reset.
__device__ void begin_step(const BatchInstance& a, const BatchStepIo& io, double dt, const Gravity& gravity) {
  const int f64 = a.state_f64;
  const long long offset = 3 * a.particle_offset;
  const void* q_in = state_at(io.q_in, f64, offset);
  const void* qd_in = state_at(io.qd_in, f64, offset);
  const void* f_in = state_at(io.f_in, f64, offset);
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) {
    const V3<double> start = v3<double>(state_load(q_in, f64, 3 * i), state_load(q_in, f64, 3 * i + 1),
                                        state_load(q_in, f64, 3 * i + 2));
    const V3<double> velocity = v3<double>(state_load(qd_in, f64, 3 * i), state_load(qd_in, f64, 3 * i + 1),
                                           state_load(qd_in, f64, 3 * i + 2));
    store3(a.position, i, start);
    store3(a.velocity, i, velocity);
    V3<double> target;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double acceleration = state_load(f_in, f64, 3 * i + c) / a.mass + gravity.g[c];
      target[c] = start[c] + dt * velocity[c] + dt * dt * acceleration;
    }
    store3(a.target, i, target);
    V3<double> boundary = v3<double>(0.0, 0.0, 0.0);
    if (a.free_[i] == 0) {
      boundary = start;
      if (a.integrate_pinned) boundary = boundary + dt * velocity;
    }
    store3(a.boundary, i, boundary);
    store3(a.x, i, start);
    store3(a.prev, i, start);
    store3(a.proj, i, v3<double>(0.0, 0.0, 0.0));
    store3(a.prev_proj, i, v3<double>(0.0, 0.0, 0.0));
  }
  if (threadIdx.x == 0) {
    a.aa_state[0] = a.aa_state[1] = a.aa_state[2] = a.aa_state[3] = 0;
    *a.iteration = 0;
    *a.active = 1;
  }
}

// ---- End of a PD step: write_state (kernels.py:404-414) and the step record.
__device__ void end_step(const BatchInstance& a, const BatchStepIo& io, double dt) {
  const int f64 = a.state_f64;
  const long long offset = 3 * a.particle_offset;
  void* q_out = state_at(io.q_out, f64, offset);
  void* qd_out = state_at(io.qd_out, f64, offset);
  double* record = io.x_record != nullptr ? io.x_record + offset : nullptr;
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double value = a.x[3 * i + c];
      state_store(q_out, f64, 3 * i + c, value);
      state_store(qd_out, f64, 3 * i + c, (value - a.position[3 * i + c]) / dt);
      if (record != nullptr) record[3 * i + c] = value;
    }
  }
}

// Step 0 of every instance (one block each) and the loop control reset.
__global__ void __launch_bounds__(kBlock) batch_prologue_kernel(const BatchInstance* insts, const BatchStepIo* io,
                                                                double dt, Gravity gravity, BatchControl* control) {
  const BatchInstance& a = insts[blockIdx.x];
  begin_step(a, io[0], dt, gravity);
  if (threadIdx.x == 0) {
    *a.step = 0;
    if (blockIdx.x == 0) {
      control->arrived = 0;
      control->active = 0;
      control->passes = 0;
    }
  }
}

// Work list of the first pass (every instance).
__global__ void __launch_bounds__(kBlock) batch_schedule_kernel(const BatchInstance* insts, ScheduleView sch) {
  build_schedule(insts, sch);
}

// ---- Local step over element tasks of active instances.
template <typename TL>
__global__ void __launch_bounds__(kBlock) batch_local_kernel(const BatchInstance* insts, const RangeTask* tasks,
                                                             ScheduleView sch) {
  __shared__ double s_grad[8 * 8 * 3];
  const int n_active = *sch.n_active;
  const int total = schedule_total(sch, kTaskLocal, n_active);
  for (int listed = blockIdx.x; listed < total; listed += gridDim.x) {
    const RangeTask t = tasks[schedule_task(sch, kTaskLocal, n_active, listed)];
    const BatchInstance& a = insts[t.inst];
    const bool warm = *a.iteration > 0;
    TL* su = static_cast<TL*>(a.svd_u);
    TL* sv = static_cast<TL*>(a.svd_v);
    if (a.hex) {
      for (int k = threadIdx.x; k < 8 * 8 * 3; k += blockDim.x) s_grad[k] = a.gradients[k];
      __syncthreads();
      const int group = (threadIdx.x & 31) >> 3;
      const int warp = threadIdx.x >> 5;
      for (int base = t.begin + warp * 4; base < t.end; base += kWarps * 4) {
        const int e = base + group;
        hex_cell<TL>(a, s_grad, e < t.end ? e : a.ne, warm, su, sv);
      }
    } else {
      for (int e = t.begin + threadIdx.x; e < t.end; e += blockDim.x) tet_element<TL>(a, e, warm, su, sv);
    }
    __syncthreads();
  }
}

// ---- Gather, vertex-plane energies and the right-hand side in labels. Four
// lanes per particle, fixed shuffle tree (the single-instance P2).
template <typename TV>
__device__ __forceinline__ void gather_task(const BatchInstance* insts, const RangeTask t) {
  const BatchInstance& a = insts[t.inst];
  TV* rhs = static_cast<TV*>(a.rhs);
  const int sub = threadIdx.x & 3;
  const int lane_group = (threadIdx.x & 31) >> 2;
  for (int base = t.begin + (threadIdx.x >> 5) * 8; base < t.end; base += kWarps * 8) {
    const int i = base + lane_group;
    const bool valid = i < t.end;
    double px = 0.0, py = 0.0, pz = 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0;
    if (valid) {
      const int k0 = a.inc_offsets[i], k1 = a.inc_offsets[i + 1];
#pragma unroll 4
      for (int k = k0 + sub; k < k1; k += 4) {
        const double* c = a.contrib + 3 * a.inc_entries[k];
        px += c[0];
        py += c[1];
        pz += c[2];
      }
      if (a.refine) {
        for (int k = a.a_off[i] + sub; k < a.a_off[i + 1]; k += 4) {
          const double v = a.a_val[k];
          const int j = a.a_col[k];
          ax += v * a.prev[3 * j];
          ay += v * a.prev[3 * j + 1];
          az += v * a.prev[3 * j + 2];
        }
      }
    }
#pragma unroll
    for (int mask = 1; mask < 4; mask <<= 1) {
      px += __shfl_xor_sync(0xffffffffu, px, mask);
      py += __shfl_xor_sync(0xffffffffu, py, mask);
      pz += __shfl_xor_sync(0xffffffffu, pz, mask);
      ax += __shfl_xor_sync(0xffffffffu, ax, mask);
      ay += __shfl_xor_sync(0xffffffffu, ay, mask);
      az += __shfl_xor_sync(0xffffffffu, az, mask);
    }
    if (valid && sub == 0) {
      const double w = a.plane_weight[i];
      if (w != 0.0) {
        const double nx = a.plane[0], ny = a.plane[1], nz = a.plane[2];
        const double xx = a.x[3 * i], xy = a.x[3 * i + 1], xz = a.x[3 * i + 2];
        const double d = nx * xx + ny * xy + nz * xz + a.plane[3];
        const double m = fmin(0.0, d);
        px += w * ((xx - m * nx) - a.boundary[3 * i]);
        py += w * ((xy - m * ny) - a.boundary[3 * i + 1]);
        pz += w * ((xz - m * nz) - a.boundary[3 * i + 2]);
      }
      a.proj[3 * i] = px;
      a.proj[3 * i + 1] = py;
      a.proj[3 * i + 2] = pz;
      const int u = a.label_of[i];
      rhs[3 * u] = static_cast<TV>(a.inertia * a.target[3 * i] + px - ax);
      rhs[3 * u + 1] = static_cast<TV>(a.inertia * a.target[3 * i + 1] + py - ay);
      rhs[3 * u + 2] = static_cast<TV>(a.inertia * a.target[3 * i + 2] + pz - az);
    }
  }
}

template <typename TV>
__global__ void __launch_bounds__(kBlock) batch_gather_kernel(const BatchInstance* insts, const RangeTask* tasks,
                                                              ScheduleView sch) {
  const int n_active = *sch.n_active;
  const int total = schedule_total(sch, kTaskGather, n_active);
  for (int listed = blockIdx.x; listed < total; listed += gridDim.x) {
    gather_task<TV>(insts, tasks[schedule_task(sch, kTaskGather, n_active, listed)]);
  }
}

// Rows [r0, r1) of a run matrix times a vector window staged in shared memory
// (win[3 * (c - c0) + component]). Rows with at most kShortRun entries are
// summed by one thread, longer rows by one warp (lane-strided, fixed shuffle
// tree): every row always by the same unit in the same order.
template <typename TV, typename Emit>
__device__ __forceinline__ void run_rows(const RunView& m, const TV* win, int c0, int r0, int r1, Emit emit) {
  const TV* values = static_cast<const TV*>(m.values);
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const int k0 = m.row_runs[r], k1 = m.row_runs[r + 1];
    if (m.run_off[k1] - m.run_off[k0] > kShortRun) continue;
    TV sx = TV(0), sy = TV(0), sz = TV(0);
    for (int k = k0; k < k1; ++k) {
      const int e0 = m.run_off[k], e1 = m.run_off[k + 1];
      const int shift = m.run_col[k] - c0 - e0;
      for (int j = e0; j < e1; ++j) {
        const TV v = values[j];
        const TV* w = win + 3 * (shift + j);
        sx += v * w[0];
        sy += v * w[1];
        sz += v * w[2];
      }
    }
    emit(r, sx, sy, sz);
  }
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int r = r0 + warp; r < r1; r += kWarps) {
    const int k0 = m.row_runs[r], k1 = m.row_runs[r + 1];
    if (m.run_off[k1] - m.run_off[k0] <= kShortRun) continue;
    TV sx = TV(0), sy = TV(0), sz = TV(0);
    for (int k = k0; k < k1; ++k) {
      const int e0 = m.run_off[k], e1 = m.run_off[k + 1];
      const int shift = m.run_col[k] - c0 - e0;
#pragma unroll 4
      for (int j = e0 + lane; j < e1; j += 32) {
        const TV v = values[j];
        const TV* w = win + 3 * (shift + j);
        sx += v * w[0];
        sy += v * w[1];
        sz += v * w[2];
      }
    }
    sx = warp_sum_t(sx);
    sy = warp_sum_t(sy);
    sz = warp_sum_t(sz);
    if (lane == 0) emit(r, sx, sy, sz);
  }
}

template <typename TV>
__device__ __forceinline__ void stage_window(const TV* vec, int c0, int c1, TV* win) {
  const int count = 3 * (c1 - c0);
  const TV* src = vec + 3 * static_cast<size_t>(c0);
  for (int k = threadIdx.x; k < count; k += blockDim.x) win[k] = src[k];
  __syncthreads();
}

// ---- y = S b (labels).
template <typename TV>
__global__ void __launch_bounds__(kBlock) batch_s_kernel(const BatchInstance* insts, const RowTask* tasks,
                                                         ScheduleView sch) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  TV* win = reinterpret_cast<TV*>(dyn_smem);
  const int n_active = *sch.n_active;
  const int total = schedule_total(sch, kTaskS, n_active);
  for (int listed = blockIdx.x; listed < total; listed += gridDim.x) {
    const RowTask t = tasks[schedule_task(sch, kTaskS, n_active, listed)];
    const BatchInstance& a = insts[t.inst];
    stage_window(static_cast<const TV*>(a.rhs), t.c0, t.c1, win);
    TV* y = static_cast<TV*>(a.y);
    run_rows<TV>(a.s, win, t.c0, t.r0, t.r1, [&](int u, TV sx, TV sy, TV sz) {
      y[3 * u] = sx;
      y[3 * u + 1] = sy;
      y[3 * u + 2] = sz;
    });
    __syncthreads();
  }
}

// ---- x = S^T y (+ x_prev when refining), Dirichlet values, particle order.
template <typename TV>
__global__ void __launch_bounds__(kBlock) batch_st_kernel(const BatchInstance* insts, const RowTask* tasks,
                                                          ScheduleView sch) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  TV* win = reinterpret_cast<TV*>(dyn_smem);
  const int n_active = *sch.n_active;
  const int total = schedule_total(sch, kTaskSt, n_active);
  for (int listed = blockIdx.x; listed < total; listed += gridDim.x) {
    const RowTask t = tasks[schedule_task(sch, kTaskSt, n_active, listed)];
    const BatchInstance& a = insts[t.inst];
    stage_window(static_cast<const TV*>(a.y), t.c0, t.c1, win);
    run_rows<TV>(a.st, win, t.c0, t.r0, t.r1, [&](int v, TV sx, TV sy, TV sz) {
      const int p = a.particle_of[v];
      V3<double> value = v3<double>(static_cast<double>(sx), static_cast<double>(sy), static_cast<double>(sz));
      if (a.refine) value = value + load3d(a.prev, p);
      if (a.free_[p] == 0) value = load3d(a.boundary, p);
      store3(a.x, p, value);
    });
    __syncthreads();
  }
}

// ---- Anderson acceleration and the convergence gate, one block per instance.
// The Gram entries dG_a . dG_b of the differences that stay in the window are
// kept per ring-slot pair; each iteration computes only the entries of the
// newest difference and the right-hand side dG_a . g, which reads every
// history vector once. The last block to finish sets the WHILE condition to
// whether any instance still iterates.
__global__ void __launch_bounds__(kBlock) batch_anderson_kernel(const BatchInstance* insts, BatchControl* control,
                                                                cudaGraphConditionalHandle handle,
                                                                unsigned max_passes, const BatchStepIo* io, int steps,
                                                                double dt, Gravity gravity, int* iteration_log,
                                                                ScheduleView sch) {
  __shared__ double s_scratch[kWarps * 2 * kMaxWindow];
  __shared__ double s_out[2 * kMaxWindow];
  __shared__ double s_gamma[kMaxWindow];
  __shared__ int s_ctl[4];
  const BatchInstance& a = insts[blockIdx.x];
  int still = 0;
  if (instance_active(a)) {
    const int n = a.n;
    const int window = a.window;
    const int capacity = window + 1;
    const size_t stride = static_cast<size_t>(3) * n;
    const int count = window > 0 ? a.aa_state[0] : 0;
    const int start = window > 0 ? a.aa_state[1] : 0;
    const int slot = window > 0 ? (start + count) % capacity : 0;
    // Pass 1: push (x_prev, G(x_prev) - x_prev), new Gram entries.
    double sums[2 * kMaxWindow];
#pragma unroll
    for (int k = 0; k < 2 * kMaxWindow; ++k) sums[k] = 0.0;
    if (window > 0) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const V3<double> xv = load3d(a.x, i);
        const V3<double> pv = load3d(a.prev, i);
        const V3<double> g = xv - pv;
        store3(a.hist_x + slot * stride, i, pv);
        store3(a.hist_g + slot * stride, i, g);
        if (count >= 1) {
          const V3<double> newest = g - load3d(a.hist_g + ((start + count - 1) % capacity) * stride, i);
          V3<double> low = load3d(a.hist_g + (start % capacity) * stride, i);
#pragma unroll
          for (int k = 0; k < kMaxWindow; ++k) {
            if (k < count) {
              const V3<double> high = k + 1 == count ? g : load3d(a.hist_g + ((start + k + 1) % capacity) * stride, i);
              const V3<double> d = high - low;
              sums[k] += dot(newest, d);
              sums[kMaxWindow + k] += dot(d, g);
              low = high;
            }
          }
        }
      }
      // Reduce the count entries of each half in one pass.
      double packed[2 * kMaxWindow];
#pragma unroll
      for (int k = 0; k < kMaxWindow; ++k) {
        packed[k] = sums[k];
        packed[kMaxWindow + k] = sums[kMaxWindow + k];
      }
      // Entries [0, count) and [kMaxWindow, kMaxWindow + count) are live; reduce all 2*kMaxWindow.
      block_sum_many<2 * kMaxWindow>(packed, count >= 1 ? 2 * kMaxWindow : 0, s_scratch, s_out);
      if (threadIdx.x == 0) {
        double* gram = a.gram;
        double reduced[kMaxWindow * (kMaxWindow + 1) / 2 + kMaxWindow];
        if (count >= 1) {
          const int newest_slot = (start + count - 1) % capacity;
          for (int k = 0; k < count; ++k) {
            const int ks = (start + k) % capacity;
            gram[newest_slot * kGramStride + ks] = s_out[k];
            gram[ks * kGramStride + newest_slot] = s_out[k];
          }
          int entry = 0;
          for (int i = 0; i < count; ++i)
            for (int j = i; j < count; ++j)
              reduced[entry++] = gram[((start + i) % capacity) * kGramStride + (start + j) % capacity];
          for (int i = 0; i < count; ++i) reduced[entry++] = s_out[kMaxWindow + i];
        }
        int accept = 0;
        aa_solve(a.aa_state, s_gamma, &accept, reduced, window, s_scratch);
        s_ctl[0] = accept;
        s_ctl[1] = a.aa_state[2];
        s_ctl[2] = a.aa_state[3];
      }
      __syncthreads();
    } else if (threadIdx.x == 0) {
      s_ctl[0] = 0;
    }
    __syncthreads();
    const int accept = s_ctl[0];
    const int used_count = s_ctl[1];
    const int used_start = s_ctl[2];
    // Pass 2: mixing (anderson.py:478-503), Dirichlet values, gate norms.
    double norms[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      V3<double> value = load3d(a.x, i);
      if (accept) {
        const int top = (used_start + used_count) % capacity;
        value = load3d(a.hist_x + top * stride, i) + load3d(a.hist_g + top * stride, i);
        for (int k = 0; k < used_count; ++k) {
          const int low = (used_start + k) % capacity;
          const int high = (used_start + k + 1) % capacity;
          const V3<double> dx = load3d(a.hist_x + high * stride, i) - load3d(a.hist_x + low * stride, i);
          const V3<double> dg = load3d(a.hist_g + high * stride, i) - load3d(a.hist_g + low * stride, i);
          value = value - s_gamma[k] * (dx + dg);
        }
      }
      if (a.free_[i] == 0) value = load3d(a.boundary, i);
      store3(a.x, i, value);
      const V3<double> previous = load3d(a.prev, i);
      const V3<double> p = load3d(a.proj, i);
      const V3<double> pp = load3d(a.prev_proj, i);
      const V3<double> step = value - previous;
      const V3<double> change = p - pp;
      norms[0] += dot(step, step);
      norms[1] += dot(previous, previous);
      norms[2] += dot(change, change);
      norms[3] += dot(pp, pp);
      store3(a.prev, i, value);
      store3(a.prev_proj, i, p);
    }
    block_sum_many<4>(norms, 4, s_scratch, s_out);
    if (threadIdx.x == 0) {
      const double step_norm = sqrt(s_out[0]);
      const double previous_norm = sqrt(s_out[1]);
      const double change_norm = sqrt(s_out[2]);
      const double projection_norm = sqrt(s_out[3]);
      const int k = *a.iteration;
      *a.iteration = k + 1;
      int finished = 0;
      if (k > 0 && step_norm <= a.rel_tol * previous_norm + a.abs_tol &&
          change_norm <= a.rel_tol * projection_norm + a.abs_tol) {
        finished = 1;
      } else if (k + 1 >= a.max_iterations) {
        finished = 1;
        atomicOr(a.status, kStatusNotConverged);
      }
      s_ctl[3] = finished;
    }
    __syncthreads();
    still = 1;
    if (s_ctl[3]) {
      // This instance's step is done: write it out and start its next step
      // right away, independently of the other instances.
      const int step = *a.step;
      end_step(a, io[step], dt);
      if (threadIdx.x == 0 && iteration_log != nullptr) iteration_log[step * gridDim.x + blockIdx.x] = *a.iteration;
      __syncthreads();
      if (step + 1 < steps) {
        begin_step(a, io[step + 1], dt, gravity);
        if (threadIdx.x == 0) *a.step = step + 1;
      } else {
        still = 0;
        if (threadIdx.x == 0) *a.active = 0;
      }
    }
  }
  if (threadIdx.x == 0) {
    if (still) atomicAdd(&control->active, 1u);
    __threadfence();
    const unsigned done = atomicAdd(&control->arrived, 1u);
    s_ctl[0] = done == gridDim.x - 1;
  }
  __syncthreads();
  if (s_ctl[0]) {
    // Last block: every instance's flag is final; list the next pass's work.
    __threadfence();
    build_schedule(insts, sch);
    if (threadIdx.x == 0) {
      const unsigned active = atomicAdd(&control->active, 0u);
      const unsigned passes = control->passes + 1;
      control->passes = passes;
      control->arrived = 0;
      control->active = 0;
      control->last_active = passes < max_passes ? active : 0u;
      if (handle != 0) cudaGraphSetConditional(handle, (active > 0 && passes < max_passes) ? 1u : 0u);
    }
  }
}

}  // namespace pdb200

// ---------------------------------------------------------------------------
// Host side.

using pdb200::BatchControl;
using pdb200::BatchInstance;
using pdb200::BatchStepIo;
using pdb200::RangeTask;
using pdb200::RowTask;

namespace {

struct InstanceBuffers {
  DeviceBuffer s_row_runs, s_run_col, s_run_off, s_values;
  DeviceBuffer st_row_runs, st_run_col, st_run_off, st_values;
  DeviceBuffer label_of, particle_of, rhs, y, svd_u, svd_v, gram, aa_state;
};

struct GraphKey {
  int steps = -1;
  double dt = 0.0;
  double gravity[3] = {0, 0, 0};
  const void* q0 = nullptr;
  const void* qd0 = nullptr;
  const void* forces = nullptr;
  long long force_stride = 0;
  void* q_traj = nullptr;
  void* qd_traj = nullptr;
  double* x_record = nullptr;
  bool operator==(const GraphKey& o) const {
    return steps == o.steps && dt == o.dt && gravity[0] == o.gravity[0] && gravity[1] == o.gravity[1] &&
           gravity[2] == o.gravity[2] && q0 == o.q0 && qd0 == o.qd0 && forces == o.forces &&
           force_stride == o.force_stride && q_traj == o.q_traj && qd_traj == o.qd_traj && x_record == o.x_record;
  }
};

}  // namespace

struct PdBatch {
  int schedule = PD_BATCH_TEAMS;
  int device = 0;
  int count = 0;
  int precision = 0;
  int state_f64 = 0;
  std::vector<PdSolver*> solvers;
  std::vector<int64_t> particle_offsets, element_offsets;
  std::vector<std::unique_ptr<InstanceBuffers>> buffers;
  // Launch-plan buffers of every instance planned for its team: the batch owns
  // them, so a later batch over the same solvers cannot invalidate this one.
  std::vector<std::unique_ptr<TeamPlanBuffers>> team_plans;
  std::vector<uint64_t> generations;  // of every solver when the batch was created
  DeviceBuffer d_instances, d_local_tasks, d_gather_tasks, d_s_tasks, d_st_tasks, d_control, d_io, d_log;
  DeviceBuffer d_task_begin, d_n_active, d_active, d_prefix;
  int grid[pdb200::kTaskKinds] = {1, 1, 1, 1};
  int n_local = 0, n_gather = 0, n_s = 0, n_st = 0;
  size_t smem_s = 0, smem_st = 0;
  unsigned max_iterations = 0;
  int64_t value_count = 0, run_count = 0;
  std::vector<int> iterations_host;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  GraphKey key;
  // Teams schedule: per-instance team sizes and argument blocks, the queue.
  std::vector<int> team_size;
  // Adjoint lanes planned from measured adjoint durations (adj_lanes > 0), else the forward's.
  DeviceBuffer d_adj_lane_start, d_adj_lane_class, d_adj_class_begin, d_adj_class_order;
  int adj_lanes = 0, adj_team_blocks = 0;
  DeviceBuffer d_forward_args, d_adjoint_args, d_lane_start, d_lane_class, d_class_begin, d_class_order,
      d_particle_offset, d_element_offset, d_class_head, d_lane_slot, d_barriers, d_team_status, d_adjoint_log,
      d_timeline;
  int team_blocks = 0, lanes = 0, classes = 0, solo_class = -1;
  unsigned long long* timers = nullptr;  // phase timers of one instance (PD_PHASE_TIMERS builds)
  int timer_instance = -1;
  size_t team_smem = 0;
  cudaStream_t capture = nullptr;  // private stream the rollout graphs are captured on
  cudaGraphExec_t adjoint_exec = nullptr;
  GraphKey adjoint_key;
  ~PdBatch() {
    if (exec != nullptr) cudaGraphExecDestroy(exec);
    if (graph != nullptr) cudaGraphDestroy(graph);
    if (adjoint_exec != nullptr) cudaGraphExecDestroy(adjoint_exec);
    if (capture != nullptr) cudaStreamDestroy(capture);
  }
};

namespace {

// Per-row column span (first column, one past the last) of a run matrix.
void row_span(const pdb200::RunMatrix& m, int r, int& lo, int& hi) {
  lo = 1 << 30;
  hi = -1;
  for (int k = m.row_runs[r]; k < m.row_runs[r + 1]; ++k) {
    lo = std::min(lo, m.run_col[k]);
    hi = std::max(hi, m.run_col[k] + (m.run_off[k + 1] - m.run_off[k]));
  }
  if (hi < 0) lo = hi = 0;
}

// Row tasks of one matrix: consecutive rows until task_nnz entries or a
// window wider than max_cols columns.
int row_tasks(const pdb200::RunMatrix& m, int inst, int task_nnz, int max_cols, std::vector<RowTask>& out,
              size_t& widest) {
  const int rows = static_cast<int>(m.row_runs.size()) - 1;
  int r = 0;
  while (r < rows) {
    RowTask t{inst, r, r, 0, 0};
    int lo = 1 << 30, hi = 0;
    long long nnz = 0;
    while (r < rows) {
      int rlo, rhi;
      row_span(m, r, rlo, rhi);
      const int nlo = std::min(lo, rlo), nhi = std::max(hi, rhi);
      const long long rnnz = m.run_off[m.row_runs[r + 1]] - m.run_off[m.row_runs[r]];
      if (t.r1 > t.r0 && (nnz + rnnz > task_nnz || nhi - nlo > max_cols)) break;
      if (nhi - nlo > max_cols) {
        return pd_set_error(PD_ERR_UNSUPPORTED,
                            "an instance is too large for the batched path (factor row wider than shared memory)");
      }
      lo = nlo;
      hi = nhi;
      nnz += rnnz;
      ++r;
      t.r1 = r;
    }
    t.c0 = lo > hi ? 0 : lo;
    t.c1 = lo > hi ? 0 : hi;
    widest = std::max(widest, static_cast<size_t>(t.c1 - t.c0));
    out.push_back(t);
  }
  return PD_OK;
}

template <typename T>
cudaError_t upload_as(DeviceBuffer& buffer, const std::vector<double>& values) {
  std::vector<T> converted(values.begin(), values.end());
  return buffer.upload(converted);
}

// Local step precision: float only in PD_PRECISION_FP32; factor products in
// float whenever the precision is not PD_PRECISION_FP64.
const void* local_kernel(int precision) {
  return precision == PD_PRECISION_FP32 ? reinterpret_cast<const void*>(&pdb200::batch_local_kernel<float>)
                                        : reinterpret_cast<const void*>(&pdb200::batch_local_kernel<double>);
}
const void* gather_kernel(int precision) {
  return precision == PD_PRECISION_FP64 ? reinterpret_cast<const void*>(&pdb200::batch_gather_kernel<double>)
                                        : reinterpret_cast<const void*>(&pdb200::batch_gather_kernel<float>);
}
const void* s_kernel(int precision) {
  return precision == PD_PRECISION_FP64 ? reinterpret_cast<const void*>(&pdb200::batch_s_kernel<double>)
                                        : reinterpret_cast<const void*>(&pdb200::batch_s_kernel<float>);
}
const void* st_kernel(int precision) {
  return precision == PD_PRECISION_FP64 ? reinterpret_cast<const void*>(&pdb200::batch_st_kernel<double>)
                                        : reinterpret_cast<const void*>(&pdb200::batch_st_kernel<float>);
}

cudaError_t add_kernel(cudaGraphNode_t* node, cudaGraph_t graph, const cudaGraphNode_t* deps, size_t ndeps,
                       const void* func, int grid, size_t smem, void** args) {
  cudaKernelNodeParams p{};
  p.func = const_cast<void*>(func);
  p.gridDim = dim3(static_cast<unsigned>(grid));
  p.blockDim = dim3(pdb200::kBlock);
  p.sharedMemBytes = static_cast<unsigned>(smem);
  p.kernelParams = args;
  p.extra = nullptr;
  return cudaGraphAddKernelNode(node, graph, deps, ndeps, &p);
}

}  // namespace

// The phases schedule: run-format factors, work-list tasks and the
// instance table of the per-phase kernels.
int create_phases(PdBatch* batch, const PdBatchOptions& opts) {
  const int count = batch->count;
  const bool fp64 = batch->precision == PD_PRECISION_FP64;
  const size_t tv = fp64 ? sizeof(double) : sizeof(float);
  const size_t tl = batch->precision == PD_PRECISION_FP32 ? sizeof(float) : sizeof(double);
  int smem_optin = 0;
  PD_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, batch->device));
  const int max_cols = static_cast<int>((static_cast<size_t>(smem_optin) - 1024) / (3 * tv));
  std::vector<BatchInstance> instances(count);
  std::vector<RangeTask> local_tasks, gather_tasks;
  std::vector<RowTask> s_tasks, st_tasks;
  std::vector<int> task_begin(static_cast<size_t>(pdb200::kTaskKinds) * (count + 1), 0);
  size_t widest_s = 0, widest_st = 0;
  int64_t particles = 0, elements = 0;
  int max_iterations = 0;
  for (int i = 0; i < count; ++i) {
    PdSolver* s = batch->solvers[i];
    auto buffers = std::make_unique<InstanceBuffers>();
    const pdb200::RunFactor runs = pdb200::build_run_factor(s->factor, opts.run_gap);
    PD_CUDA(buffers->s_row_runs.upload(runs.s.row_runs));
    PD_CUDA(buffers->s_run_col.upload(runs.s.run_col));
    PD_CUDA(buffers->s_run_off.upload(runs.s.run_off));
    PD_CUDA(buffers->st_row_runs.upload(runs.st.row_runs));
    PD_CUDA(buffers->st_run_col.upload(runs.st.run_col));
    PD_CUDA(buffers->st_run_off.upload(runs.st.run_off));
    if (fp64) {
      PD_CUDA(upload_as<double>(buffers->s_values, runs.s.values));
      PD_CUDA(upload_as<double>(buffers->st_values, runs.st.values));
    } else {
      PD_CUDA(upload_as<float>(buffers->s_values, runs.s.values));
      PD_CUDA(upload_as<float>(buffers->st_values, runs.st.values));
    }
    batch->value_count += static_cast<int64_t>(runs.s.values.size() + runs.st.values.size());
    batch->run_count += static_cast<int64_t>(runs.s.run_col.size() + runs.st.run_col.size());
    PD_CUDA(buffers->label_of.upload(runs.label_of));
    PD_CUDA(buffers->particle_of.upload(runs.particle_of));
    PD_CUDA(buffers->rhs.allocate(static_cast<size_t>(3) * s->n * tv));
    PD_CUDA(buffers->y.allocate(static_cast<size_t>(3) * s->n * tv));
    const size_t samples = static_cast<size_t>(s->ne) * (s->hex ? 8 : 1);
    if (opts.svd_warm_start) {
      PD_CUDA(buffers->svd_u.allocate(samples * 9 * tl));
      PD_CUDA(buffers->svd_v.allocate(samples * 9 * tl));
    }
    PD_CUDA(buffers->gram.allocate(static_cast<size_t>(pdb200::kGramStride) * pdb200::kGramStride * sizeof(double)));
    PD_CUDA(buffers->aa_state.allocate(8 * sizeof(int)));
    BatchInstance& a = instances[i];
    a.n = s->n;
    a.ne = s->ne;
    a.corners = s->corners;
    a.hex = s->hex;
    a.indices = s->d_indices.as<int>();
    a.gradients = s->d_gradients.as<double>();
    a.free_ = s->d_free.as<int>();
    a.inc_offsets = s->d_inc_offsets.as<int>();
    a.inc_entries = s->d_inc_entries.as<int>();
    a.plane_weight = s->d_plane_weight.as<double>();
    for (int c = 0; c < 4; ++c) a.plane[c] = s->plane[c];
    a.wc = s->d_wc.as<double>();
    a.wv = s->d_wv.as<double>();
    a.wn = s->d_wn.as<double>();
    a.wm = s->d_wm.as<double>();
    a.mdir = s->d_mdir.as<double>();
    a.mtarget = s->d_mtarget.as<double>();
    a.has_muscles = s->has_muscles ? 1 : 0;
    a.material = s->options.material;
    a.nh_mu = s->nh_mu;
    a.nh_lame = s->nh_lame;
    a.nh_penalty = s->nh_penalty;
    a.status = s->d_status.as<int>();
    a.s = {buffers->s_row_runs.as<int>(), buffers->s_run_col.as<int>(), buffers->s_run_off.as<int>(),
           buffers->s_values.ptr};
    a.st = {buffers->st_row_runs.as<int>(), buffers->st_run_col.as<int>(), buffers->st_run_off.as<int>(),
            buffers->st_values.ptr};
    a.label_of = buffers->label_of.as<int>();
    a.particle_of = buffers->particle_of.as<int>();
    a.a_off = s->d_a_off.as<int>();
    a.a_col = s->d_a_col.as<int>();
    a.a_val = s->d_a_val.as<double>();
    a.refine = fp64 ? 0 : 1;
    a.svd_u = opts.svd_warm_start ? buffers->svd_u.ptr : nullptr;
    a.svd_v = opts.svd_warm_start ? buffers->svd_v.ptr : nullptr;
    a.position = s->d_position.as<double>();
    a.velocity = s->d_velocity.as<double>();
    a.target = s->d_target.as<double>();
    a.boundary = s->d_boundary.as<double>();
    a.x = s->d_x.as<double>();
    a.prev = s->d_prev.as<double>();
    a.proj = s->d_proj.as<double>();
    a.prev_proj = s->d_prev_proj.as<double>();
    a.contrib = s->d_contrib.as<double>();
    a.rhs = buffers->rhs.ptr;
    a.y = buffers->y.ptr;
    a.window = s->options.anderson_window;
    a.hist_x = s->d_hist_x.as<double>();
    a.hist_g = s->d_hist_g.as<double>();
    a.gram = buffers->gram.as<double>();
    a.aa_state = buffers->aa_state.as<int>();
    a.step = buffers->aa_state.as<int>() + 4;
    a.iteration = s->d_iteration.as<int>();
    a.active = s->d_active.as<int>();
    a.max_iterations = s->options.max_iterations;
    a.abs_tol = s->options.abs_tol;
    a.rel_tol = s->options.rel_tol;
    a.mass = s->mass;
    a.inertia = s->inertia;
    a.integrate_pinned = s->options.integrate_pinned_velocities;
    a.state_f64 = s->options.state_precision;
    a.particle_offset = particles;
    a.element_offset = elements;
    max_iterations = std::max(max_iterations, s->options.max_iterations);
    // Tasks (contiguous per instance).
    task_begin[0 * (count + 1) + i] = static_cast<int>(local_tasks.size());
    task_begin[1 * (count + 1) + i] = static_cast<int>(gather_tasks.size());
    task_begin[2 * (count + 1) + i] = static_cast<int>(s_tasks.size());
    task_begin[3 * (count + 1) + i] = static_cast<int>(st_tasks.size());
    const int chunk = s->hex ? opts.local_cells : pdb200::kBlock;
    for (int e = 0; e < s->ne; e += chunk) local_tasks.push_back({i, e, std::min(s->ne, e + chunk)});
    for (int p = 0; p < s->n; p += pdb200::kBlock) gather_tasks.push_back({i, p, std::min(s->n, p + pdb200::kBlock)});
    if (int status = row_tasks(runs.s, i, opts.task_nnz, max_cols, s_tasks, widest_s)) return status;
    if (int status = row_tasks(runs.st, i, opts.task_nnz, max_cols, st_tasks, widest_st)) return status;
    particles += s->n;
    elements += s->ne;
    batch->buffers.push_back(std::move(buffers));
  }
  PD_CUDA(batch->d_instances.upload(instances));
  PD_CUDA(batch->d_local_tasks.upload(local_tasks));
  PD_CUDA(batch->d_gather_tasks.upload(gather_tasks));
  PD_CUDA(batch->d_s_tasks.upload(s_tasks));
  PD_CUDA(batch->d_st_tasks.upload(st_tasks));
  PD_CUDA(batch->d_control.allocate(sizeof(BatchControl)));
  task_begin[0 * (count + 1) + count] = static_cast<int>(local_tasks.size());
  task_begin[1 * (count + 1) + count] = static_cast<int>(gather_tasks.size());
  task_begin[2 * (count + 1) + count] = static_cast<int>(s_tasks.size());
  task_begin[3 * (count + 1) + count] = static_cast<int>(st_tasks.size());
  PD_CUDA(batch->d_task_begin.upload(task_begin));
  PD_CUDA(batch->d_n_active.allocate(sizeof(int)));
  PD_CUDA(batch->d_active.allocate(static_cast<size_t>(count) * sizeof(int)));
  PD_CUDA(batch->d_prefix.allocate(static_cast<size_t>(pdb200::kTaskKinds) * (count + 1) * sizeof(int)));
  batch->n_local = static_cast<int>(local_tasks.size());
  batch->n_gather = static_cast<int>(gather_tasks.size());
  batch->n_s = static_cast<int>(s_tasks.size());
  batch->n_st = static_cast<int>(st_tasks.size());
  batch->smem_s = std::max<size_t>(16, widest_s * 3 * tv);
  batch->smem_st = std::max<size_t>(16, widest_st * 3 * tv);
  batch->max_iterations = static_cast<unsigned>(max_iterations);
  // The attribute belongs to the kernel, shared by every batch on the device:
  // allow the device maximum rather than this batch's need.
  for (const void* kernel : {s_kernel(batch->precision), st_kernel(batch->precision)}) {
    cudaFuncAttributes attributes{};
    PD_CUDA(cudaFuncGetAttributes(&attributes, kernel));
    PD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem_optin - static_cast<int>(attributes.sharedSizeBytes)));
  }
  // One resident wave per work-list kernel; its blocks stride over the listed tasks.
  {
    int sms = 0;
    PD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, batch->device));
    const void* kernels[pdb200::kTaskKinds] = {local_kernel(batch->precision), gather_kernel(batch->precision),
                                               s_kernel(batch->precision), st_kernel(batch->precision)};
    const size_t smem[pdb200::kTaskKinds] = {0, 0, batch->smem_s, batch->smem_st};
    const int tasks[pdb200::kTaskKinds] = {batch->n_local, batch->n_gather, batch->n_s, batch->n_st};
    for (int k = 0; k < pdb200::kTaskKinds; ++k) {
      int per_sm = 0;
      PD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernels[k], pdb200::kBlock, smem[k]));
      batch->grid[k] = std::max(1, std::min(tasks[k], std::max(1, per_sm) * sms));
    }
  }
  return PD_OK;
}

// The teams schedule. Each instance wants a team of about
// max(nnz(S) / team_nnz, samples / team_samples) blocks, rounded to a power of
// two: its size class. The grid is cut into lanes of each class's size, with
// a share of blocks per class proportional to the class's work (factor
// entries plus element samples); every solver is planned for its class's
// team size, and the queues list each class's instances by decreasing work.
// Completion time of instances with the given durations on `lanes` lanes,
// longest first, each to the lane that frees first.
static double lpt_completion(const std::vector<double>& durations, int lanes) {
  std::vector<double> load(std::max(lanes, 1), 0.0);
  for (double d : durations) *std::min_element(load.begin(), load.end()) += d;
  return *std::max_element(load.begin(), load.end());
}

// Smallest makespan T for which every size class, given just enough lanes
// that its members (longest first) finish by T, fits the grid; `lanes_out`
// receives those lane counts in ascending class order.
template <typename Estimate>
static double plan_makespan(const std::vector<int>& team_size, Estimate estimate, int grid_cap,
                            std::vector<int>* lanes_out) {
  std::vector<int> sizes(team_size);
  std::sort(sizes.begin(), sizes.end());
  sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
  const int classes = static_cast<int>(sizes.size());
  std::vector<std::vector<double>> durations(classes);
  double low = 0.0, high = 0.0;
  for (size_t i = 0; i < team_size.size(); ++i) {
    const int c = static_cast<int>(std::lower_bound(sizes.begin(), sizes.end(), team_size[i]) - sizes.begin());
    const double d = estimate(static_cast<int>(i), team_size[i]);
    durations[c].push_back(d);
    low = std::max(low, d);
    high += d;
  }
  for (auto& d : durations) std::sort(d.begin(), d.end(), std::greater<double>());
  auto lanes_for = [&](double t, std::vector<int>& lanes) {
    int blocks = 0;
    for (int c = 0; c < classes; ++c) {
      const int members = static_cast<int>(durations[c].size());
      int l = 1;
      while (l < members && lpt_completion(durations[c], l) > t) ++l;
      lanes[c] = l;
      blocks += l * sizes[c];
    }
    return blocks;
  };
  std::vector<int> lanes(classes, 1);
  if (lanes_for(low, lanes) <= grid_cap) high = low;
  for (int it = 0; it < 48 && high > low * (1.0 + 1e-3); ++it) {
    const double mid = 0.5 * (low + high);
    if (lanes_for(mid, lanes) <= grid_cap) {
      high = mid;
    } else {
      low = mid;
    }
  }
  if (lanes_out != nullptr) {
    lanes_out->assign(classes, 1);
    lanes_for(high, *lanes_out);
  }
  return high;
}

int create_teams(PdBatch* batch, const PdBatchOptions& opts) {
  const int count = batch->count;
  int sms = 0, optin = 0;
  PD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, batch->device));
  PD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, batch->device));
  int per_sm_forward = 0, per_sm_adjoint = 0;
  PD_CUDA(pdb200::team_forward_max_blocks(batch->precision, 0, &per_sm_forward));
  PD_CUDA(pdb200::team_adjoint_max_blocks(batch->precision, 0, &per_sm_adjoint));
  // Blocks per SM the team kernels are built for: the shared-memory budget of
  // an instance is the SM's share for one of them.
  const int occupancy = std::max(1, std::min(per_sm_forward, per_sm_adjoint));
  const int grid_cap = occupancy * sms;
  // Largest class: a power of two that leaves room for one lane of every smaller class.
  int largest = 1;
  while (largest * 4 <= grid_cap && largest < 64) largest *= 2;
  int smem_per_sm = 0;
  PD_CUDA(cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, batch->device));
  // 10 KB per block: static shared memory of the team kernels and the per-block reserve.
  const int budget = std::min(optin, smem_per_sm / occupancy) - 10 * 1024;
  std::vector<double> cost(count);
  std::vector<int> cls_of(count);
  batch->team_size.assign(count, 1);
  for (int i = 0; i < count; ++i) {
    const PdSolver* s = batch->solvers[i];
    const double nnz = static_cast<double>(s->factor.s.columns.size());
    const double samples = static_cast<double>(s->ne) * (s->hex ? 8 : 1);
    const double want = std::max(1.0, std::max(nnz / opts.team_nnz, samples / opts.team_samples));
    int size = 1;
    while (size < largest && size * 1.5 < want) size *= 2;
    batch->team_size[i] = size;
    cost[i] = nnz + 64.0 * samples;
  }
  const bool measured = opts.measured_us != nullptr && opts.measured_iterations != nullptr &&
                        opts.measured_team != nullptr;
  // Measured plan: per-iteration time t(b) = c + (t0 - c) b0 / b on b blocks
  // from the time t0 per iteration seen on b0 blocks, c the fixed latency of
  // an iteration (barriers, serial sections); estimated duration = iterations
  // x t(b), work = duration x b block-us.
  std::vector<double> per_iteration(count, 0.0), iterations(count, 0.0), measured_team(count, 1.0);
  auto estimate = [&](int i, int b) {
    constexpr double kFixedUs = 40.0;
    const double t0 = per_iteration[i];
    const double scalable = std::max(t0 - kFixedUs, 0.0) * measured_team[i] / b;
    return iterations[i] * (std::min(t0, kFixedUs) + scalable);
  };
  if (measured) {
    for (int i = 0; i < count; ++i) {
      iterations[i] = std::max(1, opts.measured_iterations[i]);
      measured_team[i] = std::max(1, opts.measured_team[i]);
      per_iteration[i] = std::max(opts.measured_us[i], 0.0) / iterations[i];
      int size = 1;
      while (size < std::min(largest, opts.measured_team[i])) size *= 2;
      batch->team_size[i] = size;
    }
    // Team sizes by a greedy descent on the planned makespan: double the
    // team of the instance with the longest estimated duration while that
    // shortens the plan (plan_makespan below).
    for (int guard = 0; guard < count; ++guard) {
      const double current = plan_makespan(batch->team_size, estimate, grid_cap, nullptr);
      int worst = -1;
      for (int i = 0; i < count; ++i) {
        if (batch->team_size[i] >= largest) continue;
        if (worst < 0 || estimate(i, batch->team_size[i]) > estimate(worst, batch->team_size[worst])) worst = i;
      }
      if (worst < 0) break;
      batch->team_size[worst] *= 2;
      if (!(plan_makespan(batch->team_size, estimate, grid_cap, nullptr) < current)) {
        batch->team_size[worst] /= 2;
        break;
      }
    }
    for (int i = 0; i < count; ++i) cost[i] = estimate(i, batch->team_size[i]);
  }
  // Classes present, ascending size. A class whose share of the grid (by
  // work) is smaller than one of its teams moves down to half the size, so
  // that no class with much work is left with a single serial lane.
  std::vector<int> sizes;
  std::vector<double> work;
  std::vector<int> members;
  int classes = 0;
  for (;;) {
    sizes.clear();
    for (int i = 0; i < count; ++i) sizes.push_back(batch->team_size[i]);
    std::sort(sizes.begin(), sizes.end());
    sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
    classes = static_cast<int>(sizes.size());
    work.assign(classes, 0.0);
    members.assign(classes, 0);
    double total = 0.0;
    for (int i = 0; i < count; ++i) {
      cls_of[i] = static_cast<int>(std::lower_bound(sizes.begin(), sizes.end(), batch->team_size[i]) - sizes.begin());
      work[cls_of[i]] += cost[i];
      members[cls_of[i]] += 1;
      total += cost[i];
    }
    int shrink = -1;
    for (int c = measured ? -1 : classes - 1; c >= 0; --c) {
      const double share = grid_cap * work[c] / total;
      if (sizes[c] > 1 && share < 2.0 * sizes[c] && members[c] > 1) {
        shrink = sizes[c];
        break;
      }
    }
    if (shrink < 0) break;
    for (int i = 0; i < count; ++i)
      if (batch->team_size[i] == shrink) batch->team_size[i] = shrink / 2;
  }
  double total_work = 0.0;
  for (double w : work) total_work += w;
  std::vector<int> teams(classes, 1);
  // One-block teams are cheap and their instances often iterate longest:
  // start with up to 16 of them.
  if (sizes[0] == 1) teams[0] = std::max(1, std::min(members[0], 16));
  auto used = [&]() {
    int blocks = 0;
    for (int c = 0; c < classes; ++c) blocks += teams[c] * sizes[c];
    return blocks;
  };
  if (used() > grid_cap) return pd_set_error(PD_ERR_UNSUPPORTED, "the team classes do not fit the co-resident grid");
  if (measured) {
    std::vector<int> planned;
    plan_makespan(batch->team_size, estimate, grid_cap, &planned);
    for (int c = 0; c < classes; ++c) teams[c] = planned[c];
    if (used() > grid_cap) return pd_set_error(PD_ERR_UNSUPPORTED, "the measured plan does not fit the co-resident grid");
  }
  // Add lanes where a class's share of the grid is furthest below its share of the work.
  for (;;) {
    int best = -1;
    double best_gap = 0.0;
    for (int c = 0; c < classes; ++c) {
      if (teams[c] >= members[c] || used() + sizes[c] > grid_cap) continue;
      const double gap = work[c] / total_work - static_cast<double>(teams[c] * sizes[c]) / grid_cap;
      if (best < 0 || gap > best_gap) {
        best = c;
        best_gap = gap;
      }
    }
    if (best < 0) break;
    teams[best] += 1;
  }
  // Plans, argument blocks and queues. Each instance is planned for its team,
  // its argument blocks take the plan's pointers, and the batch takes the
  // plan's buffers (the solver plans its single-instance launch again when it
  // next steps on its own).
  size_t smem = 0;
  std::vector<pdb200::StepArgs> forward(count);
  std::vector<pdb200::AdjointArgs> adjoint(count);
  batch->team_plans.clear();
  for (int i = 0; i < count; ++i) {
    PdSolver* s = batch->solvers[i];
    if (int status = pd_plan_launch(s, batch->team_size[i], budget)) return status;
    if (int status = pd_ensure_adjoint_buffers(s)) return status;
    smem = std::max(smem, s->smem);
    fill_step_args(s, &forward[i]);
    fill_adjoint_args(s, &adjoint[i]);
    forward[i].timers = nullptr;
    batch->team_plans.emplace_back(new TeamPlanBuffers());
    batch->team_plans.back()->take(s);
  }
  std::vector<int> class_begin(classes + 1, 0), class_order;
  for (int c = 0; c < classes; ++c) {
    std::vector<int> list;
    for (int i = 0; i < count; ++i)
      if (cls_of[i] == c) list.push_back(i);
    std::stable_sort(list.begin(), list.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    class_order.insert(class_order.end(), list.begin(), list.end());
    class_begin[c + 1] = static_cast<int>(class_order.size());
  }
  std::vector<int> lane_start(1, 0), lane_class;
  for (int c = classes - 1; c >= 0; --c) {
    for (int t = 0; t < teams[c]; ++t) {
      lane_class.push_back(c);
      lane_start.push_back(lane_start.back() + sizes[c]);
    }
  }
  batch->lanes = static_cast<int>(lane_class.size());
  batch->classes = classes;
  batch->solo_class = sizes[0] == 1 ? 0 : -1;
  // The adjoint's own lane counts and queue order from its measured durations
  // (same team sizes and classes, so the same plans serve both launches).
  batch->adj_lanes = 0;
  if (measured && opts.measured_adjoint_us != nullptr) {
    auto adjoint_estimate = [&](int i, int b) {
      return std::max(opts.measured_adjoint_us[i], 0.0) * measured_team[i] / b;
    };
    std::vector<int> adj_teams;
    plan_makespan(batch->team_size, adjoint_estimate, grid_cap, &adj_teams);
    int blocks = 0;
    for (int c = 0; c < classes; ++c) blocks += adj_teams[c] * sizes[c];
    if (blocks <= grid_cap) {
      std::vector<double> adj_cost(count), adj_work(classes, 0.0);
      double adj_total = 0.0;
      for (int i = 0; i < count; ++i) {
        adj_cost[i] = adjoint_estimate(i, batch->team_size[i]);
        adj_work[cls_of[i]] += adj_cost[i];
        adj_total += adj_cost[i];
      }
      for (;;) {
        int best = -1;
        double best_gap = 0.0;
        for (int c = 0; c < classes; ++c) {
          if (adj_teams[c] >= members[c] || blocks + sizes[c] > grid_cap) continue;
          const double gap = adj_work[c] / std::max(adj_total, 1e-30) -
                             static_cast<double>(adj_teams[c] * sizes[c]) / grid_cap;
          if (best < 0 || gap > best_gap) {
            best = c;
            best_gap = gap;
          }
        }
        if (best < 0) break;
        adj_teams[best] += 1;
        blocks += sizes[best];
      }
      std::vector<int> adj_begin(classes + 1, 0), adj_order;
      for (int c = 0; c < classes; ++c) {
        std::vector<int> list;
        for (int i = 0; i < count; ++i)
          if (cls_of[i] == c) list.push_back(i);
        std::stable_sort(list.begin(), list.end(), [&](int x, int y) { return adj_cost[x] > adj_cost[y]; });
        adj_order.insert(adj_order.end(), list.begin(), list.end());
        adj_begin[c + 1] = static_cast<int>(adj_order.size());
      }
      std::vector<int> adj_start(1, 0), adj_class;
      for (int c = classes - 1; c >= 0; --c) {
        for (int t = 0; t < adj_teams[c]; ++t) {
          adj_class.push_back(c);
          adj_start.push_back(adj_start.back() + sizes[c]);
        }
      }
      PD_CUDA(batch->d_adj_lane_start.upload(adj_start));
      PD_CUDA(batch->d_adj_lane_class.upload(adj_class));
      PD_CUDA(batch->d_adj_class_begin.upload(adj_begin));
      PD_CUDA(batch->d_adj_class_order.upload(adj_order));
      batch->adj_lanes = static_cast<int>(adj_class.size());
      batch->adj_team_blocks = adj_start.back();
    }
  }
  const int lane_slots = std::max(batch->lanes, batch->adj_lanes);
  std::vector<long long> particle_offset(batch->particle_offsets.begin(), batch->particle_offsets.end() - 1);
  std::vector<long long> element_offset(batch->element_offsets.begin(), batch->element_offsets.end() - 1);
  PD_CUDA(batch->d_forward_args.upload(forward));
  PD_CUDA(batch->d_adjoint_args.upload(adjoint));
  PD_CUDA(batch->d_lane_start.upload(lane_start));
  PD_CUDA(batch->d_lane_class.upload(lane_class));
  PD_CUDA(batch->d_class_begin.upload(class_begin));
  PD_CUDA(batch->d_class_order.upload(class_order));
  PD_CUDA(batch->d_particle_offset.upload(particle_offset));
  PD_CUDA(batch->d_element_offset.upload(element_offset));
  PD_CUDA(batch->d_class_head.allocate(static_cast<size_t>(classes) * sizeof(unsigned)));
  PD_CUDA(batch->d_lane_slot.allocate(static_cast<size_t>(lane_slots) * sizeof(int)));
  PD_CUDA(batch->d_barriers.allocate(static_cast<size_t>(lane_slots) * sizeof(pdb200::GridBarrier)));
  PD_CUDA(batch->d_team_status.allocate(sizeof(int)));
  PD_CUDA(batch->d_timeline.allocate(static_cast<size_t>(count) * 4 * sizeof(unsigned long long)));
  PD_CUDA(pdb200::team_forward_max_blocks(batch->precision, smem, &per_sm_forward));
  PD_CUDA(pdb200::team_adjoint_max_blocks(batch->precision, smem, &per_sm_adjoint));
  batch->team_blocks = lane_start.back();
  if (std::max(batch->team_blocks, batch->adj_team_blocks) > std::max(1, std::min(per_sm_forward, per_sm_adjoint)) * sms)
    return pd_set_error(PD_ERR_UNSUPPORTED, "the lanes do not fit the co-resident grid");
  batch->team_smem = smem;
  PD_CUDA(cudaStreamCreateWithFlags(&batch->capture, cudaStreamNonBlocking));
  return PD_OK;
}

extern "C" int pd_batch_create(PdSolver* const* solvers, int32_t count, const PdBatchOptions* options,
                               PdBatch** out) {
  if (solvers == nullptr || out == nullptr || count < 1) return pd_set_error(PD_ERR_INVALID, "batch needs solvers");
  *out = nullptr;
  PdBatchOptions opts{};
  opts.svd_warm_start = 1;
  opts.task_nnz = 32768;
  opts.run_gap = 2;
  opts.local_cells = 64;
  opts.schedule = PD_BATCH_TEAMS;
  opts.team_nnz = 65536;
  opts.team_samples = 512;
  if (options != nullptr) opts = *options;
  if (opts.task_nnz < 256 || opts.run_gap < 0 || opts.local_cells < 4 || opts.team_nnz < 1 || opts.team_samples < 1 ||
      (opts.schedule != PD_BATCH_TEAMS && opts.schedule != PD_BATCH_PHASES))
    return pd_set_error(PD_ERR_INVALID, "batch options out of range");
  auto batch = std::make_unique<PdBatch>();
  batch->count = count;
  batch->solvers.assign(solvers, solvers + count);
  for (int i = 0; i < count; ++i) {
    const PdSolver* s = solvers[i];
    if (s == nullptr) return pd_set_error(PD_ERR_INVALID, "null solver in batch");
    if (!s->built || s->stale) return pd_set_error(PD_ERR_STATE, "every batched solver must be built (pd_build)");
    if (s->device != solvers[0]->device || s->options.precision != solvers[0]->options.precision ||
        s->options.state_precision != solvers[0]->options.state_precision || s->built_dt != solvers[0]->built_dt)
      return pd_set_error(PD_ERR_INVALID, "batched solvers must share device, precision, state precision and dt");
    if (s->activations != nullptr && !s->hex)
      return pd_set_error(PD_ERR_UNSUPPORTED, "muscle activations are not supported by the batched path");
    if (s->has_mesh_contact)
      return pd_set_error(PD_ERR_UNSUPPORTED, "mesh_contact is not supported by the batched path");
    if (s->has_friction)
      return pd_set_error(PD_ERR_UNSUPPORTED, "frictional_boundary is not supported by the batched path");
  }
  batch->device = solvers[0]->device;
  batch->precision = solvers[0]->options.precision;
  batch->state_f64 = solvers[0]->options.state_precision;
  PD_CUDA(cudaSetDevice(batch->device));
  int64_t particles = 0, elements = 0;
  for (int i = 0; i < count; ++i) {
    batch->particle_offsets.push_back(particles);
    batch->element_offsets.push_back(elements);
    particles += solvers[i]->n;
    elements += solvers[i]->ne;
  }
  batch->particle_offsets.push_back(particles);
  batch->element_offsets.push_back(elements);
  for (int i = 0; i < count; ++i) batch->generations.push_back(solvers[i]->generation);
  batch->schedule = opts.schedule;
  int max_iterations = 0;
  for (int i = 0; i < count; ++i) max_iterations = std::max(max_iterations, solvers[i]->options.max_iterations);
  batch->max_iterations = static_cast<unsigned>(max_iterations);
  if (int status = opts.schedule == PD_BATCH_PHASES ? create_phases(batch.get(), opts) : create_teams(batch.get(), opts))
    return status;
  *out = batch.release();
  return PD_OK;
}

extern "C" int pd_batch_destroy(PdBatch* batch) {
  if (batch == nullptr) return PD_OK;
  cudaSetDevice(batch->device);
  delete batch;
  return PD_OK;
}

extern "C" int pd_batch_layout(const PdBatch* batch, int64_t* particle_offsets, int64_t* element_offsets) {
  if (batch == nullptr) return pd_set_error(PD_ERR_INVALID, "null batch");
  for (int i = 0; i <= batch->count; ++i) {
    if (particle_offsets) particle_offsets[i] = batch->particle_offsets[i];
    if (element_offsets) element_offsets[i] = batch->element_offsets[i];
  }
  return PD_OK;
}

extern "C" int pd_batch_factor_stats(const PdBatch* batch, int64_t* values, int64_t* runs, int64_t* tasks) {
  if (batch == nullptr) return pd_set_error(PD_ERR_INVALID, "null batch");
  if (values) *values = batch->value_count;
  if (runs) *runs = batch->run_count;
  if (tasks) {
    tasks[0] = batch->n_local;
    tasks[1] = batch->n_gather;
    tasks[2] = batch->n_s;
    tasks[3] = batch->n_st;
  }
  return PD_OK;
}

namespace {

// Device table of the rollout's step pointers and the iteration log.
int prepare_rollout(PdBatch* b, const GraphKey& key) {
  const size_t elem = b->state_f64 ? sizeof(double) : sizeof(float);
  const size_t particles = static_cast<size_t>(b->particle_offsets.back());
  const size_t step_bytes = 3 * particles * elem;
  std::vector<BatchStepIo> table(key.steps);
  for (int t = 0; t < key.steps; ++t) {
    BatchStepIo& io = table[t];
    const char* q_traj = static_cast<const char*>(key.q_traj);
    const char* qd_traj = static_cast<const char*>(key.qd_traj);
    io.q_in = t == 0 ? key.q0 : static_cast<const void*>(q_traj + (t - 1) * step_bytes);
    io.qd_in = t == 0 ? key.qd0 : static_cast<const void*>(qd_traj + (t - 1) * step_bytes);
    io.f_in = static_cast<const char*>(key.forces) + static_cast<size_t>(t) * key.force_stride * elem;
    io.q_out = static_cast<char*>(key.q_traj) + t * step_bytes;
    io.qd_out = static_cast<char*>(key.qd_traj) + t * step_bytes;
    io.x_record = key.x_record != nullptr ? key.x_record + static_cast<size_t>(t) * 3 * particles : nullptr;
  }
  PD_CUDA(b->d_io.upload(table));
  PD_CUDA(b->d_log.allocate(static_cast<size_t>(key.steps) * b->count * sizeof(int)));
  return PD_OK;
}

int build_graph(PdBatch* b, const GraphKey& key) {
  if (b->exec != nullptr) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph != nullptr) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  if (int status = prepare_rollout(b, key)) return status;
  PD_CUDA(cudaGraphCreate(&b->graph, 0));
  const BatchInstance* insts = b->d_instances.as<BatchInstance>();
  const RangeTask* local_tasks = b->d_local_tasks.as<RangeTask>();
  const RangeTask* gather_tasks = b->d_gather_tasks.as<RangeTask>();
  const RowTask* s_tasks = b->d_s_tasks.as<RowTask>();
  const RowTask* st_tasks = b->d_st_tasks.as<RowTask>();
  BatchControl* control = b->d_control.as<BatchControl>();
  const BatchStepIo* io = b->d_io.as<BatchStepIo>();
  int* log = b->d_log.as<int>();
  pdb200::ScheduleView sch{b->count, b->d_n_active.as<int>(), b->d_active.as<int>(), b->d_prefix.as<int>(),
                           b->d_task_begin.as<int>()};
  pdb200::Gravity gravity{{key.gravity[0], key.gravity[1], key.gravity[2]}};
  double dt = key.dt;
  int steps = key.steps;
  unsigned max_passes = static_cast<unsigned>(key.steps) * (b->max_iterations + 1u) + 1u;
  cudaGraphNode_t prologue, schedule, loop;
  {
    void* args[] = {&insts, &io, &dt, &gravity, &control};
    PD_CUDA(add_kernel(&prologue, b->graph, nullptr, 0, reinterpret_cast<const void*>(&pdb200::batch_prologue_kernel),
                       b->count, 0, args));
  }
  {
    void* args[] = {&insts, &sch};
    PD_CUDA(add_kernel(&schedule, b->graph, &prologue, 1, reinterpret_cast<const void*>(&pdb200::batch_schedule_kernel),
                       1, 0, args));
  }
  cudaGraphConditionalHandle handle;
  PD_CUDA(cudaGraphConditionalHandleCreate(&handle, b->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  PD_CUDA(cudaGraphAddNode(&loop, b->graph, &schedule, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaGraphNode_t n_local, n_gather, n_s, n_st, n_aa;
  {
    void* args[] = {&insts, &local_tasks, &sch};
    PD_CUDA(add_kernel(&n_local, body, nullptr, 0, local_kernel(b->precision), b->grid[0], 0, args));
  }
  {
    void* args[] = {&insts, &gather_tasks, &sch};
    PD_CUDA(add_kernel(&n_gather, body, &n_local, 1, gather_kernel(b->precision), b->grid[1], 0, args));
  }
  {
    void* args[] = {&insts, &s_tasks, &sch};
    PD_CUDA(add_kernel(&n_s, body, &n_gather, 1, s_kernel(b->precision), b->grid[2], b->smem_s, args));
  }
  {
    void* args[] = {&insts, &st_tasks, &sch};
    PD_CUDA(add_kernel(&n_st, body, &n_s, 1, st_kernel(b->precision), b->grid[3], b->smem_st, args));
  }
  {
    void* args[] = {&insts, &control, &handle, &max_passes, &io, &steps, &dt, &gravity, &log, &sch};
    PD_CUDA(add_kernel(&n_aa, body, &n_st, 1, reinterpret_cast<const void*>(&pdb200::batch_anderson_kernel), b->count,
                       0, args));
  }
  PD_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->key = key;
  return PD_OK;
}

}  // namespace

namespace {

pdb200::TeamLaunch team_launch(const PdBatch* b, int steps, double dt, const double gravity[3], bool adjoint = false) {
  pdb200::TeamLaunch launch{};
  const bool own = adjoint && b->adj_lanes > 0;
  launch.forward = b->d_forward_args.as<pdb200::StepArgs>();
  launch.adjoint = b->d_adjoint_args.as<pdb200::AdjointArgs>();
  launch.lane_start = own ? b->d_adj_lane_start.as<int>() : b->d_lane_start.as<int>();
  launch.lane_class = own ? b->d_adj_lane_class.as<int>() : b->d_lane_class.as<int>();
  launch.class_begin = own ? b->d_adj_class_begin.as<int>() : b->d_class_begin.as<int>();
  launch.class_order = own ? b->d_adj_class_order.as<int>() : b->d_class_order.as<int>();
  launch.particle_offset = b->d_particle_offset.as<long long>();
  launch.element_offset = b->d_element_offset.as<long long>();
  launch.count = b->count;
  launch.lanes = own ? b->adj_lanes : b->lanes;
  launch.solo_class = b->solo_class;
  launch.steps = steps;
  launch.dt = dt;
  for (int c = 0; c < 3; ++c) launch.gravity[c] = gravity != nullptr ? gravity[c] : 0.0;
  launch.state_f64 = b->state_f64;
  launch.class_head = b->d_class_head.as<unsigned>();
  launch.lane_slot = b->d_lane_slot.as<int>();
  launch.lane_barrier = b->d_barriers.as<pdb200::GridBarrier>();
  launch.status = b->d_team_status.as<int>();
  launch.particles = b->particle_offsets.back();
  launch.timers = b->timers;
  launch.timer_instance = b->timer_instance;
  return launch;
}

// Captures queue reset, the given clears and one team launch into a graph on
// the batch's private stream (the caller's stream may be the legacy default
// stream, which cannot capture).
int capture_team_rollout(PdBatch* b, const pdb200::TeamLaunch& launch, bool adjoint,
                         const std::vector<std::pair<void*, size_t>>& clears, cudaGraphExec_t* exec) {
  if (*exec != nullptr) {
    cudaGraphExecDestroy(*exec);
    *exec = nullptr;
  }
  PD_CUDA(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
  cudaError_t status = cudaMemsetAsync(b->d_barriers.ptr, 0, b->d_barriers.bytes, b->capture);
  if (status == cudaSuccess) status = cudaMemsetAsync(b->d_class_head.ptr, 0, b->d_class_head.bytes, b->capture);
  if (status == cudaSuccess) status = cudaMemsetAsync(b->d_team_status.ptr, 0, b->d_team_status.bytes, b->capture);
  for (const auto& clear : clears) {
    if (status == cudaSuccess && clear.first != nullptr) status = cudaMemsetAsync(clear.first, 0, clear.second, b->capture);
  }
  if (status == cudaSuccess) {
    status = adjoint ? pdb200::launch_team_adjoint(launch, b->adj_lanes > 0 ? b->adj_team_blocks : b->team_blocks,
                                                   b->precision, b->team_smem, b->capture)
                     : pdb200::launch_team_forward(launch, b->team_blocks, b->precision, b->team_smem, b->capture);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ended = cudaStreamEndCapture(b->capture, &graph);
  if (status == cudaSuccess) status = ended;
  if (status == cudaSuccess) status = cudaGraphInstantiate(exec, graph, 0);
  if (graph != nullptr) cudaGraphDestroy(graph);
  PD_CUDA(status);
  return PD_OK;
}

}  // namespace

// A batch holds pointers into its solvers' buffers: after a rebuild or a
// window change reallocated them, it must be created again.
static int check_generations(const PdBatch* batch) {
  for (size_t i = 0; i < batch->solvers.size(); ++i) {
    if (batch->solvers[i]->generation != batch->generations[i])
      return pd_set_error(PD_ERR_STATE, "a batched solver was rebuilt or resized after the batch was created; "
                                        "create the batch again");
  }
  return PD_OK;
}

extern "C" int pd_batch_forward(PdBatch* batch, int32_t steps, double dt, const double gravity[3], const void* q0,
                                const void* qd0, const void* forces, int64_t force_step_stride, void* q_traj,
                                void* qd_traj, double* x_record, void* stream) {
  if (batch == nullptr || gravity == nullptr || q0 == nullptr || qd0 == nullptr || forces == nullptr ||
      q_traj == nullptr || qd_traj == nullptr)
    return pd_set_error(PD_ERR_INVALID, "null argument");
  if (steps < 1) return pd_set_error(PD_ERR_INVALID, "steps must be positive");
  if (force_step_stride < 0) return pd_set_error(PD_ERR_INVALID, "force step stride must be nonnegative");
  for (const PdSolver* s : batch->solvers) {
    if (!s->built || s->stale || s->built_dt != dt)
      return pd_set_error(PD_ERR_STATE, "every batched solver must be built (pd_build) for this dt");
  }
  if (int status = check_generations(batch)) return status;
  PD_CUDA(cudaSetDevice(batch->device));
  GraphKey key;
  key.steps = steps;
  key.dt = dt;
  for (int c = 0; c < 3; ++c) key.gravity[c] = gravity[c];
  key.q0 = q0;
  key.qd0 = qd0;
  key.forces = forces;
  key.force_stride = force_step_stride;
  key.q_traj = q_traj;
  key.qd_traj = qd_traj;
  key.x_record = x_record;
  if (batch->schedule == PD_BATCH_TEAMS) {
    if (batch->exec == nullptr || !(batch->key == key)) {
      PD_CUDA(batch->d_log.allocate(static_cast<size_t>(steps) * batch->count * sizeof(int)));
      pdb200::TeamLaunch launch = team_launch(batch, steps, dt, gravity);
      launch.q0 = q0;
      launch.qd0 = qd0;
      launch.forces = forces;
      launch.force_stride = force_step_stride;
      launch.q_traj = q_traj;
      launch.qd_traj = qd_traj;
      launch.x_record = x_record;
      launch.iteration_log = batch->d_log.as<int>();
      launch.timeline = batch->d_timeline.as<unsigned long long>();
      if (int status = capture_team_rollout(batch, launch, false, {}, &batch->exec)) return status;
      batch->key = key;
    }
    PD_CUDA(cudaGraphLaunch(batch->exec, static_cast<cudaStream_t>(stream)));
    return PD_OK;
  }
  if (batch->exec == nullptr || !(batch->key == key)) {
    if (int status = build_graph(batch, key)) return status;
  }
  PD_CUDA(cudaGraphLaunch(batch->exec, static_cast<cudaStream_t>(stream)));
  return PD_OK;
}

extern "C" int pd_batch_backward(PdBatch* batch, int32_t steps, double dt, const double* x_record,
                                 const void* grad_q_final, const void* grad_qd_final, void* grad_q, void* grad_qd,
                                 void* grad_forces, double* grad_materials, int32_t* iterations, void* stream) {
  if (batch == nullptr || x_record == nullptr || grad_q_final == nullptr || grad_qd_final == nullptr ||
      grad_q == nullptr || grad_qd == nullptr || grad_forces == nullptr)
    return pd_set_error(PD_ERR_INVALID, "null argument");
  if (steps < 1) return pd_set_error(PD_ERR_INVALID, "steps must be positive");
  if (batch->schedule != PD_BATCH_TEAMS)
    return pd_set_error(PD_ERR_UNSUPPORTED, "the batched adjoint runs on the teams schedule");
  for (const PdSolver* s : batch->solvers) {
    if (!s->built || s->stale || s->built_dt != dt)
      return pd_set_error(PD_ERR_STATE, "the batched adjoint needs the factors of its rollout (same dt)");
  }
  if (int status = check_generations(batch)) return status;
  PD_CUDA(cudaSetDevice(batch->device));
  GraphKey key;
  key.steps = steps;
  key.dt = dt;
  key.q0 = x_record;
  key.qd0 = grad_q_final;
  key.forces = grad_qd_final;
  key.q_traj = grad_q;
  key.qd_traj = grad_qd;
  key.x_record = const_cast<double*>(static_cast<const double*>(grad_forces));
  key.force_stride = reinterpret_cast<long long>(grad_materials);
  if (batch->adjoint_exec == nullptr || !(batch->adjoint_key == key)) {
    PD_CUDA(batch->d_adjoint_log.allocate(static_cast<size_t>(steps) * batch->count * sizeof(int)));
    pdb200::TeamLaunch launch = team_launch(batch, steps, dt, nullptr, true);
    launch.x_record = const_cast<double*>(x_record);
    launch.grad_q_final = grad_q_final;
    launch.grad_qd_final = grad_qd_final;
    launch.grad_q = grad_q;
    launch.grad_qd = grad_qd;
    launch.grad_forces = grad_forces;
    launch.grad_materials = grad_materials;
    launch.iteration_log = batch->d_adjoint_log.as<int>();
    launch.timeline = batch->d_timeline.as<unsigned long long>() + 2 * batch->count;
    const size_t elem = batch->state_f64 ? sizeof(double) : sizeof(float);
    const size_t step_bytes = static_cast<size_t>(3) * batch->particle_offsets.back() * elem;
    std::vector<std::pair<void*, size_t>> clears = {
        {grad_forces, steps * step_bytes},
        {grad_materials, static_cast<size_t>(2) * batch->element_offsets.back() * sizeof(double)}};
    if (int status = capture_team_rollout(batch, launch, true, clears, &batch->adjoint_exec)) return status;
    batch->adjoint_key = key;
  }
  PD_CUDA(cudaGraphLaunch(batch->adjoint_exec, static_cast<cudaStream_t>(stream)));
  if (iterations != nullptr) {
    PD_CUDA(cudaMemcpyAsync(iterations, batch->d_adjoint_log.ptr, static_cast<size_t>(steps) * batch->count * sizeof(int),
                            cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
    PD_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  }
  return PD_OK;
}

extern "C" int pd_batch_read(PdBatch* batch, int32_t* status, int32_t* iterations, void* stream) {
  if (batch == nullptr) return pd_set_error(PD_ERR_INVALID, "null batch");
  PD_CUDA(cudaSetDevice(batch->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (status) {
    // Read and clear, like pd_read_status: the bits of the next read start
    // from this one.
    for (int i = 0; i < batch->count; ++i) {
      PD_CUDA(cudaMemcpyAsync(status + i, batch->solvers[i]->d_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
      PD_CUDA(cudaMemsetAsync(batch->solvers[i]->d_status.ptr, 0, sizeof(int), st));
    }
  }
  if (iterations && batch->d_log.ptr != nullptr && batch->key.steps > 0) {
    PD_CUDA(cudaMemcpyAsync(iterations, batch->d_log.ptr, static_cast<size_t>(batch->key.steps) * batch->count * sizeof(int),
                            cudaMemcpyDeviceToHost, st));
  }
  PD_CUDA(cudaStreamSynchronize(st));
  return PD_OK;
}

// The same rollout with every kernel launched on its own (no graph): one
// launch per phase and pass, the loop decided on the host every 16 passes.
// Slower than the graph; it exists so that profilers that follow plain
// launches see every kernel of the batched path.
extern "C" int pd_batch_forward_stepwise(PdBatch* batch, int32_t steps, double dt, const double gravity[3],
                                         const void* q0, const void* qd0, const void* forces,
                                         int64_t force_step_stride, void* q_traj, void* qd_traj, double* x_record,
                                         void* stream) {
  if (batch == nullptr || gravity == nullptr || q0 == nullptr || qd0 == nullptr || forces == nullptr ||
      q_traj == nullptr || qd_traj == nullptr)
    return pd_set_error(PD_ERR_INVALID, "null argument");
  if (steps < 1) return pd_set_error(PD_ERR_INVALID, "steps must be positive");
  if (force_step_stride < 0) return pd_set_error(PD_ERR_INVALID, "force step stride must be nonnegative");
  if (batch->schedule != PD_BATCH_PHASES)
    return pd_set_error(PD_ERR_UNSUPPORTED, "stepwise launches exist for the phases schedule");
  for (const PdSolver* s : batch->solvers) {
    if (!s->built || s->stale || s->built_dt != dt)
      return pd_set_error(PD_ERR_STATE, "every batched solver must be built (pd_build) for this dt");
  }
  if (int status = check_generations(batch)) return status;
  PD_CUDA(cudaSetDevice(batch->device));
  GraphKey key;
  key.steps = steps;
  key.dt = dt;
  for (int c = 0; c < 3; ++c) key.gravity[c] = gravity[c];
  key.q0 = q0;
  key.qd0 = qd0;
  key.forces = forces;
  key.force_stride = force_step_stride;
  key.q_traj = q_traj;
  key.qd_traj = qd_traj;
  key.x_record = x_record;
  if (!(batch->key == key) || batch->d_io.ptr == nullptr) {
    // The step table is rebuilt: a cached graph would point at the old one.
    if (batch->exec != nullptr) {
      cudaGraphExecDestroy(batch->exec);
      batch->exec = nullptr;
    }
    if (batch->graph != nullptr) {
      cudaGraphDestroy(batch->graph);
      batch->graph = nullptr;
    }
    if (int status = prepare_rollout(batch, key)) return status;
    batch->key = key;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const BatchInstance* insts = batch->d_instances.as<BatchInstance>();
  BatchControl* control = batch->d_control.as<BatchControl>();
  const BatchStepIo* io = batch->d_io.as<BatchStepIo>();
  int* log = batch->d_log.as<int>();
  const pdb200::ScheduleView sch{batch->count, batch->d_n_active.as<int>(), batch->d_active.as<int>(),
                                 batch->d_prefix.as<int>(), batch->d_task_begin.as<int>()};
  const pdb200::Gravity g{{gravity[0], gravity[1], gravity[2]}};
  const unsigned max_passes = static_cast<unsigned>(steps) * (batch->max_iterations + 1u) + 1u;
  const int p = batch->precision;
  const RangeTask* local_tasks = batch->d_local_tasks.as<RangeTask>();
  const RangeTask* gather_tasks = batch->d_gather_tasks.as<RangeTask>();
  const RowTask* s_tasks = batch->d_s_tasks.as<RowTask>();
  const RowTask* st_tasks = batch->d_st_tasks.as<RowTask>();
  pdb200::batch_prologue_kernel<<<batch->count, pdb200::kBlock, 0, st>>>(insts, io, dt, g, control);
  pdb200::batch_schedule_kernel<<<1, pdb200::kBlock, 0, st>>>(insts, sch);
  for (unsigned pass = 0; pass < max_passes; ++pass) {
    if (p == PD_PRECISION_FP32) {
      pdb200::batch_local_kernel<float><<<batch->grid[0], pdb200::kBlock, 0, st>>>(insts, local_tasks, sch);
    } else {
      pdb200::batch_local_kernel<double><<<batch->grid[0], pdb200::kBlock, 0, st>>>(insts, local_tasks, sch);
    }
    if (p == PD_PRECISION_FP64) {
      pdb200::batch_gather_kernel<double><<<batch->grid[1], pdb200::kBlock, 0, st>>>(insts, gather_tasks, sch);
      pdb200::batch_s_kernel<double><<<batch->grid[2], pdb200::kBlock, batch->smem_s, st>>>(insts, s_tasks, sch);
      pdb200::batch_st_kernel<double><<<batch->grid[3], pdb200::kBlock, batch->smem_st, st>>>(insts, st_tasks, sch);
    } else {
      pdb200::batch_gather_kernel<float><<<batch->grid[1], pdb200::kBlock, 0, st>>>(insts, gather_tasks, sch);
      pdb200::batch_s_kernel<float><<<batch->grid[2], pdb200::kBlock, batch->smem_s, st>>>(insts, s_tasks, sch);
      pdb200::batch_st_kernel<float><<<batch->grid[3], pdb200::kBlock, batch->smem_st, st>>>(insts, st_tasks, sch);
    }
    pdb200::batch_anderson_kernel<<<batch->count, pdb200::kBlock, 0, st>>>(insts, control, 0, max_passes, io, steps,
                                                                          dt, g, log, sch);
    PD_CUDA(cudaGetLastError());
    if ((pass + 1) % 16 == 0) {
      unsigned active = 0;
      PD_CUDA(cudaMemcpyAsync(&active, &control->last_active, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
      PD_CUDA(cudaStreamSynchronize(st));
      if (active == 0) break;
    }
  }
  return PD_OK;
}

extern "C" int pd_batch_team_sizes(const PdBatch* batch, int32_t* sizes, int32_t* grid) {
  if (batch == nullptr) return pd_set_error(PD_ERR_INVALID, "null batch");
  if (sizes != nullptr) {
    for (int i = 0; i < batch->count; ++i) sizes[i] = batch->schedule == PD_BATCH_TEAMS ? batch->team_size[i] : 0;
  }
  if (grid != nullptr) *grid = batch->team_blocks;
  return PD_OK;
}

extern "C" int pd_batch_timeline(PdBatch* batch, uint64_t* forward, uint64_t* adjoint, void* stream) {
  if (batch == nullptr) return pd_set_error(PD_ERR_INVALID, "null batch");
  if (batch->schedule != PD_BATCH_TEAMS || batch->d_timeline.ptr == nullptr)
    return pd_set_error(PD_ERR_UNSUPPORTED, "timelines are recorded by the teams schedule");
  PD_CUDA(cudaSetDevice(batch->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t half = static_cast<size_t>(2) * batch->count * sizeof(uint64_t);
  const char* base = static_cast<const char*>(batch->d_timeline.ptr);
  if (forward != nullptr) PD_CUDA(cudaMemcpyAsync(forward, base, half, cudaMemcpyDeviceToHost, st));
  if (adjoint != nullptr) PD_CUDA(cudaMemcpyAsync(adjoint, base + half, half, cudaMemcpyDeviceToHost, st));
  PD_CUDA(cudaStreamSynchronize(st));
  return PD_OK;
}

extern "C" int pd_batch_set_phase_timers(PdBatch* batch, int32_t instance, unsigned long long* device_timers) {
  if (batch == nullptr) return pd_set_error(PD_ERR_INVALID, "null batch");
  batch->timers = device_timers;
  batch->timer_instance = instance;
  if (batch->exec != nullptr) {  // the captured launch holds the old setting
    cudaGraphExecDestroy(batch->exec);
    batch->exec = nullptr;
  }
  return PD_OK;
}
