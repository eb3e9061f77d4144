// The two costly stages of the factor build on the device, bit-identical to
// the host's in factor.cpp: the numeric LDL^T (sparse.py:136-151; see
// ldlt_rows_kernel) and the rows of L^{-1} (sparse.py:159-177, below).
//
// Row i of the unscaled inverse starts as e_i and, for every column k of row
// i of L in ascending order (k < i, multiplier L(i, k) != 0), subtracts
// L(i, k) times row k of the inverse; entries that end exactly zero are
// omitted. Row i only reads rows k < i, so the rows are computed level by
// level of the elimination tree (level(i) = 1 + max level(k) over the columns
// of row i): the rows of a level are independent.
//
// Within a row the columns are cut into chunks of kChunk labels aligned to
// multiples of kChunk; one block computes one (row, chunk) item in a shared
// memory accumulator. For each k the block reads only row k's entries inside
// its chunk, located through per-row chunk bounds recorded when row k was
// stored, and all its threads apply those updates at once (the entries of one
// row are distinct); a block barrier separates consecutive k, so every entry
// sees the same sequence of rounded multiplies and subtracts as the host walk
// (__dmul_rn / __dsub_rn: no contraction into fused multiply-adds). The
// nonzero entries are compacted in ascending label order into a scratch slot,
// then copied into the row pool at offsets the host assigns from the counts.
// With pd_factor_device_rows(1) the rows follow the host's grouped dense
// schedule instead (inverse_rows_group_kernel, at the end of this file).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "factor.h"

// Stage timings on stderr in builds with -DPD_FACTOR_TIMING (the timing probe).
#ifdef PD_FACTOR_TIMING
#include <chrono>
#include <cstdio>
#define PD_FT_NOW() std::chrono::steady_clock::now()
#define PD_FT_REPORT(name, t0, extra)                                                                          \
  std::fprintf(stderr, "[factor] %s %.3f s %s\n", name,                                                      \
               std::chrono::duration<double>(std::chrono::steady_clock::now() - (t0)).count(), (extra).c_str())
#else
#define PD_FT_NOW() 0
#define PD_FT_REPORT(name, t0, extra) (void)(t0)
#endif

namespace pdb200 {

namespace {

#ifndef PD_FACTOR_CHUNK
#define PD_FACTOR_CHUNK 256
#endif
constexpr int kChunk = PD_FACTOR_CHUNK;  // labels per chunk (256: a 2 KB accumulator per block)
constexpr int kThreads = 256;
constexpr int kMetaBatch = 32;  // columns of row i whose metadata one warp loads at once

struct ChunkItem {
  int32_t row;
  int32_t chunk;
  int64_t slot;  // offset of this item's scratch slot
};

__device__ __forceinline__ int block_exclusive_scan(int value, int* warp_totals, int& total) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int inclusive = value;
#pragma unroll
  for (int offset = 1; offset < 32; offset <<= 1) {
    const int other = __shfl_up_sync(0xffffffffu, inclusive, offset);
    if (lane >= offset) inclusive += other;
  }
  if (lane == 31) warp_totals[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    const int warps = blockDim.x >> 5;
    int t = lane < warps ? warp_totals[lane] : 0;
#pragma unroll
    for (int offset = 1; offset < 32; offset <<= 1) {
      const int other = __shfl_up_sync(0xffffffffu, t, offset);
      if (lane >= offset) t += other;
    }
    if (lane < warps) warp_totals[lane] = t;  // inclusive warp prefix
  }
  __syncthreads();
  total = warp_totals[(blockDim.x >> 5) - 1];
  const int before = warp == 0 ? 0 : warp_totals[warp - 1];
  return before + inclusive - value;
}

// One (row, chunk) item per block: accumulate, then compact the nonzeros.
__global__ void __launch_bounds__(kThreads) inverse_rows_chunk_kernel(
    const ChunkItem* __restrict__ items, const int64_t* __restrict__ lstart, const int32_t* __restrict__ lcols,
    const double* __restrict__ lvals, const int32_t* __restrict__ lo, const int64_t* __restrict__ row_off,
    const int64_t* __restrict__ cb_base, const int32_t* __restrict__ cb, const int32_t* __restrict__ pool_cols,
    const double* __restrict__ pool_vals, int32_t* __restrict__ scratch_cols, double* __restrict__ scratch_vals,
    int32_t* __restrict__ counts, int* __restrict__ error) {
  __shared__ double acc[kChunk];
  __shared__ double meta_coef[kMetaBatch];
  __shared__ int64_t meta_begin[kMetaBatch];
  __shared__ int64_t meta_end[kMetaBatch];
  __shared__ int warp_totals[kThreads / 32];
  const ChunkItem item = items[blockIdx.x];
  const int i = item.row;
  const int j = item.chunk;
  const int c_begin = max(lo[i], j * kChunk);
  const int c_end = min(i, (j + 1) * kChunk - 1) + 1;
  const int width = c_end - c_begin;
  for (int t = threadIdx.x; t < width; t += blockDim.x) acc[t] = (c_begin + t == i) ? 1.0 : 0.0;
  const int64_t p0 = lstart[i];
  const int64_t p1 = lstart[i + 1];
  for (int64_t base = p0; base < p1; base += kMetaBatch) {
    const int batch = static_cast<int>(p1 - base < kMetaBatch ? p1 - base : kMetaBatch);
    __syncthreads();  // the previous batch's metadata is consumed; the accumulator is initialised
    if (threadIdx.x < batch) {
      const int64_t p = base + threadIdx.x;
      const int k = lcols[p];
      const double coefficient = lvals[p];
      int64_t b = 0, e = 0;
      const int j0 = lo[k] / kChunk;
      const int j1 = k / kChunk;
      if (coefficient != 0.0 && j >= j0 && j <= j1) {
        const int32_t* bounds = cb + cb_base[k] + (j - j0);
        b = row_off[k] + bounds[0];
        e = row_off[k] + bounds[1];
      }
      meta_coef[threadIdx.x] = coefficient;
      meta_begin[threadIdx.x] = b;
      meta_end[threadIdx.x] = e;
    }
    __syncthreads();
    for (int l = 0; l < batch; ++l) {
      const int64_t b = meta_begin[l];
      const int64_t e = meta_end[l];
      if (b == e) continue;  // the same for every thread of the block
      const double coefficient = meta_coef[l];
      for (int64_t q = b + threadIdx.x; q < e; q += blockDim.x) {
        const int c = pool_cols[q] - c_begin;
        if (c < 0 || c >= width) {
          atomicOr(error, 1);
          continue;
        }
        acc[c] = __dsub_rn(acc[c], __dmul_rn(coefficient, pool_vals[q]));
      }
      __syncthreads();
    }
  }
  __syncthreads();
  // Ascending compaction: thread t owns the contiguous run [t*per, (t+1)*per).
  const int per = (width + blockDim.x - 1) / blockDim.x;
  const int t0 = min(width, static_cast<int>(threadIdx.x) * per);
  const int t1 = min(width, t0 + per);
  int mine = 0;
  for (int t = t0; t < t1; ++t) mine += acc[t] != 0.0 ? 1 : 0;
  int total = 0;
  int offset = block_exclusive_scan(mine, warp_totals, total);
  for (int t = t0; t < t1; ++t) {
    if (acc[t] != 0.0) {
      scratch_cols[item.slot + offset] = c_begin + t;
      scratch_vals[item.slot + offset] = acc[t];
      ++offset;
    }
  }
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// Moves every item's entries into the row pool and records the row offset and
// the row's chunk bounds (relative to the row's start).
__global__ void __launch_bounds__(kThreads) inverse_rows_copy_kernel(
    const ChunkItem* __restrict__ items, const int32_t* __restrict__ counts, const int64_t* __restrict__ placement,
    const int32_t* __restrict__ lo, const int64_t* __restrict__ cb_base, int32_t* __restrict__ cb,
    int64_t* __restrict__ row_off, const int32_t* __restrict__ scratch_cols, const double* __restrict__ scratch_vals,
    int32_t* __restrict__ pool_cols, double* __restrict__ pool_vals) {
  const ChunkItem item = items[blockIdx.x];
  const int count = counts[blockIdx.x];
  const int64_t out = placement[2 * blockIdx.x];
  const int64_t row_base = placement[2 * blockIdx.x + 1];
  for (int t = threadIdx.x; t < count; t += blockDim.x) {
    pool_cols[out + t] = scratch_cols[item.slot + t];
    pool_vals[out + t] = scratch_vals[item.slot + t];
  }
  if (threadIdx.x == 0) {
    const int i = item.row;
    const int j0 = lo[i] / kChunk;
    const int j1 = i / kChunk;
    if (item.chunk == j0) row_off[i] = row_base;
    cb[cb_base[i] + (item.chunk - j0)] = static_cast<int32_t>(out - row_base);
    if (item.chunk == j1) cb[cb_base[i] + (j1 - j0) + 1] = static_cast<int32_t>(out + count - row_base);
  }
}

constexpr int kLdltMaxPattern = 16384;  // strict entries of a row staged in (dynamic) shared memory

// Up to kThreads entries of one column j of L: entry 0 is the diagonal (row
// j), entry e >= 1 is row col_rows[col_start[j] + e - 1].
struct ColumnItem {
  int32_t column;
  int32_t first;
};

// Left-looking columns: every entry (i, j) of a column is the permuted A value
// minus m(i, k) e(j, k) over the columns k < j that rows i and j share, in
// ascending k, which is the sequence of rounded products and subtractions the
// host's right-looking update applies to it (pivot k updates (i, j) exactly
// when both rows hold column k). One thread per entry, merging row i's pattern
// with row j's, staged in shared memory with row j's unscaled entries; all the
// multipliers and unscaled entries read belong to columns of lower levels.
// The entries are stored unscaled; the diagonal entry is the pivot.
__global__ void __launch_bounds__(kThreads) ldlt_columns_kernel(
    const ColumnItem* __restrict__ items, const int64_t* __restrict__ row_start, const int32_t* __restrict__ pattern,
    const int64_t* __restrict__ col_start, const int32_t* __restrict__ col_rows, const int64_t* __restrict__ col_pos,
    const double* __restrict__ initial, const double* __restrict__ multipliers, double* __restrict__ unscaled,
    double* __restrict__ diagonal, int* __restrict__ fail_row) {
  extern __shared__ __align__(16) unsigned char ldlt_smem[];
  const ColumnItem item = items[blockIdx.x];
  const int j = item.column;
  const int64_t start_j = row_start[j];
  const int len_j = static_cast<int>(row_start[j + 1] - start_j - 1);
  double* e_j = reinterpret_cast<double*>(ldlt_smem);
  int32_t* pat_j = reinterpret_cast<int32_t*>(e_j + len_j);
  for (int t = threadIdx.x; t < len_j; t += blockDim.x) {
    pat_j[t] = pattern[start_j + t];
    e_j[t] = unscaled[start_j + t];
  }
  __syncthreads();
  const int count = static_cast<int>(col_start[j + 1] - col_start[j]) + 1;
  const int e = item.first + static_cast<int>(threadIdx.x);
  if (e >= count) return;
  if (e == 0) {
    const int64_t pos = start_j + len_j;
    double acc = initial[pos];
    for (int q = 0; q < len_j; ++q) acc = __dsub_rn(acc, __dmul_rn(multipliers[start_j + q], e_j[q]));
    unscaled[pos] = acc;
    diagonal[j] = acc;
    if (!isfinite(acc) || acc <= 0.0) atomicMin(fail_row, j);
    return;
  }
  const int i = col_rows[col_start[j] + e - 1];
  const int64_t pos = col_pos[col_start[j] + e - 1];  // entry (i, j): row i's columns before it are < j
  double acc = initial[pos];
  int64_t p = row_start[i];
  int q = 0;
  while (p < pos && q < len_j) {
    const int a = pattern[p];
    const int b = pat_j[q];
    if (a < b) {
      ++p;
    } else if (b < a) {
      ++q;
    } else {
      acc = __dsub_rn(acc, __dmul_rn(multipliers[p], e_j[q]));
      ++p;
      ++q;
    }
  }
  unscaled[pos] = acc;
}

// Multipliers of a level's columns: m(i, j) = e(i, j) / d_j (IEEE division).
__global__ void __launch_bounds__(kThreads) ldlt_divide_kernel(const ColumnItem* __restrict__ items,
                                                               const int64_t* __restrict__ col_start,
                                                               const int64_t* __restrict__ col_pos,
                                                               const double* __restrict__ unscaled,
                                                               const double* __restrict__ diagonal,
                                                               double* __restrict__ multipliers) {
  const ColumnItem item = items[blockIdx.x];
  const int j = item.column;
  const int count = static_cast<int>(col_start[j + 1] - col_start[j]) + 1;
  const int e = item.first + static_cast<int>(threadIdx.x);
  if (e == 0 || e >= count) return;
  const int64_t pos = col_pos[col_start[j] + e - 1];
  multipliers[pos] = unscaled[pos] / diagonal[j];
}

// Rows of L^{-1} as dense segments in groups of consecutive rows (the
// schedule of the host's inverse_rows_by_groups, planned by plan_row_groups):
// one block per (group, chunk) item of a level, one thread per label c of the
// chunk, which holds the entries (a + r, c) of the group's rows in registers.
// The thread applies every outside column k of the group in ascending order
// (row k's entry at c, read once for all the group's rows), then the group's
// own rows in ascending order from its registers, skipping zero multipliers:
// every entry sees the host walk's columns in ascending order, one
// __dmul_rn then one __dsub_rn each, and no thread reads another's entries,
// so the block has no barrier. Entries outside a row's labels [lo_i, i] are
// never read or written.
template <int kRows>
__global__ void __launch_bounds__(kRowGroupChunk)
    inverse_rows_group_kernel(const int2* items, const int32_t* group_start, const int64_t* u_start,
                              const int32_t* u_cols, const int64_t* outer_start, const double* outer,
                              const int64_t* inner_start, const double* inner, const int32_t* lo,
                              const int64_t* base, double* dense) {
  const int2 item = items[blockIdx.x];
  const int32_t g = item.x;
  const int32_t a = group_start[g];
  const int32_t rows = group_start[g + 1] - a;
  const int32_t c = item.y * kRowGroupChunk + static_cast<int32_t>(threadIdx.x);
  double acc[kRows];
#pragma unroll
  for (int r = 0; r < kRows; ++r) acc[r] = a + r == c ? 1.0 : 0.0;
  const double* multipliers = outer + outer_start[g];
  const int64_t u0 = u_start[g], u1 = u_start[g + 1];
  for (int64_t u = u0; u < u1; ++u) {
    const int32_t k = u_cols[u];
    const int32_t low = lo[k];
    if (c < low || c > k) continue;
    const double x = dense[base[k] + (c - low)];
    const double* column = multipliers + (u - u0) * rows;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      if (r < rows) {
        const double m = column[r];
        if (m != 0.0) acc[r] = __dsub_rn(acc[r], __dmul_rn(m, x));
      }
    }
  }
  const double* own = inner + inner_start[g];
#pragma unroll
  for (int kk = 0; kk + 1 < kRows; ++kk) {
    if (kk + 1 < rows) {
      const int32_t k = a + kk;
      if (c >= lo[k] && c <= k) {
        const double x = acc[kk];
#pragma unroll
        for (int r = kk + 1; r < kRows; ++r) {
          if (r < rows) {
            const double m = own[r * rows + kk];
            if (m != 0.0) acc[r] = __dsub_rn(acc[r], __dmul_rn(m, x));
          }
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    if (r < rows) {
      const int32_t i = a + r;
      if (c >= lo[i] && c <= i) dense[base[i] + (c - lo[i])] = acc[r];
    }
  }
}

// Device allocation released on scope exit.
template <typename T>
struct DeviceArray {
  T* ptr = nullptr;
  size_t size = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() {
    if (ptr != nullptr) cudaFree(ptr);
  }
  cudaError_t allocate(size_t count) {
    if (ptr != nullptr) cudaFree(ptr);
    ptr = nullptr;
    size = count;
    return cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T));
  }
  cudaError_t upload(const std::vector<T>& host, cudaStream_t stream) {
    if (cudaError_t e = allocate(host.size())) return e;
    if (host.empty()) return cudaSuccess;
    return cudaMemcpyAsync(ptr, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream);
  }
};

struct StreamGuard {
  cudaStream_t stream = nullptr;
  ~StreamGuard() {
    if (stream != nullptr) cudaStreamDestroy(stream);
  }
};

std::string cuda_error(const char* what, cudaError_t e) {
  return std::string("device factor build: ") + what + ": " + cudaGetErrorString(e);
}

#define PD_FD_CHECK(call, what)                   \
  do {                                            \
    const cudaError_t _e = (call);                \
    if (_e != cudaSuccess) return cuda_error(what, _e); \
  } while (0)

}  // namespace

std::string device_inverse_rows(const LowerFactorView& factor, InverseRows* out) {
  return g_device_rows_grouped.load() != 0 ? device_inverse_rows_grouped(factor, out)
                                           : device_inverse_rows_chunked(factor, out);
}

std::string device_inverse_rows_chunked(const LowerFactorView& factor, InverseRows* out) {
  const auto timer = PD_FT_NOW();
  const int32_t n = factor.size;
  out->start.assign(static_cast<size_t>(n) + 1, 0);
  out->columns.clear();
  out->values.clear();
  if (n == 0) return std::string();
  // Strict lower rows (the diagonal entry closing every row is dropped).
  std::vector<int64_t> lstart(static_cast<size_t>(n) + 1, 0);
  for (int32_t i = 0; i < n; ++i) lstart[i + 1] = lstart[i] + (factor.row_start[i + 1] - factor.row_start[i] - 1);
  std::vector<int32_t> lcols(static_cast<size_t>(lstart[n]));
  std::vector<double> lvals(static_cast<size_t>(lstart[n]));
  for (int32_t i = 0; i < n; ++i) {
    const int64_t from = factor.row_start[i];
    for (int64_t p = 0; p < lstart[i + 1] - lstart[i]; ++p) {
      lcols[lstart[i] + p] = factor.pattern[from + p];
      lvals[lstart[i] + p] = factor.values[from + p];
    }
  }
  // Levels, label ranges and chunks of every row.
  std::vector<int32_t> level(n, 0), lo(n);
  int32_t levels = 0;
  for (int32_t i = 0; i < n; ++i) {
    int32_t l = 0, low = i;
    for (int64_t p = lstart[i]; p < lstart[i + 1]; ++p) {
      const int32_t k = lcols[p];
      l = std::max(l, level[k] + 1);
      low = std::min(low, lo[k]);
    }
    level[i] = l;
    lo[i] = low;
    levels = std::max(levels, l + 1);
  }
  std::vector<int64_t> cb_base(n);
  int64_t cb_total = 0;
  for (int32_t i = 0; i < n; ++i) {
    cb_base[i] = cb_total;
    cb_total += (i / kChunk - lo[i] / kChunk) + 2;
  }
  std::vector<int32_t> level_count(static_cast<size_t>(levels) + 1, 0);
  for (int32_t i = 0; i < n; ++i) level_count[level[i] + 1] += 1;
  for (int32_t l = 0; l < levels; ++l) level_count[l + 1] += level_count[l];
  std::vector<int32_t> by_level(n);
  {
    std::vector<int32_t> cursor(level_count.begin(), level_count.end() - 1);
    for (int32_t i = 0; i < n; ++i) by_level[cursor[level[i]]++] = i;
  }
  std::vector<ChunkItem> items;
  std::vector<int64_t> level_items(static_cast<size_t>(levels) + 1, 0);
  int64_t scratch_max = 1;
  for (int32_t l = 0; l < levels; ++l) {
    int64_t slot = 0;
    for (int32_t r = level_count[l]; r < level_count[l + 1]; ++r) {
      const int32_t i = by_level[r];
      for (int32_t j = lo[i] / kChunk; j <= i / kChunk; ++j) {
        const int32_t c_begin = std::max(lo[i], j * kChunk);
        const int32_t c_end = std::min(i, (j + 1) * kChunk - 1) + 1;
        items.push_back(ChunkItem{i, j, slot});
        slot += c_end - c_begin;
      }
    }
    level_items[l + 1] = static_cast<int64_t>(items.size());
    scratch_max = std::max(scratch_max, slot);
  }
  int64_t items_max = 1;
  for (int32_t l = 0; l < levels; ++l) items_max = std::max(items_max, level_items[l + 1] - level_items[l]);

  StreamGuard guard;
  PD_FD_CHECK(cudaStreamCreateWithFlags(&guard.stream, cudaStreamNonBlocking), "stream");
  cudaStream_t stream = guard.stream;
  DeviceArray<int64_t> d_lstart, d_row_off, d_cb_base, d_placement;
  DeviceArray<int32_t> d_lcols, d_lo, d_cb, d_counts, d_scratch_cols;
  DeviceArray<double> d_lvals, d_scratch_vals;
  DeviceArray<ChunkItem> d_items;
  DeviceArray<int> d_error;
  PD_FD_CHECK(d_lstart.upload(lstart, stream), "upload");
  PD_FD_CHECK(d_lcols.upload(lcols, stream), "upload");
  PD_FD_CHECK(d_lvals.upload(lvals, stream), "upload");
  PD_FD_CHECK(d_lo.upload(lo, stream), "upload");
  PD_FD_CHECK(d_cb_base.upload(cb_base, stream), "upload");
  PD_FD_CHECK(d_items.upload(items, stream), "upload");
  PD_FD_CHECK(d_row_off.allocate(n), "allocate");
  PD_FD_CHECK(d_cb.allocate(static_cast<size_t>(cb_total)), "allocate");
  PD_FD_CHECK(d_counts.allocate(static_cast<size_t>(items_max)), "allocate");
  PD_FD_CHECK(d_placement.allocate(2 * static_cast<size_t>(items_max)), "allocate");
  PD_FD_CHECK(d_scratch_cols.allocate(static_cast<size_t>(scratch_max)), "allocate");
  PD_FD_CHECK(d_scratch_vals.allocate(static_cast<size_t>(scratch_max)), "allocate");
  PD_FD_CHECK(d_error.allocate(1), "allocate");
  PD_FD_CHECK(cudaMemsetAsync(d_error.ptr, 0, sizeof(int), stream), "memset");
  // The row pool grows by doubling; rows already stored move with it.
  DeviceArray<int32_t> pool_cols;
  DeviceArray<double> pool_vals;
  size_t capacity = std::max<size_t>(static_cast<size_t>(4 * lstart[n] + n), 1024);
  PD_FD_CHECK(pool_cols.allocate(capacity), "allocate pool");
  PD_FD_CHECK(pool_vals.allocate(capacity), "allocate pool");
  int64_t pool_size = 0;
  std::vector<int32_t> counts(static_cast<size_t>(items_max));
  std::vector<int64_t> placement(2 * static_cast<size_t>(items_max));
  for (int32_t l = 0; l < levels; ++l) {
    const int64_t first = level_items[l];
    const int32_t count = static_cast<int32_t>(level_items[l + 1] - first);
    inverse_rows_chunk_kernel<<<count, kThreads, 0, stream>>>(
        d_items.ptr + first, d_lstart.ptr, d_lcols.ptr, d_lvals.ptr, d_lo.ptr, d_row_off.ptr, d_cb_base.ptr, d_cb.ptr,
        pool_cols.ptr, pool_vals.ptr, d_scratch_cols.ptr, d_scratch_vals.ptr, d_counts.ptr, d_error.ptr);
    PD_FD_CHECK(cudaGetLastError(), "launch");
    PD_FD_CHECK(cudaMemcpyAsync(counts.data(), d_counts.ptr, count * sizeof(int32_t), cudaMemcpyDeviceToHost, stream),
                "counts");
    PD_FD_CHECK(cudaStreamSynchronize(stream), "level");
    int64_t row_base = pool_size;
    for (int32_t t = 0; t < count; ++t) {
      const ChunkItem& item = items[first + t];
      if (item.chunk == lo[item.row] / kChunk) row_base = pool_size;
      placement[2 * t] = pool_size;
      placement[2 * t + 1] = row_base;
      pool_size += counts[t];
    }
    if (static_cast<size_t>(pool_size) > capacity) {
      size_t grown = capacity;
      while (grown < static_cast<size_t>(pool_size)) grown *= 2;
      DeviceArray<int32_t> cols;
      DeviceArray<double> vals;
      PD_FD_CHECK(cols.allocate(grown), "grow pool");
      PD_FD_CHECK(vals.allocate(grown), "grow pool");
      const size_t used = static_cast<size_t>(placement[0]);
      if (used > 0) {
        PD_FD_CHECK(cudaMemcpyAsync(cols.ptr, pool_cols.ptr, used * sizeof(int32_t), cudaMemcpyDeviceToDevice, stream),
                    "grow pool");
        PD_FD_CHECK(cudaMemcpyAsync(vals.ptr, pool_vals.ptr, used * sizeof(double), cudaMemcpyDeviceToDevice, stream),
                    "grow pool");
      }
      PD_FD_CHECK(cudaStreamSynchronize(stream), "grow pool");
      std::swap(pool_cols.ptr, cols.ptr);
      std::swap(pool_vals.ptr, vals.ptr);
      pool_cols.size = grown;
      pool_vals.size = grown;
      capacity = grown;
    }
    PD_FD_CHECK(cudaMemcpyAsync(d_placement.ptr, placement.data(), 2 * count * sizeof(int64_t), cudaMemcpyHostToDevice,
                                stream),
                "placement");
    inverse_rows_copy_kernel<<<count, kThreads, 0, stream>>>(d_items.ptr + first, d_counts.ptr, d_placement.ptr,
                                                             d_lo.ptr, d_cb_base.ptr, d_cb.ptr, d_row_off.ptr,
                                                             d_scratch_cols.ptr, d_scratch_vals.ptr, pool_cols.ptr,
                                                             pool_vals.ptr);
    PD_FD_CHECK(cudaGetLastError(), "launch");
  }
  int error = 0;
  std::vector<int64_t> row_off(n);
  std::vector<int32_t> cb(static_cast<size_t>(cb_total));
  std::vector<int32_t> pool_c(static_cast<size_t>(pool_size));
  std::vector<double> pool_v(static_cast<size_t>(pool_size));
  PD_FD_CHECK(cudaMemcpyAsync(&error, d_error.ptr, sizeof(int), cudaMemcpyDeviceToHost, stream), "read back");
  PD_FD_CHECK(cudaMemcpyAsync(row_off.data(), d_row_off.ptr, n * sizeof(int64_t), cudaMemcpyDeviceToHost, stream),
              "read back");
  if (cb_total > 0) {
    PD_FD_CHECK(cudaMemcpyAsync(cb.data(), d_cb.ptr, cb.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, stream),
                "read back");
  }
  if (pool_size > 0) {
    PD_FD_CHECK(cudaMemcpyAsync(pool_c.data(), pool_cols.ptr, pool_c.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                stream),
                "read back");
    PD_FD_CHECK(cudaMemcpyAsync(pool_v.data(), pool_vals.ptr, pool_v.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                stream),
                "read back");
  }
  PD_FD_CHECK(cudaStreamSynchronize(stream), "read back");
  if (error != 0) return "device inverse rows: an entry fell outside its chunk";
  // Rows in elimination order.
  for (int32_t i = 0; i < n; ++i) {
    const int64_t length = cb[cb_base[i] + (i / kChunk - lo[i] / kChunk) + 1];
    out->start[i + 1] = out->start[i] + length;
  }
  out->columns.resize(static_cast<size_t>(out->start[n]));
  out->values.resize(static_cast<size_t>(out->start[n]));
  for (int32_t i = 0; i < n; ++i) {
    const int64_t length = out->start[i + 1] - out->start[i];
    std::copy(pool_c.begin() + row_off[i], pool_c.begin() + row_off[i] + length, out->columns.begin() + out->start[i]);
    std::copy(pool_v.begin() + row_off[i], pool_v.begin() + row_off[i] + length, out->values.begin() + out->start[i]);
  }
  PD_FT_REPORT("inverse rows", timer, std::string("levels ") + std::to_string(levels) + " items " +
                                         std::to_string(items.size()) + " nnz " + std::to_string(out->start[n]));
  return std::string();
}

std::string device_ldlt(const SymbolicView& symbolic, double* values, double* diagonal) {
  const auto timer = PD_FT_NOW();
  const int32_t n = symbolic.size;
  if (n == 0) return std::string();
  const int64_t nnz = symbolic.row_start[n];
  const int64_t col_nnz = symbolic.col_start[n];
  std::vector<int32_t> level(n, 0);
  int32_t levels = 0;
  int64_t longest = 0;
  for (int32_t i = 0; i < n; ++i) {
    const int64_t strict = symbolic.row_start[i + 1] - 1 - symbolic.row_start[i];
    longest = std::max(longest, strict);
    if (strict > kLdltMaxPattern) {
      PD_FT_REPORT("ldlt fallback", timer, std::string("row length ") + std::to_string(strict));
      return "device LDLT: a row of L has " + std::to_string(strict) + " entries (at most " +
             std::to_string(kLdltMaxPattern) + " are staged)";
    }
    int32_t l = 0;
    for (int64_t p = symbolic.row_start[i]; p < symbolic.row_start[i + 1] - 1; ++p)
      l = std::max(l, level[symbolic.pattern[p]] + 1);
    level[i] = l;
    levels = std::max(levels, l + 1);
  }
  // Work items level by level: every column split into groups of kThreads entries.
  std::vector<std::vector<int32_t>> columns_of(levels);
  for (int32_t j = 0; j < n; ++j) columns_of[level[j]].push_back(j);
  std::vector<ColumnItem> items;
  std::vector<int64_t> level_items(static_cast<size_t>(levels) + 1, 0);
  std::vector<int64_t> level_longest(levels, 0);
  for (int32_t l = 0; l < levels; ++l) {
    for (int32_t j : columns_of[l]) {
      const int32_t count = static_cast<int32_t>(symbolic.col_start[j + 1] - symbolic.col_start[j]) + 1;
      for (int32_t first = 0; first < count; first += kThreads) items.push_back(ColumnItem{j, first});
      level_longest[l] = std::max(level_longest[l], symbolic.row_start[j + 1] - 1 - symbolic.row_start[j]);
    }
    level_items[l + 1] = static_cast<int64_t>(items.size());
  }
  StreamGuard guard;
  PD_FD_CHECK(cudaStreamCreateWithFlags(&guard.stream, cudaStreamNonBlocking), "stream");
  cudaStream_t stream = guard.stream;
  DeviceArray<int64_t> d_row_start, d_col_start, d_col_pos;
  DeviceArray<int32_t> d_pattern, d_col_rows;
  DeviceArray<double> d_initial, d_multipliers, d_unscaled, d_diagonal;
  DeviceArray<ColumnItem> d_items;
  DeviceArray<int> d_fail;
  auto upload = [&](auto& array, const auto* host, size_t count) {
    cudaError_t e = array.allocate(count);
    if (e == cudaSuccess && count > 0)
      e = cudaMemcpyAsync(array.ptr, host, count * sizeof(*host), cudaMemcpyHostToDevice, stream);
    return e;
  };
  PD_FD_CHECK(upload(d_row_start, symbolic.row_start, static_cast<size_t>(n) + 1), "upload");
  PD_FD_CHECK(upload(d_pattern, symbolic.pattern, static_cast<size_t>(nnz)), "upload");
  PD_FD_CHECK(upload(d_col_start, symbolic.col_start, static_cast<size_t>(n) + 1), "upload");
  PD_FD_CHECK(upload(d_col_rows, symbolic.col_rows, static_cast<size_t>(col_nnz)), "upload");
  PD_FD_CHECK(upload(d_col_pos, symbolic.col_pos, static_cast<size_t>(col_nnz)), "upload");
  PD_FD_CHECK(upload(d_initial, values, static_cast<size_t>(nnz)), "upload");
  PD_FD_CHECK(upload(d_items, items.data(), items.size()), "upload");
  PD_FD_CHECK(d_multipliers.allocate(static_cast<size_t>(nnz)), "allocate");
  PD_FD_CHECK(d_unscaled.allocate(static_cast<size_t>(nnz)), "allocate");
  PD_FD_CHECK(d_diagonal.allocate(n), "allocate");
  PD_FD_CHECK(d_fail.allocate(1), "allocate");
  PD_FD_CHECK(cudaMemcpyAsync(d_fail.ptr, &n, sizeof(int), cudaMemcpyHostToDevice, stream), "upload");
  const size_t smem_max = static_cast<size_t>(longest) * (sizeof(double) + sizeof(int32_t));
  PD_FD_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(&ldlt_columns_kernel),
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(std::max<size_t>(smem_max, 1))),
              "shared memory");
  // Levels in order on one stream: a level's columns read only columns of lower levels.
  for (int32_t l = 0; l < levels; ++l) {
    const int64_t first = level_items[l];
    const int32_t count = static_cast<int32_t>(level_items[l + 1] - first);
    const size_t smem = static_cast<size_t>(level_longest[l]) * (sizeof(double) + sizeof(int32_t));
    ldlt_columns_kernel<<<count, kThreads, smem, stream>>>(d_items.ptr + first, d_row_start.ptr, d_pattern.ptr,
                                                           d_col_start.ptr, d_col_rows.ptr, d_col_pos.ptr,
                                                           d_initial.ptr, d_multipliers.ptr, d_unscaled.ptr,
                                                           d_diagonal.ptr, d_fail.ptr);
    PD_FD_CHECK(cudaGetLastError(), "launch");
    ldlt_divide_kernel<<<count, kThreads, 0, stream>>>(d_items.ptr + first, d_col_start.ptr, d_col_pos.ptr,
                                                       d_unscaled.ptr, d_diagonal.ptr, d_multipliers.ptr);
    PD_FD_CHECK(cudaGetLastError(), "launch");
  }
  int fail = n;
  std::vector<double> multipliers(static_cast<size_t>(nnz)), pivots(n);
  PD_FD_CHECK(cudaMemcpyAsync(&fail, d_fail.ptr, sizeof(int), cudaMemcpyDeviceToHost, stream), "read back");
  PD_FD_CHECK(cudaMemcpyAsync(multipliers.data(), d_multipliers.ptr, multipliers.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, stream),
              "read back");
  PD_FD_CHECK(cudaMemcpyAsync(pivots.data(), d_diagonal.ptr, pivots.size() * sizeof(double), cudaMemcpyDeviceToHost,
                              stream),
              "read back");
  PD_FD_CHECK(cudaStreamSynchronize(stream), "read back");
  if (fail < n) {
    return "matrix is not positive definite: LDLT pivot " + std::to_string(fail) + " is " +
           std::to_string(pivots[fail]);
  }
  for (int32_t i = 0; i < n; ++i) {
    for (int64_t p = symbolic.row_start[i]; p < symbolic.row_start[i + 1] - 1; ++p) values[p] = multipliers[p];
    values[symbolic.row_start[i + 1] - 1] = pivots[i];
    diagonal[i] = pivots[i];
  }
  PD_FT_REPORT("ldlt", timer, std::string("levels ") + std::to_string(levels) + " items " +
                                  std::to_string(items.size()));
  return std::string();
}


// The grouped dense rows of L^{-1} on the current device: the host plans the
// groups (plan_row_groups), every level's items launch back to back on one
// stream (no host round trip between levels: every row has its place in the
// dense array from the start), and the host compacts the dense rows. An
// order whose dense rows would be too large uses the chunked rows instead.
std::string device_inverse_rows_grouped(const LowerFactorView& factor, InverseRows* out) {
  if (factor.size == 0) {
    out->start.assign(1, 0);
    out->columns.clear();
    out->values.clear();
    return std::string();
  }
  RowGroups plan;
  if (!plan_row_groups(factor, &plan)) return device_inverse_rows_chunked(factor, out);
  const int32_t n = factor.size;
  const int32_t levels = static_cast<int32_t>(plan.level_start.size()) - 1;
  std::vector<int2> items;
  std::vector<int64_t> level_items(static_cast<size_t>(levels) + 1, 0);
  for (int32_t l = 0; l < levels; ++l) {
    for (int32_t q = plan.level_start[l]; q < plan.level_start[l + 1]; ++q) {
      const int32_t g = plan.groups_by_level[q];
      for (int32_t j = plan.group_lo[g] / kRowGroupChunk; j <= (plan.group_start[g + 1] - 1) / kRowGroupChunk; ++j)
        items.push_back(make_int2(g, j));
    }
    level_items[l + 1] = static_cast<int64_t>(items.size());
  }
  StreamGuard guard;
  PD_FD_CHECK(cudaStreamCreateWithFlags(&guard.stream, cudaStreamNonBlocking), "stream");
  cudaStream_t stream = guard.stream;
  DeviceArray<int2> d_items;
  DeviceArray<int32_t> d_group_start, d_u_cols, d_lo;
  DeviceArray<int64_t> d_u_start, d_outer_start, d_inner_start, d_base;
  DeviceArray<double> d_outer, d_inner, d_dense;
  PD_FD_CHECK(d_items.upload(items, stream), "upload");
  PD_FD_CHECK(d_group_start.upload(plan.group_start, stream), "upload");
  PD_FD_CHECK(d_u_cols.upload(plan.u_cols, stream), "upload");
  PD_FD_CHECK(d_lo.upload(plan.lo, stream), "upload");
  PD_FD_CHECK(d_u_start.upload(plan.u_start, stream), "upload");
  PD_FD_CHECK(d_outer_start.upload(plan.outer_start, stream), "upload");
  PD_FD_CHECK(d_inner_start.upload(plan.inner_start, stream), "upload");
  PD_FD_CHECK(d_base.upload(plan.base, stream), "upload");
  PD_FD_CHECK(d_outer.upload(plan.outer, stream), "upload");
  PD_FD_CHECK(d_inner.upload(plan.inner, stream), "upload");
  const size_t slots = static_cast<size_t>(plan.base[n]);
  PD_FD_CHECK(d_dense.allocate(slots), "allocate dense rows");
  for (int32_t l = 0; l < levels; ++l) {
    const int64_t first = level_items[l];
    const int64_t count = level_items[l + 1] - first;
    if (count == 0) continue;
    inverse_rows_group_kernel<kRowGroupRows><<<static_cast<unsigned>(count), kRowGroupChunk, 0, stream>>>(
        d_items.ptr + first, d_group_start.ptr, d_u_start.ptr, d_u_cols.ptr, d_outer_start.ptr, d_outer.ptr,
        d_inner_start.ptr, d_inner.ptr, d_lo.ptr, d_base.ptr, d_dense.ptr);
    PD_FD_CHECK(cudaGetLastError(), "launch");
  }
  std::vector<double> dense(slots);
  if (slots > 0) {
    PD_FD_CHECK(cudaMemcpyAsync(dense.data(), d_dense.ptr, slots * sizeof(double), cudaMemcpyDeviceToHost, stream),
                "read back");
  }
  PD_FD_CHECK(cudaStreamSynchronize(stream), "rows of L^-1");
  compact_dense_rows(plan, dense.data(), out);
  return std::string();
}

}  // namespace pdb200
