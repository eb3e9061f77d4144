// Host construction of the exact inverse factor A^{-1} = S^T S.
//
// The algorithm and its floating-point evaluation order follow the reference
// setup in src/newton_solver_diff_phd/_src/solvers/diff_phd/sparse.py, so the
// CSR arrays are bit-identical to the reference's for the same input rows.
// The data structures are this file's own: index arrays, marker stamps and
// an elimination-tree symbolic phase instead of Python sets and dictionaries.
// Compile without floating-point contraction (-ffp-contract=off): every
// update must round the product before the subtraction, as NumPy does.
#include "factor.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

namespace pdb200 {

// Rows of L^{-1} whose update work (entries of the earlier rows they
// combine) reaches this are split over host threads.
std::atomic<int64_t> g_parallel_row_work{1 << 16};

// Factors with at least this many entries of L take the numeric LDL^T and the
// rows of L^{-1} over host threads level by level (bit-identical).
std::atomic<int64_t> g_parallel_level_entries{int64_t{1} << 15};
std::atomic<int32_t> g_device_rows_grouped{0};

namespace {

// A fixed set of worker threads that run one task per worker and wait for
// all of them (one row of the inverse at a time).
class RowPool {
 public:
  explicit RowPool(unsigned workers) {
    for (unsigned w = 1; w < workers; ++w) threads_.emplace_back([this, w] { loop(w); });
    count_ = workers;
  }
  ~RowPool() {
    {
      std::lock_guard<std::mutex> lock(mutex_);
      stop_ = true;
      ++generation_;
    }
    wake_.notify_all();
    for (auto& t : threads_) t.join();
  }
  unsigned size() const { return count_; }
  // Runs task(w) for w = 0 .. size()-1, worker 0 on the calling thread.
  void run(const std::function<void(unsigned)>& task) {
    {
      std::lock_guard<std::mutex> lock(mutex_);
      task_ = &task;
      pending_ = count_ - 1;
      ++generation_;
    }
    wake_.notify_all();
    task(0);
    std::unique_lock<std::mutex> lock(mutex_);
    done_.wait(lock, [this] { return pending_ == 0; });
  }

 private:
  void loop(unsigned w) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(unsigned)>* task;
      {
        std::unique_lock<std::mutex> lock(mutex_);
        wake_.wait(lock, [&] { return generation_ != seen; });
        seen = generation_;
        if (stop_) return;
        task = task_;
      }
      (*task)(w);
      {
        std::lock_guard<std::mutex> lock(mutex_);
        if (--pending_ == 0) done_.notify_one();
      }
    }
  }
  std::vector<std::thread> threads_;
  std::mutex mutex_;
  std::condition_variable wake_, done_;
  const std::function<void(unsigned)>* task_ = nullptr;
  uint64_t generation_ = 0;
  unsigned pending_ = 0, count_ = 1;
  bool stop_ = false;
};

using Adjacency = std::vector<std::vector<int32_t>>;

// Minimum-degree elimination order of the subgraph induced by `vertices`
// (sparse.py:18-28): repeatedly remove the vertex of smallest (degree, index)
// and join its remaining neighbours into a clique.
std::vector<int32_t> minimum_degree(const std::vector<int32_t>& vertices, const Adjacency& adjacency,
                                    std::vector<int32_t>& local) {
  const int32_t m = static_cast<int32_t>(vertices.size());
  for (int32_t a = 0; a < m; ++a) local[vertices[a]] = a;
  std::vector<std::vector<int32_t>> graph(m);
  for (int32_t a = 0; a < m; ++a) {
    for (int32_t other : adjacency[vertices[a]]) {
      const int32_t b = local[other];
      if (b >= 0 && b < m && vertices[b] == other) graph[a].push_back(b);
    }
    std::sort(graph[a].begin(), graph[a].end());
  }
  std::vector<char> alive(m, 1);
  std::vector<int32_t> order;
  order.reserve(m);
  std::vector<int32_t> merged;
  for (int32_t step = 0; step < m; ++step) {
    int32_t best = -1;
    size_t best_degree = 0;
    // Local ids follow ascending vertex ids (vertices is sorted), so the
    // first minimum of the scan breaks ties by the smallest index.
    for (int32_t a = 0; a < m; ++a) {
      if (!alive[a]) continue;
      if (best < 0 || graph[a].size() < best_degree) {
        best = a;
        best_degree = graph[a].size();
      }
    }
    alive[best] = 0;
    order.push_back(vertices[best]);
    const std::vector<int32_t> neighbors = graph[best];
    for (int32_t other : neighbors) {
      std::vector<int32_t>& list = graph[other];
      merged.clear();
      std::set_union(list.begin(), list.end(), neighbors.begin(), neighbors.end(), std::back_inserter(merged));
      list.clear();
      for (int32_t value : merged) {
        if (value != other && value != best) list.push_back(value);
      }
    }
    graph[best].clear();
  }
  for (int32_t v : vertices) local[v] = -1;
  return order;
}

struct Dissection {
  const Adjacency& adjacency;
  std::vector<int32_t> stamp;     // membership token per vertex
  std::vector<int32_t> distance;  // BFS distance per vertex
  std::vector<int32_t> local;     // scratch map for minimum_degree
  int32_t token = 0;

  explicit Dissection(const Adjacency& graph)
      : adjacency(graph), stamp(graph.size(), -1), distance(graph.size(), -1), local(graph.size(), -1) {}

  // Breadth-first distances from `start` inside the current token's set,
  // visiting neighbours in ascending order (sparse.py:31-40). Returns the
  // reached vertices in discovery order.
  std::vector<int32_t> bfs(int32_t start, int32_t set_token) {
    std::vector<int32_t> queue;
    queue.push_back(start);
    distance[start] = 0;
    stamp[start] = set_token + 1;  // reached marker
    for (size_t head = 0; head < queue.size(); ++head) {
      const int32_t node = queue[head];
      for (int32_t other : adjacency[node]) {
        if (stamp[other] == set_token) {
          stamp[other] = set_token + 1;
          distance[other] = distance[node] + 1;
          queue.push_back(other);
        }
      }
    }
    return queue;
  }

  int32_t new_token(const std::vector<int32_t>& vertices) {
    token += 2;
    for (int32_t v : vertices) stamp[v] = token;
    return token;
  }

  void visit(std::vector<int32_t> vertices, std::vector<int32_t>& order) {
    std::sort(vertices.begin(), vertices.end());
    if (vertices.size() <= 24) {
      const std::vector<int32_t> leaf = minimum_degree(vertices, adjacency, local);
      order.insert(order.end(), leaf.begin(), leaf.end());
      return;
    }
    int32_t set_token = new_token(vertices);
    // Start at the smallest (degree inside the set, index) (sparse.py:47).
    int32_t start = -1;
    size_t start_degree = 0;
    for (int32_t v : vertices) {
      size_t degree = 0;
      for (int32_t other : adjacency[v]) degree += stamp[other] == set_token;
      if (start < 0 || degree < start_degree) {
        start = v;
        start_degree = degree;
      }
    }
    std::vector<int32_t> reached = bfs(start, set_token);
    if (reached.size() != vertices.size()) {
      // Components in order: the start's, then by smallest remaining index.
      std::vector<std::vector<int32_t>> components;
      components.push_back(reached);
      for (int32_t v : vertices) {
        if (stamp[v] == set_token) components.push_back(bfs(v, set_token));
      }
      for (auto& component : components) visit(component, order);
      return;
    }
    // Farthest vertex: largest distance, smallest index on ties (sparse.py:57).
    int32_t farthest = -1;
    for (int32_t v : vertices) {
      if (farthest < 0 || distance[v] > distance[farthest]) farthest = v;
    }
    set_token = new_token(vertices);
    bfs(farthest, set_token);
    int32_t levels_count = 0;
    for (int32_t v : vertices) levels_count = std::max(levels_count, distance[v] + 1);
    std::vector<int64_t> cumulative(levels_count, 0);
    for (int32_t v : vertices) cumulative[distance[v]] += 1;
    for (int32_t l = 1; l < levels_count; ++l) cumulative[l] += cumulative[l - 1];
    // np.searchsorted(cumsum, n / 2) with side='left'.
    const double half = static_cast<double>(vertices.size()) / 2.0;
    int32_t cut = levels_count;
    for (int32_t l = 0; l < levels_count; ++l) {
      if (static_cast<double>(cumulative[l]) >= half) {
        cut = l;
        break;
      }
    }
    std::vector<int32_t> lower, upper, separator;
    for (int32_t v : vertices) {
      if (distance[v] < cut) {
        lower.push_back(v);
      } else if (distance[v] > cut) {
        upper.push_back(v);
      } else {
        separator.push_back(v);
      }
    }
    if (lower.empty() || upper.empty()) {
      const std::vector<int32_t> all = minimum_degree(vertices, adjacency, local);
      order.insert(order.end(), all.begin(), all.end());
      return;
    }
    visit(lower, order);
    visit(upper, order);
    const std::vector<int32_t> last = minimum_degree(separator, adjacency, local);
    order.insert(order.end(), last.begin(), last.end());
  }
};

}  // namespace

std::vector<int32_t> nested_dissection(const Adjacency& adjacency) {
  Dissection dissection(adjacency);
  std::vector<int32_t> all(adjacency.size());
  std::iota(all.begin(), all.end(), 0);
  std::vector<int32_t> order;
  order.reserve(adjacency.size());
  dissection.visit(all, order);
  return order;
}

// The numeric LDL^T as left-looking columns over host threads, for large
// factors. Entry (i, j) is the permuted A value minus m(i, k) e(j, k) over the
// columns k < j that rows i and j share, in ascending k: the sequence of
// rounded products and subtractions the right-looking update applies to it,
// so the factor is bit-identical. Columns are processed level by level of the
// elimination tree (a column reads only columns of lower levels); within a
// level every entry is independent, so the top of the tree, one column per
// level, is split over the threads entry by entry. `values` holds the lower
// triangle of A at the row positions on entry and the multipliers (strict
// positions) and pivots (diagonal positions) on return; the caller checks the
// pivots in elimination order.
void ldlt_left_looking(int32_t size, const std::vector<int64_t>& row_start, const std::vector<int32_t>& pattern,
                       const std::vector<std::vector<int32_t>>& columns,
                       const std::vector<std::vector<int64_t>>& column_positions, std::vector<double>& values,
                       std::vector<double>& diagonal, RowPool& pool) {
  std::vector<int32_t> level(size, 0);
  int32_t levels = 0;
  for (int32_t i = 0; i < size; ++i) {
    int32_t l = 0;
    for (int64_t p = row_start[i]; p < row_start[i + 1] - 1; ++p) l = std::max(l, level[pattern[p]] + 1);
    level[i] = l;
    levels = std::max(levels, l + 1);
  }
  std::vector<int32_t> level_count(static_cast<size_t>(levels) + 1, 0);
  for (int32_t j = 0; j < size; ++j) level_count[level[j] + 1] += 1;
  for (int32_t l = 0; l < levels; ++l) level_count[l + 1] += level_count[l];
  std::vector<int32_t> by_level(size);
  {
    std::vector<int32_t> cursor(level_count.begin(), level_count.end() - 1);
    for (int32_t j = 0; j < size; ++j) by_level[cursor[level[j]]++] = j;
  }
  std::vector<double> unscaled(values.size(), 0.0);
  std::vector<int64_t> first_entry;  // per column of the level: its first flat entry
  const unsigned workers = pool.size();
  // Levels of at most kDenseColumns columns with at least kDenseEntries
  // entries (the top of the tree) scatter each column's row j into a dense
  // array over the labels, so an entry (i, j) walks row i alone: its columns
  // k < j that row j lacks read a zero, and subtracting a signed zero leaves
  // every nonzero value unchanged (an entry that is exactly zero may change
  // the sign of its zero; zero multipliers are skipped by the rows of L^{-1}).
  // Such a column k may sit at this level or above, where row i still holds
  // A(i, k): a finite value times zero (`values` is written only by the
  // division pass that follows each level's entry pass).
  // The dense arrays take at most 2^24 doubles.
  const int32_t kDenseColumns =
      static_cast<int32_t>(std::min<int64_t>(64, std::max<int64_t>(1, (int64_t{1} << 24) / std::max(size, 1))));
  constexpr int64_t kDenseEntries = 256;
  std::vector<double> dense_rows;
  std::vector<int32_t> dense_slot(size, -1);
  for (int32_t l = 0; l < levels; ++l) {
    const int32_t c0 = level_count[l], c1 = level_count[l + 1];
    first_entry.assign(1, 0);
    for (int32_t c = c0; c < c1; ++c)
      first_entry.push_back(first_entry.back() + static_cast<int64_t>(columns[by_level[c]].size()) + 1);
    const int64_t total = first_entry.back();
    const bool dense = c1 - c0 <= kDenseColumns && total >= kDenseEntries;
    auto scatter_rows = [&](bool clear) {
      for (int32_t c = c0; c < c1; ++c) {
        const int32_t j = by_level[c];
        double* row = dense_rows.data() + static_cast<size_t>(c - c0) * size;
        dense_slot[j] = c - c0;
        for (int64_t q = row_start[j]; q < row_start[j + 1] - 1; ++q) row[pattern[q]] = clear ? 0.0 : unscaled[q];
      }
    };
    if (dense) {
      if (dense_rows.empty()) dense_rows.assign(static_cast<size_t>(kDenseColumns) * size, 0.0);
      scatter_rows(false);
    }
    const int64_t chunk = std::max<int64_t>(16, total / (4 * static_cast<int64_t>(workers)) + 1);
    // Entry e of the level's c-th column: 0 is the diagonal, e >= 1 row columns[j][e - 1].
    auto for_entries = [&](const std::function<void(int32_t, int64_t)>& body) {
      std::atomic<int64_t> next{0};
      auto run = [&](unsigned) {
        for (int64_t lo = next.fetch_add(chunk); lo < total; lo = next.fetch_add(chunk)) {
          const int64_t hi = std::min(total, lo + chunk);
          int64_t c = std::upper_bound(first_entry.begin(), first_entry.end(), lo) - first_entry.begin() - 1;
          for (int64_t f = lo; f < hi; ++f) {
            while (f >= first_entry[c + 1]) ++c;
            body(by_level[c0 + c], f - first_entry[c]);
          }
        }
      };
      if (total <= chunk) {
        run(0);
      } else {
        pool.run(run);
      }
    };
    for_entries([&](int32_t j, int64_t e) {
      const int64_t start_j = row_start[j];
      const int64_t end_j = row_start[j + 1] - 1;  // the diagonal position of row j
      if (e == 0) {
        double acc = values[end_j];
        for (int64_t q = start_j; q < end_j; ++q) {
          const double product = values[q] * unscaled[q];
          acc = acc - product;
        }
        unscaled[end_j] = acc;
        return;
      }
      if (dense) {
        // Entries 1 + 4 m .. 4 + 4 m of the column are computed together by
        // the task of the first: four independent chains side by side, each
        // in its own order.
        if ((e - 1) % 4 != 0) return;
        const double* row_j = dense_rows.data() + static_cast<size_t>(dense_slot[j]) * size;
        const int64_t count = std::min<int64_t>(4, static_cast<int64_t>(columns[j].size()) - (e - 1));
        int64_t p[4] = {0, 0, 0, 0}, end[4] = {0, 0, 0, 0};
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        int64_t common = std::numeric_limits<int64_t>::max();
        for (int64_t t = 0; t < count; ++t) {
          end[t] = column_positions[j][e - 1 + t];
          p[t] = row_start[columns[j][e - 1 + t]];
          acc[t] = values[end[t]];
          common = std::min(common, end[t] - p[t]);
        }
        if (count == 4) {
          for (int64_t q = 0; q < common; ++q) {
            for (int t = 0; t < 4; ++t) {
              const double product = values[p[t] + q] * row_j[pattern[p[t] + q]];
              acc[t] = acc[t] - product;
            }
          }
          for (int t = 0; t < 4; ++t) p[t] += common;
        }
        for (int64_t t = 0; t < count; ++t) {
          for (int64_t q = p[t]; q < end[t]; ++q) {
            const double product = values[q] * row_j[pattern[q]];
            acc[t] = acc[t] - product;
          }
          unscaled[end[t]] = acc[t];
        }
        return;
      }
      const int32_t i = columns[j][e - 1];
      const int64_t pos = column_positions[j][e - 1];
      double acc = values[pos];
      int64_t p = row_start[i];
      int64_t q = start_j;
      while (p < pos && q < end_j) {
        const int32_t a = pattern[p];
        const int32_t b = pattern[q];
        if (a < b) {
          ++p;
        } else if (b < a) {
          ++q;
        } else {
          const double product = values[p] * unscaled[q];
          acc = acc - product;
          ++p;
          ++q;
        }
      }
      unscaled[pos] = acc;
    });
    for_entries([&](int32_t j, int64_t e) {
      const int64_t end_j = row_start[j + 1] - 1;
      if (e == 0) {
        diagonal[j] = unscaled[end_j];
        values[end_j] = unscaled[end_j];
        return;
      }
      const int64_t pos = column_positions[j][e - 1];
      values[pos] = unscaled[pos] / unscaled[end_j];
    });
    if (dense) scatter_rows(true);
  }
}

// dst[u] = dst[u] - coefficient * src[u] over `count` entries: one rounded
// multiply, then one rounded subtract per entry (no contraction), so every
// entry sees the host walk's operations; lanes are independent, so vector
// code gives the same bits. Compiled for AVX2 and the baseline, chosen at
// load time.
__attribute__((target_clones("avx2", "default"))) static void subtract_scaled(double* __restrict dst,
                                                                       const double* __restrict src,
                                                                       double coefficient, int32_t count) {
  for (int32_t u = 0; u < count; ++u) {
    const double product = coefficient * src[u];
    dst[u] = dst[u] - product;
  }
}

// dst[u] = (((dst[u] - m0 x0[u]) - m1 x1[u]) - m2 x2[u]) - m3 x3[u]: four
// updates of each entry in order, every product and difference rounded.
__attribute__((target_clones("avx2", "default"))) static void subtract_scaled4(
    double* __restrict dst, const double* __restrict x0, const double* __restrict x1, const double* __restrict x2,
    const double* __restrict x3, const double* m, int32_t count) {
  const double m0 = m[0], m1 = m[1], m2 = m[2], m3 = m[3];
  for (int32_t u = 0; u < count; ++u) {
    double value = dst[u];
    const double p0 = m0 * x0[u];
    value = value - p0;
    const double p1 = m1 * x1[u];
    value = value - p1;
    const double p2 = m2 * x2[u];
    value = value - p2;
    const double p3 = m3 * x3[u];
    dst[u] = value - p3;
  }
}

// Rows of L^{-1} over host threads in groups of consecutive rows. Row i of
// L^{-1} is nonzero only on the labels [lo_i, i] of its elimination subtree
// (lo_i = min(i, lo_k over its columns k)); with the nested-dissection order
// that range is almost fully dense, so rows are stored as dense segments and
// row i's update by row k is a contiguous subtract over row k's range, which
// lies inside row i's. Rows that share most of their columns form a group
// (up to kRowGroupRows consecutive rows): per column chunk of kRowGroupChunk
// labels the group applies each outside column k (k below the group's first
// row, in ascending order) to all its rows that hold it, so row k's chunk is
// read once for the group, then its own rows in ascending order. Each entry
// of a row therefore sees its columns k in ascending order, one multiply and
// one subtract each, and zero multipliers are skipped as in the walk; updates
// by row k's exact zeros subtract signed zeros, which leave every nonzero
// value unchanged, and exact zeros are omitted at the end: the rows are
// bit-identical to the walk's. Groups are scheduled level by level (a group
// reads only groups of lower levels) as (group, chunk) tasks.
bool plan_row_groups(const LowerFactorView& f, RowGroups* plan) {
  constexpr double kShare = 0.5;  // a row joins when half its outside columns are the group's
  const int32_t n = f.size;
  if (n == 0) {
    *plan = RowGroups();
    plan->base.assign(1, 0);
    plan->group_start.assign(1, 0);
    plan->u_start.assign(1, 0);
    plan->outer_start.assign(1, 0);
    plan->inner_start.assign(1, 0);
    plan->level_start.assign(1, 0);
    return true;
  }
  std::vector<int32_t>& lo = plan->lo;
  lo.assign(n, 0);
  std::vector<int32_t> parent(n, -1);
  std::vector<int64_t> subtree(n, 1);
  for (int32_t i = 0; i < n; ++i) {
    int32_t low = i;
    for (int64_t p = f.row_start[i]; p < f.row_start[i + 1] - 1; ++p) {
      const int32_t k = f.pattern[p];
      low = std::min(low, lo[k]);
      if (parent[k] < 0) parent[k] = i;
    }
    lo[i] = low;
  }
  int64_t structural = 0;
  for (int32_t k = 0; k < n; ++k) {
    structural += subtree[k];
    if (parent[k] >= 0) subtree[parent[k]] += subtree[k];
  }
  std::vector<int64_t>& base = plan->base;
  base.assign(static_cast<size_t>(n) + 1, 0);
  for (int32_t i = 0; i < n; ++i) base[i + 1] = base[i] + (i - lo[i] + 1);
  if (base[n] > 2 * structural) return false;

  // Groups of consecutive rows.
  std::vector<int32_t>& group_start = plan->group_start;
  std::vector<int32_t> group_of(n);
  group_start.assign(1, 0);
  {
    std::vector<int32_t> mark(n, -1);
    int32_t a = 0;
    for (int32_t r = 0; r < n; ++r) {
      if (r > a) {
        int32_t outside = 0, shared = 0;
        for (int64_t p = f.row_start[r]; p < f.row_start[r + 1] - 1; ++p) {
          const int32_t k = f.pattern[p];
          if (k < a) {
            ++outside;
            shared += mark[k] == a;
          }
        }
        if (r - a >= kRowGroupRows || shared < kShare * outside) {
          a = r;
          group_start.push_back(r);
        }
      }
      for (int64_t p = f.row_start[r]; p < f.row_start[r + 1] - 1; ++p) {
        const int32_t k = f.pattern[p];
        if (k < a) mark[k] = a;
      }
      group_of[r] = static_cast<int32_t>(group_start.size()) - 1;
    }
    group_start.push_back(n);
  }
  const int32_t groups = static_cast<int32_t>(group_start.size()) - 1;
  plan->u_start.assign(static_cast<size_t>(groups) + 1, 0);
  plan->outer_start.assign(static_cast<size_t>(groups) + 1, 0);
  plan->inner_start.assign(static_cast<size_t>(groups) + 1, 0);
  plan->group_lo.assign(groups, 0);
  plan->u_cols.clear();
  plan->outer.clear();
  plan->inner.clear();
  std::vector<int32_t>& u_cols = plan->u_cols;
  std::vector<double>& outer = plan->outer;
  std::vector<double>& inner = plan->inner;
  std::vector<int32_t> level(groups, 0);
  int32_t levels = 0;
  {
    std::vector<int32_t> seen(n, -1);
    for (int32_t g = 0; g < groups; ++g) {
      const int32_t a = group_start[g], b = group_start[g + 1], rows = b - a;
      const size_t u0 = u_cols.size();
      int32_t low = a;
      for (int32_t r = a; r < b; ++r) {
        low = std::min(low, lo[r]);
        for (int64_t p = f.row_start[r]; p < f.row_start[r + 1] - 1; ++p) {
          const int32_t k = f.pattern[p];
          if (k < a && seen[k] != g) {
            seen[k] = g;
            u_cols.push_back(k);
          }
        }
      }
      std::sort(u_cols.begin() + static_cast<std::ptrdiff_t>(u0), u_cols.end());
      plan->group_lo[g] = low;
      int32_t l = 0;
      for (size_t u = u0; u < u_cols.size(); ++u) l = std::max(l, level[group_of[u_cols[u]]] + 1);
      level[g] = l;
      levels = std::max(levels, l + 1);
      plan->u_start[g + 1] = static_cast<int64_t>(u_cols.size());
      const size_t o0 = outer.size(), i0 = inner.size();
      outer.resize(o0 + (u_cols.size() - u0) * rows, 0.0);
      inner.resize(i0 + static_cast<size_t>(rows) * rows, 0.0);
      for (int32_t r = a; r < b; ++r) {
        for (int64_t p = f.row_start[r]; p < f.row_start[r + 1] - 1; ++p) {
          const int32_t k = f.pattern[p];
          if (k < a) {
            const size_t u = std::lower_bound(u_cols.begin() + static_cast<std::ptrdiff_t>(u0), u_cols.end(), k) -
                             (u_cols.begin() + static_cast<std::ptrdiff_t>(u0));
            outer[o0 + u * rows + (r - a)] = f.values[p];
          } else {
            inner[i0 + static_cast<size_t>(r - a) * rows + (k - a)] = f.values[p];
          }
        }
      }
      plan->outer_start[g + 1] = static_cast<int64_t>(outer.size());
      plan->inner_start[g + 1] = static_cast<int64_t>(inner.size());
    }
  }
  std::vector<int32_t>& level_start = plan->level_start;
  level_start.assign(static_cast<size_t>(levels) + 1, 0);
  for (int32_t g = 0; g < groups; ++g) level_start[level[g] + 1] += 1;
  for (int32_t l = 0; l < levels; ++l) level_start[l + 1] += level_start[l];
  plan->groups_by_level.assign(groups, 0);
  {
    std::vector<int32_t> cursor(level_start.begin(), level_start.end() - 1);
    for (int32_t g = 0; g < groups; ++g) plan->groups_by_level[cursor[level[g]]++] = g;
  }
  return true;
}

void compact_dense_rows(const RowGroups& plan, const double* dense, InverseRows* out) {
  const int32_t n = static_cast<int32_t>(plan.lo.size());
  out->start.assign(static_cast<size_t>(n) + 1, 0);
  const unsigned workers = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  RowPool pool(workers);
  auto ranges = [&](const std::function<void(int32_t, int32_t)>& body) {
    pool.run([&](unsigned w) {
      body(static_cast<int32_t>(static_cast<int64_t>(n) * w / workers),
           static_cast<int32_t>(static_cast<int64_t>(n) * (w + 1) / workers));
    });
  };
  ranges([&](int32_t r0, int32_t r1) {
    for (int32_t i = r0; i < r1; ++i) {
      int64_t kept = 0;
      for (int64_t q = plan.base[i]; q < plan.base[i + 1]; ++q) kept += dense[q] != 0.0;
      out->start[i + 1] = kept;
    }
  });
  for (int32_t i = 0; i < n; ++i) out->start[i + 1] += out->start[i];
  out->columns.resize(static_cast<size_t>(out->start[n]));
  out->values.resize(static_cast<size_t>(out->start[n]));
  ranges([&](int32_t r0, int32_t r1) {
    for (int32_t i = r0; i < r1; ++i) {
      int64_t at = out->start[i];
      for (int64_t q = plan.base[i]; q < plan.base[i + 1]; ++q) {
        if (dense[q] != 0.0) {
          out->columns[at] = plan.lo[i] + static_cast<int32_t>(q - plan.base[i]);
          out->values[at] = dense[q];
          ++at;
        }
      }
    }
  });
}

bool inverse_rows_by_groups(const LowerFactorView& f, InverseRows* out, RowPool& pool) {
  RowGroups plan;
  if (!plan_row_groups(f, &plan)) return false;
  const std::vector<int32_t>& lo = plan.lo;
  const std::vector<int64_t>& base = plan.base;
  std::vector<double> dense(static_cast<size_t>(base[f.size]));
  struct Item {
    int32_t group, chunk;
  };
  std::vector<Item> items;
  std::vector<std::vector<double>> tiles(pool.size(),
                                         std::vector<double>(static_cast<size_t>(kRowGroupRows) * kRowGroupChunk));
  double* d = dense.data();
  const int32_t levels = static_cast<int32_t>(plan.level_start.size()) - 1;
  for (int32_t l = 0; l < levels; ++l) {
    items.clear();
    for (int32_t q = plan.level_start[l]; q < plan.level_start[l + 1]; ++q) {
      const int32_t g = plan.groups_by_level[q];
      for (int32_t j = plan.group_lo[g] / kRowGroupChunk; j <= (plan.group_start[g + 1] - 1) / kRowGroupChunk; ++j)
        items.push_back(Item{g, j});
    }
    const int64_t count = static_cast<int64_t>(items.size());
    std::atomic<int64_t> next{0};
    auto work = [&](unsigned w) {
      double* tile = tiles[w].data();
      for (int64_t t = next.fetch_add(1); t < count; t = next.fetch_add(1)) {
        const int32_t g = items[t].group;
        const int32_t a = plan.group_start[g], rows = plan.group_start[g + 1] - a;
        const int32_t c0 = items[t].chunk * kRowGroupChunk, c1 = c0 + kRowGroupChunk;
        auto row_of = [&](int32_t r) { return tile + static_cast<size_t>(r) * kRowGroupChunk; };
        for (int32_t r = 0; r < rows; ++r) {
          std::fill(row_of(r), row_of(r) + kRowGroupChunk, 0.0);
          if (a + r >= c0 && a + r < c1) row_of(r)[a + r - c0] = 1.0;
        }
        const double* multipliers = plan.outer.data() + plan.outer_start[g];
        // Outside columns meeting the chunk, four at a time: on the labels all
        // four cover, one pass per row applies them in ascending order (a zero
        // multiplier subtracts a signed zero there); elsewhere each column
        // applies alone, in ascending order.
        int64_t u = plan.u_start[g];
        const int64_t u_end = plan.u_start[g + 1];
        while (u < u_end) {
          int64_t picked[4];
          int32_t from[4], to[4];
          int found = 0;
          for (; u < u_end && found < 4; ++u) {
            const int32_t k = plan.u_cols[u];
            from[found] = std::max(lo[k], c0);
            to[found] = std::min(k + 1, c1);
            if (from[found] < to[found]) picked[found++] = u;
          }
          const double* source[4];
          const double* column[4];
          for (int t = 0; t < found; ++t) {
            const int32_t k = plan.u_cols[picked[t]];
            source[t] = d + base[k] + (from[t] - lo[k]);
            column[t] = multipliers + (picked[t] - plan.u_start[g]) * rows;
          }
          const int32_t common_from = found == 4 ? std::max(std::max(from[0], from[1]), std::max(from[2], from[3])) : 0;
          const int32_t common_to = found == 4 ? std::min(std::min(to[0], to[1]), std::min(to[2], to[3])) : 0;
          const bool blocked = found == 4 && common_from < common_to;
          for (int32_t r = 0; r < rows; ++r) {
            double* row = row_of(r);
            if (!blocked) {
              for (int t = 0; t < found; ++t) {
                if (column[t][r] == 0.0) continue;
                subtract_scaled(row + (from[t] - c0), source[t], column[t][r], to[t] - from[t]);
              }
              continue;
            }
            const double m[4] = {column[0][r], column[1][r], column[2][r], column[3][r]};
            if (m[0] == 0.0 && m[1] == 0.0 && m[2] == 0.0 && m[3] == 0.0) continue;
            for (int t = 0; t < 4; ++t) {
              if (m[t] == 0.0) continue;
              if (from[t] < common_from)
                subtract_scaled(row + (from[t] - c0), source[t], m[t], common_from - from[t]);
              if (common_to < to[t])
                subtract_scaled(row + (common_to - c0), source[t] + (common_to - from[t]), m[t], to[t] - common_to);
            }
            const double* x[4];
            for (int t = 0; t < 4; ++t) x[t] = source[t] + (common_from - from[t]);
            subtract_scaled4(row + (common_from - c0), x[0], x[1], x[2], x[3], m, common_to - common_from);
          }
        }
        const double* own = plan.inner.data() + plan.inner_start[g];
        for (int32_t kk = 0; kk + 1 < rows; ++kk) {
          const int32_t k = a + kk;
          const int32_t from = std::max(lo[k], c0), to = std::min(k + 1, c1);
          if (from >= to) continue;
          for (int32_t r = kk + 1; r < rows; ++r) {
            const double coefficient = own[static_cast<size_t>(r) * rows + kk];
            if (coefficient == 0.0) continue;
            subtract_scaled(row_of(r) + (from - c0), row_of(kk) + (from - c0), coefficient, to - from);
          }
        }
        for (int32_t r = 0; r < rows; ++r) {
          const int32_t i = a + r;
          const int32_t from = std::max(lo[i], c0), to = std::min(i + 1, c1);
          if (from < to) std::copy(row_of(r) + (from - c0), row_of(r) + (to - c0), d + base[i] + (from - lo[i]));
        }
      }
    };
    if (count > 1) {
      pool.run(work);
    } else {
      work(0);
    }
  }
  compact_dense_rows(plan, d, out);
  return true;
}

std::string build_inverse_factor(int32_t size, const int32_t* row_offsets, const int32_t* row_columns,
                                 const double* row_values, InverseFactor* out, const InverseRowsProvider& provider,
                                 const LdltProvider& ldlt_provider) {
  if (size < 0) return "matrix size must be nonnegative";
  // --- _validate_rows (sparse.py:73-95) ---------------------------------
  std::vector<std::vector<std::pair<int32_t, double>>> rows(size);
  for (int32_t i = 0; i < size; ++i) {
    if (row_offsets[i + 1] < row_offsets[i]) return "row offsets must be nondecreasing";
    for (int32_t p = row_offsets[i]; p < row_offsets[i + 1]; ++p) {
      const int32_t j = row_columns[p];
      const double value = row_values[p];
      if (j < 0 || j >= size) return "matrix column indices must be integers in [0, size)";
      if (!std::isfinite(value)) return "matrix coefficients must be finite";
      if (value != 0.0) rows[i].emplace_back(j, value);
    }
    std::sort(rows[i].begin(), rows[i].end(),
              [](const auto& a, const auto& b) { return a.first < b.first; });
    for (size_t p = 1; p < rows[i].size(); ++p) {
      if (rows[i][p].first == rows[i][p - 1].first) return "matrix rows must not repeat a column";
    }
    double diagonal = 0.0;
    for (const auto& entry : rows[i]) {
      if (entry.first == i) diagonal = entry.second;
    }
    if (!(diagonal > 0.0)) return "matrix must be positive definite with positive diagonal entries";
  }
  int64_t matrix_nnz = 0;
  for (int32_t i = 0; i < size; ++i) {
    matrix_nnz += static_cast<int64_t>(rows[i].size());
    for (const auto& entry : rows[i]) {
      const auto& other = rows[entry.first];
      auto it = std::lower_bound(other.begin(), other.end(), std::make_pair(i, 0.0),
                                 [](const auto& a, const auto& b) { return a.first < b.first; });
      if (it == other.end() || it->first != i || it->second != entry.second) {
        return "matrix_rows must contain both halves of an exactly symmetric matrix";
      }
    }
  }
  // --- Ordering -----------------------------------------------------------
  Adjacency adjacency(size);
  for (int32_t i = 0; i < size; ++i) {
    for (const auto& entry : rows[i]) {
      if (entry.first != i) adjacency[i].push_back(entry.first);
    }
  }
  std::vector<int32_t> permutation = nested_dissection(adjacency);
  std::vector<int32_t> inverse(size);
  for (int32_t k = 0; k < size; ++k) inverse[permutation[k]] = k;

  // --- Symbolic fill (sparse.py:98-124) via the elimination tree ----------
  // Column k of L holds {i > k : A(i,k) != 0} and the columns of its
  // elimination-tree children; this is the structure the reference's
  // set-based fill discovery produces.
  std::vector<std::vector<int32_t>> lower_a(size);  // permuted strict-lower A entries per column
  for (int32_t i = 0; i < size; ++i) {
    const int32_t pi = inverse[i];
    for (const auto& entry : rows[i]) {
      const int32_t pj = inverse[entry.first];
      if (pj < pi) lower_a[pj].push_back(pi);
    }
  }
  std::vector<std::vector<int32_t>> columns(size);
  std::vector<std::vector<int32_t>> children(size);
  std::vector<int32_t> marker(size, -1);
  for (int32_t k = 0; k < size; ++k) {
    std::vector<int32_t>& column = columns[k];
    for (int32_t i : lower_a[k]) {
      if (marker[i] != k) {
        marker[i] = k;
        column.push_back(i);
      }
    }
    for (int32_t c : children[k]) {
      for (int32_t i : columns[c]) {
        if (i > k && marker[i] != k) {
          marker[i] = k;
          column.push_back(i);
        }
      }
    }
    std::sort(column.begin(), column.end());
    if (!column.empty()) children[column.front()].push_back(k);
    std::vector<int32_t>().swap(lower_a[k]);
  }
  std::vector<std::vector<int32_t>>().swap(children);
  // Row patterns, each ending with its diagonal.
  std::vector<int32_t> row_counts(size, 1);
  for (int32_t k = 0; k < size; ++k) {
    for (int32_t i : columns[k]) row_counts[i] += 1;
  }
  std::vector<int64_t> row_start(size + 1, 0);
  for (int32_t i = 0; i < size; ++i) row_start[i + 1] = row_start[i] + row_counts[i];
  const int64_t pattern_nnz = row_start[size];
  std::vector<int32_t> pattern(pattern_nnz);
  std::vector<double> values(pattern_nnz, 0.0);
  {
    std::vector<int64_t> cursor(row_start.begin(), row_start.end() - 1);
    for (int32_t k = 0; k < size; ++k) {
      for (int32_t i : columns[k]) pattern[cursor[i]++] = k;
    }
    for (int32_t i = 0; i < size; ++i) pattern[cursor[i]++] = i;
  }
  // Positions of column k inside each row of columns[k].
  std::vector<std::vector<int64_t>> column_positions(size);
  for (int32_t k = 0; k < size; ++k) column_positions[k].reserve(columns[k].size());
  for (int32_t i = 0; i < size; ++i) {
    for (int64_t p = row_start[i]; p < row_start[i + 1] - 1; ++p) column_positions[pattern[p]].push_back(p);
  }
  // Initial values: the permuted lower triangle of A.
  for (int32_t i = 0; i < size; ++i) {
    const int32_t pi = inverse[i];
    for (const auto& entry : rows[i]) {
      const int32_t pj = inverse[entry.first];
      if (pj <= pi) {
        const int32_t* first = pattern.data() + row_start[pi];
        const int32_t* last = pattern.data() + row_start[pi + 1];
        const int32_t* at = std::lower_bound(first, last, pj);
        values[row_start[pi] + (at - first)] = entry.second;
      }
    }
  }
  std::vector<std::vector<std::pair<int32_t, double>>>().swap(rows);

  // --- Numeric right-looking LDL^T (sparse.py:136-151) --------------------
  std::vector<double> diagonal(size);
  std::vector<double> entries;
  std::vector<int64_t> locations;
  bool factored = false;
  if (ldlt_provider) {
    std::vector<int64_t> col_start(static_cast<size_t>(size) + 1, 0);
    for (int32_t k = 0; k < size; ++k) col_start[k + 1] = col_start[k] + static_cast<int64_t>(columns[k].size());
    std::vector<int32_t> col_rows(static_cast<size_t>(col_start[size]));
    std::vector<int64_t> col_pos(static_cast<size_t>(col_start[size]));
    std::vector<int32_t> column_index(static_cast<size_t>(pattern_nnz), -1);
    for (int32_t k = 0; k < size; ++k) {
      for (size_t o = 0; o < columns[k].size(); ++o) {
        col_rows[col_start[k] + o] = columns[k][o];
        col_pos[col_start[k] + o] = column_positions[k][o];
        column_index[column_positions[k][o]] = static_cast<int32_t>(o);
      }
    }
    SymbolicView view;
    view.size = size;
    view.row_start = row_start.data();
    view.pattern = pattern.data();
    view.col_start = col_start.data();
    view.col_rows = col_rows.data();
    view.column_index = column_index.data();
    view.col_pos = col_pos.data();
    const std::string error = ldlt_provider(view, values.data(), diagonal.data());
    if (error.rfind("device LDLT:", 0) != 0) {
      if (!error.empty()) return error;
      factored = true;
    }
  }
  // Large factors: left-looking columns over the host threads (bit-identical).
  if (!factored && pattern_nnz >= g_parallel_level_entries.load()) {
    const unsigned hardware = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (hardware > 1) {
      RowPool pool(hardware);
      ldlt_left_looking(size, row_start, pattern, columns, column_positions, values, diagonal, pool);
      for (int32_t k = 0; k < size; ++k) {
        const double pivot = diagonal[k];
        if (!std::isfinite(pivot) || pivot <= 0.0) {
          return "matrix is not positive definite: LDLT pivot " + std::to_string(k) + " is " + std::to_string(pivot);
        }
      }
      factored = true;
    }
  }
  for (int32_t k = factored ? size : 0; k < size; ++k) {
    const double pivot = values[row_start[k + 1] - 1];
    if (!std::isfinite(pivot) || pivot <= 0.0) {
      return "matrix is not positive definite: LDLT pivot " + std::to_string(k) + " is " + std::to_string(pivot);
    }
    diagonal[k] = pivot;
    const std::vector<int32_t>& neighbors = columns[k];
    const std::vector<int64_t>& positions = column_positions[k];
    const size_t count = neighbors.size();
    entries.resize(count);
    for (size_t o = 0; o < count; ++o) entries[o] = values[positions[o]];
    for (size_t o = 0; o < count; ++o) {
      const double multiplier = entries[o] / pivot;
      values[positions[o]] = multiplier;
      // Walk row i for columns neighbors[0..o]; all lie after column k.
      int64_t p = positions[o] + 1;
      for (size_t o2 = 0; o2 <= o; ++o2) {
        const int32_t j = neighbors[o2];
        while (pattern[p] < j) ++p;
        const double product = multiplier * entries[o2];
        values[p] = values[p] - product;
      }
    }
  }
  std::vector<std::vector<int64_t>>().swap(column_positions);
  std::vector<std::vector<int32_t>>().swap(columns);

  // --- Inverse rows (sparse.py:159-177) ----------------------------------
  // Unscaled rows of L^{-1} in elimination order, stored CSR. A row with much
  // update work is split by column range over host threads: every thread
  // walks the same earlier rows in the same order and applies only the
  // updates of its columns, so each entry sees the same sequence of rounded
  // operations as the sequential walk and the factor stays bit-identical.
  std::vector<int64_t> inv_start(1, 0);
  std::vector<int32_t> inv_columns;
  std::vector<double> inv_values;
  if (provider) {
    LowerFactorView view;
    view.size = size;
    view.row_start = row_start.data();
    view.pattern = pattern.data();
    view.values = values.data();
    InverseRows rows_out;
    const std::string error = provider(view, &rows_out);
    if (!error.empty()) return error;
    if (rows_out.start.size() != static_cast<size_t>(size) + 1 ||
        rows_out.columns.size() != static_cast<size_t>(rows_out.start.back()) ||
        rows_out.values.size() != rows_out.columns.size()) {
      return "inverse rows provider returned inconsistent arrays";
    }
    if (rows_out.columns.size() > static_cast<size_t>(std::numeric_limits<int32_t>::max())) {
      return "inverse factor fill exceeds int32 sparse indexing";
    }
    inv_start = std::move(rows_out.start);
    inv_columns = std::move(rows_out.columns);
    inv_values = std::move(rows_out.values);
  }
  const unsigned hardware = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  bool rows_done = static_cast<bool>(provider);
  if (!rows_done && hardware > 1 && pattern_nnz >= g_parallel_level_entries.load()) {
    LowerFactorView view;
    view.size = size;
    view.row_start = row_start.data();
    view.pattern = pattern.data();
    view.values = values.data();
    InverseRows rows_out;
    RowPool level_pool(hardware);
    if (inverse_rows_by_groups(view, &rows_out, level_pool)) {
      if (rows_out.columns.size() > static_cast<size_t>(std::numeric_limits<int32_t>::max())) {
        return "inverse factor fill exceeds int32 sparse indexing";
      }
      inv_start = std::move(rows_out.start);
      inv_columns = std::move(rows_out.columns);
      inv_values = std::move(rows_out.values);
      rows_done = true;
    }
  }
  std::vector<double> current(rows_done ? 0 : size, 0.0);
  std::vector<int32_t> touched_mark(rows_done ? 0 : size, -1);
  std::vector<int32_t> touched;
  std::unique_ptr<RowPool> pool;
  std::vector<std::vector<std::pair<int32_t, double>>> pieces;
  const int64_t parallel_work = g_parallel_row_work.load();
  for (int32_t i = rows_done ? size : 0; i < size; ++i) {
    int64_t work = 0;
    for (int64_t p = row_start[i]; p < row_start[i + 1] - 1; ++p) work += inv_start[pattern[p] + 1] - inv_start[pattern[p]];
    // Split only rows whose earlier rows are long: every range costs one
    // binary search per earlier row.
    const int64_t terms = row_start[i + 1] - 1 - row_start[i];
    if (hardware > 1 && work >= parallel_work && work >= 512 * terms) {
      if (!pool) {
        pool.reset(new RowPool(hardware));
        pieces.resize(2 * hardware);
      }
      // Column ranges handed out dynamically, several per thread, for balance.
      const int chunks = static_cast<int>(pieces.size());
      const int64_t span = static_cast<int64_t>(i) + 1;  // row i of L^{-1} has columns 0 .. i
      std::atomic<int> next_chunk{0};
      pool->run([&](unsigned) {
        std::vector<int32_t> mine;
        for (int chunk = next_chunk++; chunk < chunks; chunk = next_chunk++) {
        const int32_t lo = static_cast<int32_t>(span * chunk / chunks);
        const int32_t hi = static_cast<int32_t>(span * (chunk + 1) / chunks);
        std::vector<std::pair<int32_t, double>>& piece = pieces[chunk];
        piece.clear();
        mine.clear();
        if (i >= lo && i < hi) {
          current[i] = 1.0;
          touched_mark[i] = i;
          mine.push_back(i);
        }
        for (int64_t p = row_start[i]; p < row_start[i + 1] - 1; ++p) {
          const int32_t k = pattern[p];
          const double coefficient = values[p];
          if (coefficient == 0.0) continue;
          const int32_t* first = inv_columns.data() + inv_start[k];
          const int32_t* last = inv_columns.data() + inv_start[k + 1];
          const int32_t* begin = std::lower_bound(first, last, lo);
          const int32_t* end = std::lower_bound(begin, last, hi);
          for (const int32_t* c_at = begin; c_at < end; ++c_at) {
            const int32_t c = *c_at;
            if (touched_mark[c] != i) {
              touched_mark[c] = i;
              mine.push_back(c);
            }
            const double product = coefficient * inv_values[c_at - inv_columns.data()];
            current[c] = current[c] - product;
          }
        }
        std::sort(mine.begin(), mine.end());
        for (int32_t c : mine) {
          if (current[c] != 0.0) piece.emplace_back(c, current[c]);
          current[c] = 0.0;
        }
        }
      });
      for (int chunk = 0; chunk < chunks; ++chunk) {
        for (const auto& entry : pieces[chunk]) {
          inv_columns.push_back(entry.first);
          inv_values.push_back(entry.second);
        }
      }
      if (inv_columns.size() > static_cast<size_t>(std::numeric_limits<int32_t>::max())) {
        return "inverse factor fill exceeds int32 sparse indexing";
      }
      inv_start.push_back(static_cast<int64_t>(inv_columns.size()));
      continue;
    }
    touched.clear();
    current[i] = 1.0;
    touched_mark[i] = i;
    touched.push_back(i);
    for (int64_t p = row_start[i]; p < row_start[i + 1] - 1; ++p) {
      const int32_t k = pattern[p];
      const double coefficient = values[p];
      if (coefficient == 0.0) continue;  // subtracting a signed zero leaves every entry's value unchanged
      for (int64_t q = inv_start[k]; q < inv_start[k + 1]; ++q) {
        const int32_t c = inv_columns[q];
        if (touched_mark[c] != i) {
          touched_mark[c] = i;
          touched.push_back(c);
        }
        const double product = coefficient * inv_values[q];
        current[c] = current[c] - product;
      }
    }
    std::sort(touched.begin(), touched.end());
    for (int32_t c : touched) {
      if (current[c] != 0.0) {
        inv_columns.push_back(c);
        inv_values.push_back(current[c]);
      }
      current[c] = 0.0;
    }
    if (inv_columns.size() > static_cast<size_t>(std::numeric_limits<int32_t>::max())) {
      return "inverse factor fill exceeds int32 sparse indexing";
    }
    inv_start.push_back(static_cast<int64_t>(inv_columns.size()));
  }
  const int64_t nnz = static_cast<int64_t>(inv_columns.size());

  // --- CSR of S (rows: elimination order, columns: original, sorted) ------
  // Rows are independent: host threads take ranges of rows. Every value is
  // the same product inv_value * (1 / sqrt(pivot)) as in a sequential pass.
  out->size = size;
  out->permutation = permutation;
  out->diagonal = diagonal;
  out->factorization_nnz = static_cast<int64_t>(size) + (pattern_nnz - size);
  out->matrix_nnz = matrix_nnz;
  Csr& s = out->s;
  s.offsets.assign(size + 1, 0);
  s.columns.resize(nnz);
  s.values.resize(nnz);
  for (int32_t i = 0; i < size; ++i) s.offsets[i + 1] = static_cast<int32_t>(inv_start[i + 1]);
  const unsigned workers = (nnz >= (1 << 20) && hardware > 1) ? hardware : 1;
  std::unique_ptr<RowPool> csr_pool(workers > 1 ? new RowPool(workers) : nullptr);
  auto parallel_rows = [&](const std::function<void(int32_t, int32_t)>& body) {
    if (!csr_pool) {
      body(0, size);
      return;
    }
    const int32_t chunk = std::max<int32_t>(1, size / static_cast<int32_t>(8 * workers));
    std::atomic<int32_t> next{0};
    csr_pool->run([&](unsigned) {
      for (int32_t lo = next.fetch_add(chunk); lo < size; lo = next.fetch_add(chunk)) body(lo, std::min(size, lo + chunk));
    });
  };
  std::atomic<bool> overflow{false};
  parallel_rows([&](int32_t lo, int32_t hi) {
    std::vector<std::pair<int32_t, double>> row;
    for (int32_t i = lo; i < hi; ++i) {
      const double scale = 1.0 / std::sqrt(diagonal[i]);
      row.clear();
      for (int64_t q = inv_start[i]; q < inv_start[i + 1]; ++q) {
        row.emplace_back(permutation[inv_columns[q]], inv_values[q] * scale);
      }
      std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      const int64_t base = inv_start[i];
      for (size_t q = 0; q < row.size(); ++q) {
        s.columns[base + q] = row[q].first;
        s.values[base + q] = row[q].second;
        if (!std::isfinite(row[q].second)) overflow = true;
      }
    }
  });
  if (overflow) return "inverse factor overflowed float64";
  std::vector<int32_t>().swap(inv_columns);
  std::vector<double>().swap(inv_values);
  // --- CSR of S^T -----------------------------------------------------------
  // Within a column, entries keep ascending row order: each worker counts the
  // columns of a contiguous range of rows, and the ranges' cursors start
  // where the previous ranges' entries end.
  Csr& st = out->st;
  st.offsets.assign(size + 1, 0);
  st.columns.resize(nnz);
  st.values.resize(nnz);
  const int32_t ranges = csr_pool ? static_cast<int32_t>(workers) : 1;
  std::vector<std::vector<int32_t>> counts(ranges, std::vector<int32_t>(size, 0));
  auto range_rows = [&](int32_t r, int32_t& lo, int32_t& hi) {
    lo = static_cast<int32_t>(static_cast<int64_t>(size) * r / ranges);
    hi = static_cast<int32_t>(static_cast<int64_t>(size) * (r + 1) / ranges);
  };
  auto each_range = [&](const std::function<void(int32_t)>& body) {
    if (!csr_pool) {
      body(0);
      return;
    }
    csr_pool->run([&](unsigned w) { body(static_cast<int32_t>(w)); });
  };
  each_range([&](int32_t r) {
    int32_t lo, hi;
    range_rows(r, lo, hi);
    std::vector<int32_t>& count = counts[r];
    for (int64_t q = s.offsets[lo]; q < s.offsets[hi]; ++q) count[s.columns[q]] += 1;
  });
  for (int32_t c = 0; c < size; ++c) {
    int32_t total = 0;
    for (int32_t r = 0; r < ranges; ++r) total += counts[r][c];
    st.offsets[c + 1] = st.offsets[c] + total;
  }
  for (int32_t c = 0; c < size; ++c) {
    int32_t cursor = st.offsets[c];
    for (int32_t r = 0; r < ranges; ++r) {
      const int32_t count = counts[r][c];
      counts[r][c] = cursor;
      cursor += count;
    }
  }
  each_range([&](int32_t r) {
    int32_t lo, hi;
    range_rows(r, lo, hi);
    std::vector<int32_t>& cursor = counts[r];
    for (int32_t row = lo; row < hi; ++row) {
      for (int32_t q = s.offsets[row]; q < s.offsets[row + 1]; ++q) {
        const int32_t at = cursor[s.columns[q]]++;
        st.columns[at] = row;
        st.values[at] = s.values[q];
      }
    }
  });
  return std::string();
}

}  // namespace pdb200
