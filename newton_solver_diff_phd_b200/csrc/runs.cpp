// Postorder relabelling of the inverse factor into run matrices.
#include "runs.h"

#include <algorithm>
#include <utility>

namespace pdb200 {

namespace {

// Appends one row given as (label, value) pairs sorted by label.
void append_row(RunMatrix& m, const std::vector<std::pair<int32_t, double>>& entries, int max_gap) {
  for (size_t k = 0; k < entries.size(); ++k) {
    const int32_t label = entries[k].first;
    const bool extend = k > 0 && label - entries[k - 1].first - 1 <= max_gap;
    if (extend) {
      for (int32_t gap = entries[k - 1].first + 1; gap < label; ++gap) m.values.push_back(0.0);
    } else {
      m.run_col.push_back(label);
      m.run_off.push_back(static_cast<int32_t>(m.values.size()));
    }
    m.values.push_back(entries[k].second);
  }
  m.row_runs.push_back(static_cast<int32_t>(m.run_col.size()));
}

void finish(RunMatrix& m) { m.run_off.push_back(static_cast<int32_t>(m.values.size())); }

}  // namespace

RunFactor build_run_factor(const InverseFactor& factor, int max_gap) {
  const int32_t n = factor.size;
  std::vector<int32_t> position(n);
  for (int32_t r = 0; r < n; ++r) position[factor.permutation[r]] = r;
  // Elimination forest from the stored structure of S: rows ascend, so the
  // first row r > j that holds column j is the parent of j.
  std::vector<int32_t> parent(n, -1);
  for (int32_t r = 0; r < n; ++r) {
    for (int32_t k = factor.s.offsets[r]; k < factor.s.offsets[r + 1]; ++k) {
      const int32_t j = position[factor.s.columns[k]];
      if (j < r && parent[j] < 0) parent[j] = r;
    }
  }
  // Postorder: children in increasing order, roots in increasing order.
  std::vector<int32_t> child_start(n + 1, 0), children(n);
  for (int32_t j = 0; j < n; ++j)
    if (parent[j] >= 0) ++child_start[parent[j] + 1];
  for (int32_t j = 0; j < n; ++j) child_start[j + 1] += child_start[j];
  {
    std::vector<int32_t> fill(child_start.begin(), child_start.end() - 1);
    for (int32_t j = 0; j < n; ++j)
      if (parent[j] >= 0) children[fill[parent[j]]++] = j;
  }
  std::vector<int32_t> post(n, -1);
  int32_t next = 0;
  std::vector<std::pair<int32_t, int32_t>> stack;  // (node, next child index)
  for (int32_t root = 0; root < n; ++root) {
    if (parent[root] >= 0) continue;
    stack.emplace_back(root, child_start[root]);
    while (!stack.empty()) {
      auto& top = stack.back();
      if (top.second < child_start[top.first + 1]) {
        const int32_t child = children[top.second++];
        stack.emplace_back(child, child_start[child]);
      } else {
        post[top.first] = next++;
        stack.pop_back();
      }
    }
  }
  RunFactor out;
  out.label_of.resize(n);
  out.particle_of.resize(n);
  std::vector<int32_t> row_of_label(n);
  for (int32_t r = 0; r < n; ++r) row_of_label[post[r]] = r;
  for (int32_t p = 0; p < n; ++p) {
    out.label_of[p] = post[position[p]];
    out.particle_of[out.label_of[p]] = p;
  }
  std::vector<std::pair<int32_t, double>> entries;
  out.s.row_runs.push_back(0);
  for (int32_t u = 0; u < n; ++u) {
    const int32_t r = row_of_label[u];
    entries.clear();
    for (int32_t k = factor.s.offsets[r]; k < factor.s.offsets[r + 1]; ++k)
      entries.emplace_back(out.label_of[factor.s.columns[k]], factor.s.values[k]);
    std::sort(entries.begin(), entries.end());
    append_row(out.s, entries, max_gap);
  }
  finish(out.s);
  out.st.row_runs.push_back(0);
  for (int32_t v = 0; v < n; ++v) {
    const int32_t p = out.particle_of[v];
    entries.clear();
    for (int32_t k = factor.st.offsets[p]; k < factor.st.offsets[p + 1]; ++k)
      entries.emplace_back(post[factor.st.columns[k]], factor.st.values[k]);
    std::sort(entries.begin(), entries.end());
    append_row(out.st, entries, max_gap);
  }
  finish(out.st);
  return out;
}

}  // namespace pdb200
