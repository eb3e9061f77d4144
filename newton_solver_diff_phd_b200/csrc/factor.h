// Exact sparse inverse factor A^{-1} = S^T S of a constant SPD scalar matrix.
//
// Host-side setup of the DiffPhD global step. It follows the reference's
// SparseInverse setup (src/newton_solver_diff_phd/_src/solvers/diff_phd/sparse.py):
// nested dissection with minimum-degree leaves (:18-70), symbolic fill and a
// right-looking numeric LDL^T in a fixed update order (:98-156), inverse rows
// with exact-zero omission (:159-177) and CSR output sorted by column
// (:180-191, :301-314). Every floating-point update is one rounded multiply
// followed by one rounded subtract, as NumPy evaluates them, so the factor is
// bit-identical to the reference's for the same input rows.
#pragma once

#include <atomic>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace pdb200 {

struct Csr {
  std::vector<int32_t> offsets;
  std::vector<int32_t> columns;
  std::vector<double> values;
};

struct InverseFactor {
  int32_t size = 0;
  std::vector<int32_t> permutation;  // elimination order -> original index
  std::vector<double> diagonal;      // LDL^T pivots in elimination order
  Csr s;                             // rows: elimination order, columns: original index
  Csr st;                            // S^T: rows original index, columns elimination order
  int64_t factorization_nnz = 0;     // size + strict lower nnz(L)
  int64_t matrix_nnz = 0;
};

// Update work (entries of earlier rows combined) from which one row of the
// inverse is split over host threads; the result is bit-identical either way.
extern std::atomic<int64_t> g_parallel_row_work;

// Entries of L from which the numeric LDL^T (left-looking columns) and the
// rows of L^{-1} (chunked rows) run over host threads level by level of the
// elimination tree instead of sequentially (bit-identical).
extern std::atomic<int64_t> g_parallel_level_entries;

// The rows of the unit lower factor L in elimination order after the numeric
// LDL^T: row i holds its columns k < i in ascending order with the
// multipliers L(i, k), then its diagonal entry (position row_start[i+1] - 1,
// not used by the inverse rows).
struct LowerFactorView {
  int32_t size = 0;
  const int64_t* row_start = nullptr;  // [size + 1]
  const int32_t* pattern = nullptr;
  const double* values = nullptr;
};

// Unscaled rows of L^{-1} in elimination order, columns ascending, entries
// that are exactly zero omitted (sparse.py:159-177).
struct InverseRows {
  std::vector<int64_t> start;  // [size + 1]
  std::vector<int32_t> columns;
  std::vector<double> values;
};

// Computes the inverse rows somewhere else (the device); returns an empty
// string on success. Must produce exactly the rows of the host walk.
using InverseRowsProvider = std::function<std::string(const LowerFactorView&, InverseRows*)>;

// The structure of the numeric LDL^T: the rows of L (columns k < i ascending,
// then the diagonal) and, for every column k, the rows i > k it holds in
// ascending order (col_start / col_rows) with, for every strict entry p of
// the row arrays, the index of its row within its column (column_index).
struct SymbolicView {
  int32_t size = 0;
  const int64_t* row_start = nullptr;  // [size + 1]
  const int32_t* pattern = nullptr;
  const int64_t* col_start = nullptr;  // [size + 1]
  const int32_t* col_rows = nullptr;
  const int32_t* column_index = nullptr;  // per row-array position; -1 at the diagonal
  const int64_t* col_pos = nullptr;       // per column entry: its position in the row arrays
};

// The numeric LDL^T somewhere else: `values` holds the permuted lower
// triangle of A at the row-array positions on entry; on success the strict
// positions hold the multipliers L(i, k), the diagonal positions and
// `diagonal` the pivots, exactly as the host's right-looking factorisation
// leaves them (every entry updated by ascending pivots, one rounded multiply
// then one rounded subtract each). Errors use the host's messages.
using LdltProvider = std::function<std::string(const SymbolicView&, double* values, double* diagonal)>;

// Rows of L^{-1} as dense segments in groups of consecutive rows (the host's
// level path and, on request, the device's): row i is stored over the labels
// [lo[i], i] of its elimination subtree at dense[base[i] + c - lo[i]]; group g
// holds rows group_start[g] .. group_start[g+1]-1 (at most kRowGroupRows),
// its outside columns u_cols[u_start[g] .. u_start[g+1]) ascending, the
// multipliers outer[outer_start[g] + u * rows + r] of row a + r at outside
// column u and inner[inner_start[g] + r * rows + kk] at the group's own row
// a + kk (zero where the row lacks the column), and the lowest label of its
// rows; groups_by_level lists the groups level by level (a group reads only
// groups of lower levels), level_start indexing it.
constexpr int32_t kRowGroupChunk = 256;
constexpr int32_t kRowGroupRows = 32;
struct RowGroups {
  std::vector<int32_t> lo;
  std::vector<int64_t> base;  // [size + 1]
  std::vector<int32_t> group_start, group_lo;
  std::vector<int64_t> u_start, outer_start, inner_start;
  std::vector<int32_t> u_cols;
  std::vector<double> outer, inner;
  std::vector<int32_t> level_start, groups_by_level;
};
// Plans the groups; false when the dense segments would hold more than twice
// the rows' structural entries (an order far from a postorder).
bool plan_row_groups(const LowerFactorView& factor, RowGroups* plan);
// The rows of L^{-1} from their dense segments: exact zeros omitted, columns
// ascending (over host threads).
void compact_dense_rows(const RowGroups& plan, const double* dense, InverseRows* out);
// Which device computes the rows of L^{-1} when the build runs on the device:
// 0 the chunked rows (default), 1 the grouped dense segments.
extern std::atomic<int32_t> g_device_rows_grouped;
std::string device_inverse_rows_grouped(const LowerFactorView& factor, InverseRows* out);
std::string device_inverse_rows_chunked(const LowerFactorView& factor, InverseRows* out);
// The numeric LDL^T on the current CUDA device, column by column within
// levels of the elimination tree (pd_factor_device.cu). Rows longer than the
// shared memory staging allows return an error starting with "device LDLT:".
std::string device_ldlt(const SymbolicView& symbolic, double* values, double* diagonal);

// The inverse rows on the current CUDA device, level by level of the
// elimination tree (pd_factor_device.cu); bit-identical to the host walk.
std::string device_inverse_rows(const LowerFactorView& factor, InverseRows* out);

// Validates rows (finite, positive diagonal, exact symmetry) and builds the
// factor. Returns an empty string on success, otherwise the reason. With a
// provider, the inverse rows come from it instead of the host walk.
std::string build_inverse_factor(int32_t size, const int32_t* row_offsets, const int32_t* row_columns,
                                 const double* row_values, InverseFactor* out,
                                 const InverseRowsProvider& provider = InverseRowsProvider(),
                                 const LdltProvider& ldlt_provider = LdltProvider());

// Nested-dissection order of an undirected graph given as sorted adjacency
// lists without self loops (the reference _nested_dissection).
std::vector<int32_t> nested_dissection(const std::vector<std::vector<int32_t>>& adjacency);

}  // namespace pdb200
