// Index-free storage of the inverse factor for the batched path.
//
// Row r (elimination order) of S = D^{-1/2} L^{-1} P^T is nonzero exactly at
// the particles whose elimination positions are r and the descendants of r in
// the elimination tree (L^{-1}_{rj} != 0 iff r is an ancestor of j). Numbering
// the nodes by a postorder of that tree turns every descendant set into one
// contiguous label range, so a row of S is one run [first, r] of consecutive
// labels and needs no column indices; a row of S^T (the ancestors of a node)
// is a few runs, one per chain of the tree it climbs.
//
// The factor arrays are unchanged: a run matrix stores the same values as
// the CSR factor, in label order, with explicit zeros only where a gap of at
// most `max_gap` omitted exact zeros is bridged. The tree is read from the
// stored structure of S (the first row below the diagonal that holds column
// j is the parent of j), so omitted zeros can only split runs, never lose an
// entry.
#pragma once

#include <cstdint>
#include <vector>

#include "factor.h"

namespace pdb200 {

struct RunMatrix {
  std::vector<int32_t> row_runs;  // [rows + 1]: runs of row u are [row_runs[u], row_runs[u + 1])
  std::vector<int32_t> run_col;   // [runs]: first column label of the run
  std::vector<int32_t> run_off;   // [runs + 1]: value offsets; run k holds run_off[k+1] - run_off[k] values
  std::vector<double> values;     // [run_off.back()]
};

struct RunFactor {
  std::vector<int32_t> label_of;     // particle -> label
  std::vector<int32_t> particle_of;  // label -> particle
  RunMatrix s;                       // rows and columns in labels
  RunMatrix st;                      // S^T, rows and columns in labels
};

RunFactor build_run_factor(const InverseFactor& factor, int max_gap);

}  // namespace pdb200
