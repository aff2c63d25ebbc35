// mldg_tri.h -- host-side schedule of the chunked, level-scheduled sparse
// unit-triangular solve (see k_trsv in mldg_kernels.cuh).
#pragma once
#include <vector>

namespace mldg {

struct TriSchedule {
  int n = 0, R = 0, nchunks = 0;
  std::vector<int> chunk_lvl;  // nchunks + 1 : first level index of each chunk
  std::vector<int> lvl_ptr;    // levels + 1  : first position of each level
  std::vector<int> prow;       // n           : internal row at each position
  std::vector<int> pirp;       // n + 1       : entry offsets in position order
  std::vector<int> pja;        // nnz         : internal column ids
  std::vector<double> pval;    // nnz
  int max_levels_per_chunk = 0;
};

// (irp, ja, val): strictly triangular CSR, 0-based.  upper == true stores
// the factor reversed (internal row i' = n-1-i) so that it is lower in
// internal numbering.  R: rows per chunk.
void build_tri_schedule(int n, const int *irp, const int *ja, const double *val, bool upper, int R,
                        TriSchedule *s);

}  // namespace mldg
