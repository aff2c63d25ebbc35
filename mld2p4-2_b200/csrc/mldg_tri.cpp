// mldg_tri.cpp -- host-side schedule of the chunked, level-scheduled sparse
// unit-triangular solve.  Within each chunk of R consecutive internal rows,
// row levels count intra-chunk dependencies only; rows are then stored in
// (chunk, level, row) order so a CTA walks one chunk level by level.
#include "mldg_tri.h"

#include <algorithm>

namespace mldg {

void build_tri_schedule(int n, const int *irp, const int *ja, const double *val, bool upper, int R,
                        TriSchedule *s) {
  s->n = n;
  s->R = R;
  s->nchunks = n > 0 ? (n + R - 1) / R : 0;
  s->chunk_lvl.assign((size_t)s->nchunks + 1, 0);
  s->lvl_ptr.clear();
  s->prow.assign((size_t)n, 0);
  s->pirp.assign((size_t)n + 1, 0);
  const long nnz = n > 0 ? irp[n] : 0;
  s->pja.resize((size_t)nnz);
  s->pval.resize((size_t)nnz);
  s->max_levels_per_chunk = 0;
  auto orig = [&](int ip) { return upper ? n - 1 - ip : ip; };
  std::vector<int> lev((size_t)n, 0);
  std::vector<int> cnt;
  int pos = 0;
  for (int c = 0; c < s->nchunks; ++c) {
    const int s0 = c * R, e0 = std::min(n, s0 + R);
    int maxlev = 0;
    for (int ip = s0; ip < e0; ++ip) {
      const int o = orig(ip);
      int l = 0;
      for (int k = irp[o]; k < irp[o + 1]; ++k) {
        const int jp = upper ? n - 1 - ja[k] : ja[k];
        if (jp >= s0) l = std::max(l, lev[jp] + 1);
      }
      lev[ip] = l;
      maxlev = std::max(maxlev, l);
    }
    cnt.assign((size_t)maxlev + 2, 0);
    for (int ip = s0; ip < e0; ++ip) cnt[lev[ip] + 1]++;
    for (int l = 0; l <= maxlev; ++l) cnt[l + 1] += cnt[l];
    s->chunk_lvl[c] = (int)s->lvl_ptr.size();
    for (int l = 0; l <= maxlev; ++l) s->lvl_ptr.push_back(pos + cnt[l]);
    for (int ip = s0; ip < e0; ++ip) s->prow[pos + cnt[lev[ip]]++] = ip;
    pos += e0 - s0;
    s->max_levels_per_chunk = std::max(s->max_levels_per_chunk, maxlev + 1);
  }
  s->chunk_lvl[s->nchunks] = (int)s->lvl_ptr.size();
  s->lvl_ptr.push_back(n);
  // rows in position order: offsets by a prefix sum, then an independent copy per row
  long q = 0;
  for (int p = 0; p < n; ++p) {
    const int o = orig(s->prow[p]);
    s->pirp[p] = (int)q;
    q += irp[o + 1] - irp[o];
  }
  s->pirp[n] = (int)q;
#pragma omp parallel for schedule(static, 4096)
  for (int p = 0; p < n; ++p) {
    const int o = orig(s->prow[p]);
    long t = s->pirp[p];
    for (int k = irp[o]; k < irp[o + 1]; ++k, ++t) {
      s->pja[t] = upper ? n - 1 - ja[k] : ja[k];
      s->pval[t] = val[k];
    }
  }
}

}  // namespace mldg
