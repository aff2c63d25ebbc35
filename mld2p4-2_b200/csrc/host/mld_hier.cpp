// mld_hier.cpp -- host-side producers of the level hierarchy (see mld_hier.h).
//
// Built with -ffp-contract=off: each a*b+c below is two roundings, in the
// order the reference writes it.  Sparse products run row-parallel (OpenMP);
// each row is accumulated in a fixed order, so results do not depend on the
// thread count.
#include "mld_hier.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "mldg.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace mld {

// PSBLAS 3.5 d_epstol, the pivot threshold of mld_dilu0_fact.f90:436
static const double kEpsTol = 1.1102230246251565e-16;

// ---------------------------------------------------------------------------
void gen_pde3d(int idim, int hden, const double *coef, CSR &a) {
  const double a1 = coef[0], a2 = coef[1], a3 = coef[2];
  const double b1 = coef[3], b2 = coef[4], b3 = coef[5], c = coef[6];
  const double h = 1.0 / (double)(idim + hden);
  const double h2 = h * h, dh2 = 2.0 * h;
  // stencil values, (x-1),(y-1),(z-1),C,(z+1),(y+1),(x+1)
  const double vxm = -a1 / h2 - b1 / dh2, vym = -a2 / h2 - b2 / dh2, vzm = -a3 / h2 - b3 / dh2;
  const double vc = 2.0 * (a1 + a2 + a3) / h2 + c;
  const double vzp = -a3 / h2 + b3 / dh2, vyp = -a2 / h2 + b2 / dh2, vxp = -a1 / h2 + b1 / dh2;
  const int64_t s2 = (int64_t)idim * idim, n = s2 * idim;
  a.nr = a.nc = (int)n;
  a.irp.assign((size_t)n + 1, 0);
  // row lengths first so rows can be filled in parallel
  for (int64_t r = 0; r < n; ++r) {
    const int ix = (int)(r / s2), iy = (int)((r / idim) % idim), iz = (int)(r % idim);
    a.irp[r + 1] = 1 + (ix > 0) + (iy > 0) + (iz > 0) + (iz < idim - 1) + (iy < idim - 1) +
                   (ix < idim - 1);
  }
  for (int64_t r = 0; r < n; ++r) a.irp[r + 1] += a.irp[r];
  a.ja.resize((size_t)a.irp[n]);
  a.val.resize((size_t)a.irp[n]);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; ++r) {
    const int ix = (int)(r / s2), iy = (int)((r / idim) % idim), iz = (int)(r % idim);
    int k = a.irp[r];
    auto put = [&](int64_t col, double v) {
      a.ja[k] = (int)col;
      a.val[k] = v;
      ++k;
    };
    if (ix > 0) put(r - s2, vxm);
    if (iy > 0) put(r - idim, vym);
    if (iz > 0) put(r - 1, vzm);
    put(r, vc);
    if (iz < idim - 1) put(r + 1, vzp);
    if (iy < idim - 1) put(r + idim, vyp);
    if (ix < idim - 1) put(r + s2, vxp);
  }
}

void gen_kappa3d(int idim, const double *kappa, CSR &a) {
  const double h = 1.0 / (double)(idim + 1);
  const double ih2 = 1.0 / (h * h);
  const int64_t s2 = (int64_t)idim * idim, n = s2 * idim;
  a.nr = a.nc = (int)n;
  a.irp.assign((size_t)n + 1, 0);
  for (int64_t r = 0; r < n; ++r) {
    const int ix = (int)(r / s2), iy = (int)((r / idim) % idim), iz = (int)(r % idim);
    a.irp[r + 1] = 1 + (ix > 0) + (iy > 0) + (iz > 0) + (iz < idim - 1) + (iy < idim - 1) +
                   (ix < idim - 1);
  }
  for (int64_t r = 0; r < n; ++r) a.irp[r + 1] += a.irp[r];
  a.ja.resize((size_t)a.irp[n]);
  a.val.resize((size_t)a.irp[n]);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; ++r) {
    const int ix = (int)(r / s2), iy = (int)((r / idim) % idim), iz = (int)(r % idim);
    const double kc = kappa[r];
    auto face = [&](bool inside, int64_t nb) {
      if (!inside) return kc;  // Dirichlet boundary face
      const double kn = kappa[nb];
      return 2.0 * kc * kn / (kc + kn);
    };
    const bool in[6] = {ix > 0, iy > 0, iz > 0, iz < idim - 1, iy < idim - 1, ix < idim - 1};
    const int64_t nb[6] = {r - s2, r - idim, r - 1, r + 1, r + idim, r + s2};
    double f[6];
    double diag = 0.0;
    for (int q = 0; q < 6; ++q) {
      f[q] = face(in[q], nb[q]);
      diag = diag + f[q];
    }
    int k = a.irp[r];
    for (int q = 0; q < 3; ++q)
      if (in[q]) {
        a.ja[k] = (int)nb[q];
        a.val[k++] = -f[q] * ih2;
      }
    a.ja[k] = (int)r;
    a.val[k++] = diag * ih2;
    for (int q = 3; q < 6; ++q)
      if (in[q]) {
        a.ja[k] = (int)nb[q];
        a.val[k++] = -f[q] * ih2;
      }
  }
}

// ---------------------------------------------------------------------------
static std::vector<double> diag_of(const CSR &a) {
  std::vector<double> d((size_t)a.nr, 0.0);
  for (int i = 0; i < a.nr; ++i)
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k)
      if (a.ja[k] == i) d[i] += a.val[k];
  return d;
}

CSR transpose(const CSR &a) {
  CSR t;
  t.nr = a.nc;
  t.nc = a.nr;
  t.irp.assign((size_t)t.nr + 1, 0);
  const int64_t nnz = a.nnz();
  t.ja.resize((size_t)nnz);
  t.val.resize((size_t)nnz);
  for (int64_t k = 0; k < nnz; ++k) t.irp[a.ja[k] + 1]++;
  for (int j = 0; j < t.nr; ++j) t.irp[j + 1] += t.irp[j];
  std::vector<int> fill(t.irp.begin(), t.irp.end() - 1);
  for (int i = 0; i < a.nr; ++i)
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k) {
      const int p = fill[a.ja[k]]++;
      t.ja[p] = i;
      t.val[p] = a.val[k];
    }
  return t;
}

// Row-parallel Gustavson product; row i accumulates a_ik*b_kj in the order of
// row i of a, then row k of b (first contribution assigned, later ones added);
// output columns ascending.  Stands in for psb_spspmm at
// mlprec/impl/mld_daggrmat_smth_asb.f90:316,345,399.
CSR spgemm(const CSR &a, const CSR &b) {
  CSR c;
  c.nr = a.nr;
  c.nc = b.nc;
  c.irp.assign((size_t)c.nr + 1, 0);
#pragma omp parallel
  {
    std::vector<int> mark((size_t)b.nc, -1);
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < a.nr; ++i) {
      int cnt = 0;
      for (int ka = a.irp[i]; ka < a.irp[i + 1]; ++ka) {
        const int k = a.ja[ka];
        for (int kb = b.irp[k]; kb < b.irp[k + 1]; ++kb) {
          const int j = b.ja[kb];
          if (mark[j] != i) {
            mark[j] = i;
            ++cnt;
          }
        }
      }
      c.irp[i + 1] = cnt;
    }
  }
  for (int i = 0; i < c.nr; ++i) c.irp[i + 1] += c.irp[i];
  c.ja.resize((size_t)c.irp[c.nr]);
  c.val.resize((size_t)c.irp[c.nr]);
#pragma omp parallel
  {
    std::vector<int> mark((size_t)b.nc, -1);
    std::vector<double> acc((size_t)b.nc, 0.0);
    std::vector<int> cols;
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < a.nr; ++i) {
      cols.clear();
      for (int ka = a.irp[i]; ka < a.irp[i + 1]; ++ka) {
        const int k = a.ja[ka];
        const double av = a.val[ka];
        for (int kb = b.irp[k]; kb < b.irp[k + 1]; ++kb) {
          const int j = b.ja[kb];
          const double p = av * b.val[kb];
          if (mark[j] != i) {
            mark[j] = i;
            acc[j] = p;
            cols.push_back(j);
          } else {
            acc[j] = acc[j] + p;
          }
        }
      }
      std::sort(cols.begin(), cols.end());
      int q = c.irp[i];
      for (int j : cols) {
        c.ja[q] = j;
        c.val[q] = acc[j];
        ++q;
      }
    }
  }
  return c;
}

// ---------------------------------------------------------------------------
// Decoupled aggregation on one rank, natural order
// (mlprec/impl/mld_d_dec_map_bld.f90:127-312).  Aggregates are 0-based.
int dec_aggregate(const CSR &a, double theta, std::vector<int> &ilaggr, int &naggr) {
  const int nr = a.nr;
  const std::vector<double> dg = diag_of(a);
  const int unset = -(nr + 1);
  ilaggr.assign((size_t)nr, unset);
  std::vector<int> nbr;
  nbr.reserve(64);
  auto strong = [&](int i, int k) {
    const int j = a.ja[k];
    return j >= 0 && j < nr && std::fabs(a.val[k]) > theta * std::sqrt(std::fabs(dg[i] * dg[j]));
  };
  int na = 0;
  // phase one: an untouched strongly-coupled neighbourhood becomes an aggregate
  for (int i = 0; i < nr; ++i) {
    if (ilaggr[i] != unset) continue;
    nbr.clear();
    bool disjoint = true;
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k)
      if (strong(i, k)) {
        nbr.push_back(a.ja[k]);
        if (ilaggr[a.ja[k]] != unset) disjoint = false;
      }
    if (disjoint) {
      ++na;
      for (int j : nbr) ilaggr[j] = na;
      ilaggr[i] = na;
    }
  }
  // phase two: join the most strongly coupled phase-one aggregate
  const std::vector<int> first(ilaggr);
  for (int i = 0; i < nr; ++i) {
    if (ilaggr[i] != unset) continue;
    double cpl = 0.0;
    int best = -1;
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k) {
      if (!strong(i, k)) continue;
      const double v = std::fabs(a.val[k]);
      if (first[a.ja[k]] > 0 && v > cpl) {
        best = a.ja[k];
        cpl = v;
      }
    }
    if (best >= 0) ilaggr[i] = ilaggr[best];
  }
  // phase three: leftovers and their unaggregated strong neighbours
  for (int i = 0; i < nr; ++i) {
    if (ilaggr[i] >= 0) continue;
    nbr.clear();
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k)
      if (strong(i, k) && ilaggr[a.ja[k]] < 0) nbr.push_back(a.ja[k]);
    ++na;
    ilaggr[i] = na;
    for (int j : nbr) ilaggr[j] = na;
  }
  for (int i = 0; i < nr; ++i) {
    if (ilaggr[i] <= 0) return -1;
    ilaggr[i] -= 1;
  }
  naggr = na;
  return 0;
}

// Smoothed prolongator P = (I - omega D^{-1} A) P_tent, omega = 4/(3 ||D^{-1}A||_inf),
// R = P^T, Ac = R (A P)   (mlprec/impl/mld_daggrmat_smth_asb.f90:174-401)
// C = A B on a CUDA device (mldg_spgemm), the same arrays as spgemm(a, b)
static CSR spgemm_dev(const CSR &a, const CSR &b, int device) {
  mldg_csr ac{a.nr, a.nc, a.irp.data(), a.ja.data(), a.val.data()};
  mldg_csr bc{b.nr, b.nc, b.irp.data(), b.ja.data(), b.val.data()};
  int32_t *irp = nullptr, *ja = nullptr;
  double *val = nullptr, ms = 0;
  int nr = 0, nc = 0;
  const int rc = mldg_spgemm(device, &ac, &bc, &irp, &ja, &val, &nr, &nc, &ms);
  if (rc != 0) throw std::runtime_error("sparse product on the GPU failed (code " + std::to_string(rc) + ")");
  CSR c;
  c.nr = nr;
  c.nc = nc;
  c.irp.assign(irp, irp + nr + 1);
  c.ja.assign(ja, ja + c.irp[nr]);
  c.val.assign(val, val + c.irp[nr]);
  mldg_free(irp);
  mldg_free(ja);
  mldg_free(val);
  if (std::getenv("MLDG_TIMING"))
    std::fprintf(stderr, "mldg timing: sparse product on the GPU %d x %d (%d entries): %.3f ms device\n", nr, nc,
                 c.irp[nr], ms);
  return c;
}

void smoothed_aggr_asb(const CSR &a, const std::vector<int> &ilaggr, int naggr, double &omega, int device,
                       CSR &P, CSR &R, CSR &Ac) {
  const int nr = a.nr;
  std::vector<double> dinv = diag_of(a);
  for (double &v : dinv) v = (v != 0.0) ? 1.0 / v : 1.0;
  CSR s = a;
  double anorm = 0.0;
  for (int i = 0; i < nr; ++i) {
    double rs = 0.0;
    for (int k = s.irp[i]; k < s.irp[i + 1]; ++k) {
      s.val[k] = dinv[i] * s.val[k];
      rs = rs + std::fabs(s.val[k]);
    }
    anorm = std::max(anorm, rs);
  }
  omega = 4.0 / (3.0 * anorm);
  for (int i = 0; i < nr; ++i)
    for (int k = s.irp[i]; k < s.irp[i + 1]; ++k)
      s.val[k] = (s.ja[k] == i) ? 1.0 - omega * s.val[k] : -omega * s.val[k];
  CSR pt;
  pt.nr = nr;
  pt.nc = naggr;
  pt.irp.resize((size_t)nr + 1);
  pt.ja.assign(ilaggr.begin(), ilaggr.end());
  pt.val.assign((size_t)nr, 1.0);
  for (int i = 0; i <= nr; ++i) pt.irp[i] = i;
  if (device >= 0) {
    P = spgemm_dev(s, pt, device);
    CSR ap = spgemm_dev(a, P, device);
    R = transpose(P);
    Ac = spgemm_dev(R, ap, device);
    return;
  }
  P = spgemm(s, pt);
  CSR ap = spgemm(a, P);
  R = transpose(P);
  Ac = spgemm(R, ap);
}

// ILU(0), mlprec/impl/mld_dilu0_fact.f90:284-477 (ialg = ILU_N)
// The same factorisation on a CUDA device (mldg_ilu0_factor): 0, 1 + the
// row whose pivot is too small, or -1 with msg set on a CUDA error.
int ilu0_factor_gpu(const CSR &a, CSR &L, CSR &U, std::vector<double> &d, int device, std::string &msg) {
  const int m = a.nr;
  const int64_t nz = (int64_t)a.irp[m];
  L = CSR();
  U = CSR();
  L.nr = L.nc = U.nr = U.nc = m;
  L.irp.assign((size_t)m + 1, 0);
  U.irp.assign((size_t)m + 1, 0);
  L.ja.resize((size_t)std::max<int64_t>(nz, 1));
  L.val.resize((size_t)std::max<int64_t>(nz, 1));
  U.ja.resize((size_t)std::max<int64_t>(nz, 1));
  U.val.resize((size_t)std::max<int64_t>(nz, 1));
  d.assign((size_t)m, 0.0);
  mldg_csr c{m, m, a.irp.data(), a.ja.data(), a.val.data()};
  int bad = -1;
  double ms = 0;
  const int rc = mldg_ilu0_factor(device, &c, L.irp.data(), L.ja.data(), L.val.data(), U.irp.data(), U.ja.data(),
                                  U.val.data(), d.data(), &bad, &ms);
  if (rc == 2) return 1 + bad;
  if (rc != 0) {
    msg = "ILU(0) on the GPU failed (code " + std::to_string(rc) + ")";
    return -1;
  }
  L.ja.resize((size_t)L.irp[m]);
  L.val.resize((size_t)L.irp[m]);
  U.ja.resize((size_t)U.irp[m]);
  U.val.resize((size_t)U.irp[m]);
  if (std::getenv("MLDG_TIMING"))
    std::fprintf(stderr, "mldg timing: ILU(0) on the GPU, n=%d: %.3f ms device\n", m, ms);
  return 0;
}

int ilu0_factor(const CSR &a, CSR &L, CSR &U, std::vector<double> &d) {
  const int m = a.nr;
  L = CSR();
  U = CSR();
  L.nr = L.nc = U.nr = U.nc = m;
  L.irp.assign((size_t)m + 1, 0);
  U.irp.assign((size_t)m + 1, 0);
  // split pass: sizes, then copy (ilu_copyin, :551-660)
  for (int i = 0; i < m; ++i) {
    int nl = 0, nu = 0;
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k) {
      const int j = a.ja[k];
      nl += (j < i);
      nu += (j > i && j < m);
    }
    L.irp[i + 1] = L.irp[i] + nl;
    U.irp[i + 1] = U.irp[i] + nu;
  }
  L.ja.resize((size_t)L.irp[m]);
  L.val.resize((size_t)L.irp[m]);
  U.ja.resize((size_t)U.irp[m]);
  U.val.resize((size_t)U.irp[m]);
  d.assign((size_t)m, 0.0);
  for (int i = 0; i < m; ++i) {
    int pl = L.irp[i], pu = U.irp[i];
    double dia = 0.0;
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k) {
      const int j = a.ja[k];
      if (j < i) {
        L.ja[pl] = j;
        L.val[pl++] = a.val[k];
      } else if (j == i) {
        dia = a.val[k];
      } else if (j < m) {
        U.ja[pu] = j;
        U.val[pu++] = a.val[k];
      }
    }
    const int le = L.irp[i + 1], ue = U.irp[i + 1];
    // eliminate with rows k < i, updating the pattern-matching entries only
    for (int kk = L.irp[i]; kk < le; ++kk) {
      const int k = L.ja[kk];
      const double temp = L.val[kk];
      L.val[kk] = temp * d[k];
      int p1 = kk + 1, p2 = U.irp[i];
      for (int jj = U.irp[k]; jj < U.irp[k + 1]; ++jj) {
        const int j = U.ja[jj];
        if (j < i) {
          while (p1 < le && L.ja[p1] < j) ++p1;
          if (p1 < le && L.ja[p1] == j) {
            L.val[p1] = L.val[p1] - temp * U.val[jj];
            ++p1;
          }
        } else if (j == i) {
          dia = dia - temp * U.val[jj];
        } else {
          while (p2 < ue && U.ja[p2] < j) ++p2;
          if (p2 < ue && U.ja[p2] == j) {
            U.val[p2] = U.val[p2] - temp * U.val[jj];
            ++p2;
          }
        }
      }
    }
    if (std::fabs(dia) < kEpsTol) return 1 + i;  // pivot too small (:436-445)
    dia = 1.0 / dia;
    d[i] = dia;
    for (int kk = U.irp[i]; kk < ue; ++kk) U.val[kk] = U.val[kk] * dia;
  }
  return 0;
}

// ---------------------------------------------------------------------------
int hierarchy_build(const CSR &a, const Parms &p, std::vector<Level> &lv, std::string &msg) {
  lv.clear();
  if (a.nr <= 0 || a.nc != a.nr) {
    msg = "hierarchy_build: matrix must be square and non-empty";
    return 30;
  }
  const int nplevs = std::max(2, p.max_levs);
  int64_t casize = p.min_coarse_size;
  if (casize < 0) {
    casize = (int64_t)std::pow((double)a.nr, 1.0 / 3.0);
    casize = std::max<int64_t>(casize, 1) * 40;
  }
  lv.reserve((size_t)nplevs);  // references into lv stay valid below
  lv.emplace_back();
  lv[0].A = a;
  int newsz = 0;
  for (int i = 1; i < nplevs; ++i) {
    const CSR &af = lv[i - 1].A;
    std::vector<int> il;
    int na = 0;
    if (dec_aggregate(af, p.aggr_thresh, il, na) != 0) {
      msg = "aggregation left unaggregated rows";
      return 4000;
    }
    const double ratio = (double)af.nr / (double)na;
    if (na <= casize) newsz = i;
    if (i > 1) {
      if (ratio < p.min_cr_ratio) newsz = (ratio > 1) ? i : i - 1;
      if (na == lv[i - 1].naggr) newsz = i - 1;
    }
    if (newsz > 0 && newsz < i) break;  // the previous level becomes the coarsest
    lv.emplace_back();
    Level &L = lv.back();
    L.ilaggr = std::move(il);
    L.naggr = na;
    try {
      smoothed_aggr_asb(af, L.ilaggr, na, L.omega, p.setup_device, L.P, L.R, L.A);
    } catch (const std::exception &e) {
      msg = e.what();
      return 2;
    }
    if (newsz > 0) break;
  }
  return 0;
}

int smoothers_build(std::vector<Level> &lv, const Parms &p, std::string &msg) {
  const int nlev = (int)lv.size();
  for (int l = 0; l < nlev; ++l) {
    Level &L = lv[l];
    const bool coarse = (l == nlev - 1) && nlev > 1;
    L.kind = coarse ? p.coarse_solver : p.smoother;
    L.sweeps_pre = coarse ? p.coarse_sweeps : p.sweeps_pre;
    L.sweeps_post = coarse ? p.coarse_sweeps : p.sweeps_post;
    L.damping = p.damping;
    const CSR &a = L.A;
    const int n = a.nr;
    L.ND = CSR();
    L.L = CSR();
    L.U = CSR();
    if (L.kind == SM_JACOBI) {
      // ND = A - diag(A) (clip_diag); d = 1/a_ii, 0 -> 1
      L.ND.nr = L.ND.nc = n;
      L.ND.irp.assign((size_t)n + 1, 0);
      for (int i = 0; i < n; ++i) {
        int c = 0;
        for (int k = a.irp[i]; k < a.irp[i + 1]; ++k) c += (a.ja[k] != i);
        L.ND.irp[i + 1] = L.ND.irp[i] + c;
      }
      L.ND.ja.reserve((size_t)L.ND.irp[n]);
      L.ND.val.reserve((size_t)L.ND.irp[n]);
      for (int i = 0; i < n; ++i)
        for (int k = a.irp[i]; k < a.irp[i + 1]; ++k)
          if (a.ja[k] != i) {
            L.ND.ja.push_back(a.ja[k]);
            L.ND.val.push_back(a.val[k]);
          }
      L.d = diag_of(a);
      for (double &v : L.d) v = (v == 0.0) ? 1.0 : 1.0 / v;
    } else if (L.kind == SM_BJAC) {
      // one rank: the off-block part (columns > nrow) is empty
      const int rc = p.setup_device >= 0 ? ilu0_factor_gpu(a, L.L, L.U, L.d, p.setup_device, msg)
                                       : ilu0_factor(a, L.L, L.U, L.d);
      if (rc < 0) return 2;
      if (rc != 0) {
        msg = "ILU(0): pivot too small at level " + std::to_string(l) + " row " + std::to_string(rc - 1);
        return 2;
      }
    } else if (L.kind == SM_FBGS) {
      // GS / BWGS solvers (mld_d_gs_solver_bld.f90:73-81): strict lower and
      // strict upper triangles and the diagonal; the GS solve divides by a_ii
      L.L.nr = L.L.nc = L.U.nr = L.U.nc = n;
      L.L.irp.assign((size_t)n + 1, 0);
      L.U.irp.assign((size_t)n + 1, 0);
      L.d.assign((size_t)n, 0.0);
      for (int i = 0; i < n; ++i) {
        for (int k = a.irp[i]; k < a.irp[i + 1]; ++k) {
          const int j = a.ja[k];
          if (j < i) {
            L.L.ja.push_back(j);
            L.L.val.push_back(a.val[k]);
          } else if (j > i) {
            L.U.ja.push_back(j);
            L.U.val.push_back(a.val[k]);
          } else {
            L.d[i] = a.val[k];
          }
        }
        L.L.irp[i + 1] = (int)L.L.ja.size();
        L.U.irp[i + 1] = (int)L.U.ja.size();
        if (L.d[i] == 0.0) {
          msg = "Gauss-Seidel: zero diagonal at level " + std::to_string(l) + " row " + std::to_string(i);
          return 2;
        }
      }
    } else {
      msg = "unsupported smoother kind";
      return 30;
    }
  }
  return 0;
}

}  // namespace mld
