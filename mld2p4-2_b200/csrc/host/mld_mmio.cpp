// mld_mmio.cpp -- MatrixMarket I/O of a whole hierarchy in the file layout of
// the reference's prec%dump (mlprec/mld_d_prec_type.f90:698-729), so that a
// hierarchy built by a real MLD2P4 installation can be handed to the GPU
// apply unchanged, and one built here can be inspected with the reference's
// tools.
//
// File names (rank 0 of one process, levels numbered from 1 = finest):
//   <prefix>_p000_l<LLL>_ac.mtx, _r.mtx, _p.mtx      level >= 2
//     (mld_d_base_onelev_dump.f90:112-121: ac, map_X2Y, map_Y2X)
//   <prefix>_sm_p000_l<LLL>_nd.mtx                   jac smoother ND
//     (mld_d_jac_smoother_dmp.f90:75-79)
//   <prefix>_sm_p000_l<LLL>_lower.mtx, _diag.mtx, _upper.mtx
//     ILU solver (mld_d_ilu_solver_dmp.f90:40-48): unit L, 1/pivot, scaled U
//   <prefix>_sm_p000_l<LLL>_diag.mtx                 diag solver (1/a_ii)
//     (mld_d_diag_solver_dmp.f90:77-79)
//   <prefix>_sm_p000_l<LLL>_lower/_upper.mtx         GS solver: tril(A) with
//   <prefix>_sm2a_p000_l<LLL>_lower/_upper.mtx       the diagonal / strict
//     upper; BWGS solver: strict lower / triu(A) with the diagonal
//     (mld_d_gs_solver_dmp.f90:77-82, mld_d_base_onelev_dump.f90:126-129)
// Sparse files are "coordinate real general" (1-based), vectors "array real
// general", as PSBLAS prints them.
#include "mld_mmio.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace mld {

namespace {

std::string lower_str(std::string s) {
  for (char &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

}  // namespace

bool file_exists(const std::string &f) {
  std::ifstream in(f);
  return (bool)in;
}

std::string dump_name(const std::string &prefix, const char *part, int level, const char *what) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "_p000_l%03d_%s.mtx", level, what);
  return prefix + part + buf;
}

int read_mm_csr(const std::string &fname, CSR &a, std::string &msg) {
  std::ifstream in(fname);
  if (!in) {
    msg = "cannot open " + fname;
    return 1;
  }
  std::string line;
  if (!std::getline(in, line) || lower_str(line).find("%%matrixmarket matrix coordinate") != 0) {
    msg = fname + ": not a MatrixMarket coordinate matrix";
    return 2;
  }
  const bool symmetric = lower_str(line).find("symmetric") != std::string::npos;
  while (std::getline(in, line))
    if (!line.empty() && line[0] != '%') break;
  long nr = 0, nc = 0, nz = 0;
  {
    std::istringstream hs(line);
    if (!(hs >> nr >> nc >> nz) || nr < 0 || nc < 0 || nz < 0) {
      msg = fname + ": bad size line";
      return 3;
    }
  }
  std::vector<int> ri, ci;
  std::vector<double> vv;
  ri.reserve((size_t)nz * (symmetric ? 2 : 1));
  for (long k = 0; k < nz; ++k) {
    long i, j;
    double v;
    if (!(in >> i >> j >> v) || i < 1 || i > nr || j < 1 || j > nc) {
      msg = fname + ": bad entry " + std::to_string(k + 1);
      return 4;
    }
    ri.push_back((int)(i - 1));
    ci.push_back((int)(j - 1));
    vv.push_back(v);
    if (symmetric && i != j) {
      ri.push_back((int)(j - 1));
      ci.push_back((int)(i - 1));
      vv.push_back(v);
    }
  }
  // CSR with rows sorted by column; duplicates are summed (coordinate semantics)
  a.nr = (int)nr;
  a.nc = (int)nc;
  a.irp.assign((size_t)nr + 1, 0);
  for (int i : ri) a.irp[(size_t)i + 1]++;
  for (long i = 0; i < nr; ++i) a.irp[(size_t)i + 1] += a.irp[(size_t)i];
  std::vector<int> pos(a.irp.begin(), a.irp.end() - 1), ja(ri.size());
  std::vector<double> val(ri.size());
  for (size_t k = 0; k < ri.size(); ++k) {
    const int p = pos[(size_t)ri[k]]++;
    ja[(size_t)p] = ci[k];
    val[(size_t)p] = vv[k];
  }
  a.ja.clear();
  a.val.clear();
  std::vector<int> irp2((size_t)nr + 1, 0);
  std::vector<std::pair<int, double>> row;
  for (long i = 0; i < nr; ++i) {
    row.clear();
    for (int k = a.irp[(size_t)i]; k < a.irp[(size_t)i + 1]; ++k) row.push_back({ja[(size_t)k], val[(size_t)k]});
    std::stable_sort(row.begin(), row.end(), [](const std::pair<int, double> &x, const std::pair<int, double> &y) {
      return x.first < y.first;
    });
    for (size_t q = 0; q < row.size(); ++q) {
      if (q > 0 && row[q].first == row[q - 1].first) {
        a.val.back() += row[q].second;
      } else {
        a.ja.push_back(row[q].first);
        a.val.push_back(row[q].second);
      }
    }
    irp2[(size_t)i + 1] = (int)a.ja.size();
  }
  a.irp = irp2;
  return 0;
}

int write_mm_csr(const std::string &fname, const CSR &a, const std::string &head, std::string &msg) {
  FILE *f = std::fopen(fname.c_str(), "w");
  if (!f) {
    msg = "cannot write " + fname;
    return 1;
  }
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%% %s\n%%\n", head.c_str());
  std::fprintf(f, "%d %d %lld\n", a.nr, a.nc, (long long)a.nnz());
  for (int i = 0; i < a.nr; ++i)
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k) std::fprintf(f, "%d %d %.17g\n", i + 1, a.ja[k] + 1, a.val[k]);
  const bool ok = std::fclose(f) == 0;
  if (!ok) msg = "error writing " + fname;
  return ok ? 0 : 2;
}

int read_mm_vec(const std::string &fname, std::vector<double> &v, std::string &msg) {
  std::ifstream in(fname);
  if (!in) {
    msg = "cannot open " + fname;
    return 1;
  }
  std::string line;
  if (!std::getline(in, line) || lower_str(line).find("%%matrixmarket matrix array") != 0) {
    msg = fname + ": not a MatrixMarket array";
    return 2;
  }
  while (std::getline(in, line))
    if (!line.empty() && line[0] != '%') break;
  long nr = 0, nc = 0;
  std::istringstream hs(line);
  if (!(hs >> nr >> nc) || nr < 0 || nc != 1) {
    msg = fname + ": expected one column";
    return 3;
  }
  v.resize((size_t)nr);
  for (long i = 0; i < nr; ++i)
    if (!(in >> v[(size_t)i])) {
      msg = fname + ": short array";
      return 4;
    }
  return 0;
}

int write_mm_vec(const std::string &fname, const std::vector<double> &v, const std::string &head,
                 std::string &msg) {
  FILE *f = std::fopen(fname.c_str(), "w");
  if (!f) {
    msg = "cannot write " + fname;
    return 1;
  }
  std::fprintf(f, "%%%%MatrixMarket matrix array real general\n%% %s\n%%\n%zu 1\n", head.c_str(), v.size());
  for (double x : v) std::fprintf(f, "%.17g\n", x);
  const bool ok = std::fclose(f) == 0;
  if (!ok) msg = "error writing " + fname;
  return ok ? 0 : 2;
}

// lower/upper triangle with or without the diagonal
static CSR tri_part(const CSR &a, bool lower, bool with_diag, const std::vector<double> *d) {
  CSR t;
  t.nr = a.nr;
  t.nc = a.nc;
  t.irp.assign((size_t)a.nr + 1, 0);
  for (int i = 0; i < a.nr; ++i) {
    bool diag_done = !with_diag;
    auto put_diag = [&]() {
      if (!diag_done && d) {
        t.ja.push_back(i);
        t.val.push_back((*d)[(size_t)i]);
      }
      diag_done = true;
    };
    if (!lower) put_diag();
    for (int k = a.irp[i]; k < a.irp[i + 1]; ++k) {
      const int j = a.ja[k];
      if ((lower && j < i) || (!lower && j > i)) {
        t.ja.push_back(j);
        t.val.push_back(a.val[k]);
      }
    }
    if (lower) put_diag();
    t.irp[(size_t)i + 1] = (int)t.ja.size();
  }
  return t;
}

int dump_hierarchy(const std::vector<Level> &lv, const std::string &prefix, std::string &msg) {
  const std::string head = "MLD2P4 hierarchy (GPU drop-in host build)";
  int rc = 0;
  for (size_t l = 0; l < lv.size() && rc == 0; ++l) {
    const Level &L = lv[l];
    const int lev = (int)l + 1;
    if (lev >= 2) {
      rc = write_mm_csr(dump_name(prefix, "", lev, "ac"), L.A, head, msg);
      if (!rc) rc = write_mm_csr(dump_name(prefix, "", lev, "r"), L.R, head, msg);
      if (!rc) rc = write_mm_csr(dump_name(prefix, "", lev, "p"), L.P, head, msg);
    }
    if (rc) break;
    if (L.kind == SM_BJAC) {
      CSR nd;
      nd.nr = nd.nc = L.A.nr;
      nd.irp.assign((size_t)L.A.nr + 1, 0);
      rc = write_mm_csr(dump_name(prefix, "_sm", lev, "nd"), L.ND.present() ? L.ND : nd, head, msg);
      if (!rc) rc = write_mm_csr(dump_name(prefix, "_sm", lev, "lower"), L.L, head, msg);
      if (!rc) rc = write_mm_vec(dump_name(prefix, "_sm", lev, "diag"), L.d, head, msg);
      if (!rc) rc = write_mm_csr(dump_name(prefix, "_sm", lev, "upper"), L.U, head, msg);
    } else if (L.kind == SM_JACOBI) {
      rc = write_mm_csr(dump_name(prefix, "_sm", lev, "nd"), L.ND, head, msg);
      if (!rc) rc = write_mm_vec(dump_name(prefix, "_sm", lev, "diag"), L.d, head, msg);
    } else if (L.kind == SM_FBGS) {
      // GS: tril(A) with the diagonal + strict upper; BWGS: strict lower + triu(A) with the diagonal
      rc = write_mm_csr(dump_name(prefix, "_sm", lev, "lower"), tri_part(L.L, true, true, &L.d), head, msg);
      if (!rc) rc = write_mm_csr(dump_name(prefix, "_sm", lev, "upper"), L.U, head, msg);
      if (!rc) rc = write_mm_csr(dump_name(prefix, "_sm2a", lev, "lower"), L.L, head, msg);
      if (!rc) rc = write_mm_csr(dump_name(prefix, "_sm2a", lev, "upper"), tri_part(L.U, false, true, &L.d), head, msg);
    }
  }
  return rc;
}

int load_hierarchy(const std::string &prefix, int nlev, const CSR &a0, const Parms &p, std::vector<Level> &lv,
                   std::string &msg) {
  if (nlev < 1) {
    msg = "load: nlev < 1";
    return 30;
  }
  lv.assign((size_t)nlev, Level());
  lv[0].A = a0;
  for (int l = 0; l < nlev; ++l) {
    Level &L = lv[(size_t)l];
    const int lev = l + 1;
    int rc = 0;
    if (lev >= 2) {
      rc = read_mm_csr(dump_name(prefix, "", lev, "ac"), L.A, msg);
      if (!rc) rc = read_mm_csr(dump_name(prefix, "", lev, "r"), L.R, msg);
      if (!rc) rc = read_mm_csr(dump_name(prefix, "", lev, "p"), L.P, msg);
      if (rc) return 30;
    }
    const bool coarse = (l == nlev - 1) && nlev > 1;
    L.sweeps_pre = coarse ? p.coarse_sweeps : p.sweeps_pre;
    L.sweeps_post = coarse ? p.coarse_sweeps : p.sweeps_post;
    L.damping = p.damping;
    const std::string lo = dump_name(prefix, "_sm", lev, "lower"), up = dump_name(prefix, "_sm", lev, "upper");
    const std::string dg = dump_name(prefix, "_sm", lev, "diag"), nd = dump_name(prefix, "_sm", lev, "nd");
    if (file_exists(dump_name(prefix, "_sm2a", lev, "lower"))) {
      // FBGS: the GS solver's tril(A) with the diagonal gives L and d
      CSR gl, gu;
      rc = read_mm_csr(lo, gl, msg);
      if (!rc) rc = read_mm_csr(up, gu, msg);
      if (rc) return 30;
      L.kind = SM_FBGS;
      L.L = tri_part(gl, true, false, nullptr);
      L.U = tri_part(gu, false, false, nullptr);
      L.d.assign((size_t)gl.nr, 0.0);
      for (int i = 0; i < gl.nr; ++i)
        for (int k = gl.irp[i]; k < gl.irp[i + 1]; ++k)
          if (gl.ja[k] == i) L.d[(size_t)i] = gl.val[k];
    } else if (file_exists(lo)) {
      L.kind = SM_BJAC;
      rc = read_mm_csr(lo, L.L, msg);
      if (!rc) rc = read_mm_csr(up, L.U, msg);
      if (!rc) rc = read_mm_vec(dg, L.d, msg);
      if (!rc && file_exists(nd)) rc = read_mm_csr(nd, L.ND, msg);
      if (rc) return 30;
      if (L.ND.present() && L.ND.nnz() == 0) L.ND = CSR();
    } else if (file_exists(dg)) {
      L.kind = SM_JACOBI;
      rc = read_mm_vec(dg, L.d, msg);
      if (!rc && file_exists(nd)) rc = read_mm_csr(nd, L.ND, msg);
      if (rc) return 30;
      if (!L.ND.present()) {
        // A without its diagonal (clip_diag)
        L.ND = tri_part(L.A, true, false, nullptr);
        CSR up2 = tri_part(L.A, false, false, nullptr);
        CSR m;
        m.nr = m.nc = L.A.nr;
        m.irp.assign((size_t)m.nr + 1, 0);
        for (int i = 0; i < m.nr; ++i) {
          for (int k = L.ND.irp[i]; k < L.ND.irp[i + 1]; ++k) {
            m.ja.push_back(L.ND.ja[k]);
            m.val.push_back(L.ND.val[k]);
          }
          for (int k = up2.irp[i]; k < up2.irp[i + 1]; ++k) {
            m.ja.push_back(up2.ja[k]);
            m.val.push_back(up2.val[k]);
          }
          m.irp[(size_t)i + 1] = (int)m.ja.size();
        }
        L.ND = m;
      }
    } else {
      msg = "load: no smoother files for level " + std::to_string(lev) + " (" + lo + ", " + dg + ")";
      return 30;
    }
  }
  return 0;
}

}  // namespace mld
