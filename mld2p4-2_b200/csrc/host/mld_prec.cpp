// mld_prec.cpp -- host-side mirror of mld_dprec_type (see include/mld_prec.h).
//
// Keeps the reference's object protocol: init fills defaults, set routes
// keywords, hierarchy_build / smoothers_build produce the level data on the
// host, and the smoothers build hands the frozen hierarchy to the GPU through
// the mldg C ABI.  apply and the Krylov driver then run on the device.
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mld_hier.h"
#include "mld_mmio.h"
#include "mld_prec.h"
#include "mldg.h"

struct mldp_prec {
  int device = 0;
  bool inited = false;
  std::string ptype;
  mld::Parms parms;
  std::string unsupported;      // first unsupported setting, reported at build
  int precision = MLDG_PREC_FP64;
  int cycle = MLDG_CYCLE_V;
  std::vector<mld::Level> lv;
  bool hier_built = false, smoothers_built = false;
  mldg_handle *gpu = nullptr;
  std::string err;
};

namespace {

std::string upper(const char *s) {
  std::string r = s ? s : "";
  for (char &c : r) c = (char)std::toupper((unsigned char)c);
  while (!r.empty() && r.back() == ' ') r.pop_back();
  return r;
}

int fail(mldp_prec *p, int code, const std::string &m) {
  if (p) p->err = m;
  return code;
}

mld::CSR make_csr(int n, const int32_t *irp, const int32_t *ja, const double *val) {
  mld::CSR a;
  a.nr = a.nc = n;
  a.irp.assign(irp, irp + n + 1);
  a.ja.assign(ja, ja + irp[n]);
  a.val.assign(val, val + irp[n]);
  return a;
}

mldg_csr view(const mld::CSR &c) {
  mldg_csr v;
  v.nrows = c.nr;
  v.ncols = c.nc;
  v.irp = c.present() ? c.irp.data() : nullptr;
  v.ja = c.ja.data();
  v.val = c.val.data();
  return v;
}

// string values -> keyword codes (mld_stringval, mld_base_prec_type.F90:378-485)
int smoother_code(const std::string &v) {
  if (v == "JACOBI" || v == "DIAG") return mld::SM_JACOBI;
  if (v == "BJAC" || v == "ILU") return mld::SM_BJAC;
  return -1;
}

}  // namespace

extern "C" int mldp_create(mldp_prec **out, int device) {
  if (!out) return MLDG_ERR_ARG;
  *out = new mldp_prec();
  (*out)->device = device;
  return 0;
}

extern "C" int mldp_init(mldp_prec *p, const char *ptype) {
  if (!p) return MLDG_ERR_ARG;
  const std::string t = upper(ptype);
  p->parms = mld::Parms();
  p->lv.clear();
  p->hier_built = p->smoothers_built = false;
  p->unsupported.clear();
  p->precision = MLDG_PREC_FP64;
  p->cycle = MLDG_CYCLE_V;
  if (t == "ML") {
    // mld_dprecinit.F90:188-207: VCYCLE, FBGS smoother, ILU coarse solver
    // (no UMFPACK/MUMPS/SuperLU): BJAC + ILU(0), replicated coarse matrix.
    p->parms.max_levs = 20;
    p->parms.smoother = mld::SM_FBGS;
    p->parms.coarse_solver = mld::SM_BJAC;
    p->parms.coarse_sweeps = 1;
  } else if (t == "BJAC" || t == "JACOBI") {
    p->parms.max_levs = 1;
    p->parms.smoother = smoother_code(t);
  } else if (t == "FBGS") {
    // mld_dprecinit.F90:162-166: one level, forward GS then backward GS
    p->parms.max_levs = 1;
    p->parms.smoother = mld::SM_FBGS;
  } else {
    return fail(p, MLDG_ERR_ARG, "init: unknown preconditioner type '" + t + "'");
  }
  p->ptype = t;
  p->inited = true;
  return 0;
}

static int set_common(mldp_prec *p, const std::string &w, const std::string *sv, const int *iv,
                      const double *rv, int ilev) {
  if (!p) return MLDG_ERR_ARG;
  if (!p->inited) return fail(p, 3111, "set before init");
  if (ilev >= 0) return fail(p, MLDG_ERR_ARG, "set: per-level settings (ilev) are not supported");
  mld::Parms &q = p->parms;
  auto ival = [&]() -> int { return iv ? *iv : (rv ? (int)*rv : std::atoi(sv->c_str())); };
  auto rval = [&]() -> double { return rv ? *rv : (iv ? (double)*iv : std::atof(sv->c_str())); };
  auto need = [&](const char *expect) {
    if (!sv || upper(sv->c_str()) != expect) {
      if (p->unsupported.empty()) p->unsupported = w + "=" + (sv ? *sv : std::to_string(ival()));
    }
  };
  if (w == "SMOOTHER_TYPE") {
    const std::string v = sv ? upper(sv->c_str()) : "";
    const int c = v == "FBGS" ? (int)mld::SM_FBGS : smoother_code(v);
    if (c < 0) {
      if (p->unsupported.empty()) p->unsupported = w + "=" + v;
    } else {
      q.smoother = c;
    }
  } else if (w == "SUB_SOLVE") {
    const int c = smoother_code(sv ? upper(sv->c_str()) : "");
    if (c < 0) {
      if (p->unsupported.empty()) p->unsupported = w;
    } else {
      q.smoother = c;
    }
  } else if (w == "SMOOTHER_SWEEPS") {
    q.sweeps_pre = q.sweeps_post = ival();
  } else if (w == "SMOOTHER_DAMPING") {  // extension
    q.damping = rval();
  } else if (w == "SUB_FILLIN" || w == "COARSE_FILLIN") {
    if (ival() != 0 && p->unsupported.empty()) p->unsupported = w + " > 0 (ILU(k))";
  } else if (w == "ML_CYCLE") {
    const std::string v = sv ? upper(sv->c_str()) : "";
    if (v == "VCYCLE" || v == "MULT")
      p->cycle = MLDG_CYCLE_V;
    else if (v == "WCYCLE")
      p->cycle = MLDG_CYCLE_W;
    else if (v == "KCYCLE")
      p->cycle = MLDG_CYCLE_K;
    else if (v == "KCYCLESYM")
      p->cycle = MLDG_CYCLE_KSYM;
    else if (v == "ADD")
      p->cycle = MLDG_CYCLE_ADD;
    else if (p->unsupported.empty())
      p->unsupported = w + "=" + v;
  } else if (w == "COARSE_SOLVE") {
    const std::string v = sv ? upper(sv->c_str()) : "";
    if (v == "BJAC" || v == "ILU")
      q.coarse_solver = mld::SM_BJAC;
    else if (v == "JACOBI")
      q.coarse_solver = mld::SM_JACOBI;
    else if (p->unsupported.empty())
      p->unsupported = w + "=" + v;
  } else if (w == "COARSE_SUBSOLVE") {
    const int c = smoother_code(sv ? upper(sv->c_str()) : "");
    if (c < 0) {
      if (p->unsupported.empty()) p->unsupported = w;
    } else {
      q.coarse_solver = c;
    }
  } else if (w == "COARSE_SWEEPS") {
    q.coarse_sweeps = ival();
  } else if (w == "COARSE_MAT") {
    // DIST / REPL coincide on one rank
  } else if (w == "MIN_COARSE_SIZE") {
    q.min_coarse_size = std::max(ival(), -1);
  } else if (w == "MAX_LEVS") {
    q.max_levs = std::max(ival(), 1);
  } else if (w == "MIN_CR_RATIO") {
    q.min_cr_ratio = rval();
  } else if (w == "AGGR_THRESH") {
    q.aggr_thresh = rval();
  } else if (w == "OUTER_SWEEPS") {
    if (ival() != 1 && p->unsupported.empty()) p->unsupported = "OUTER_SWEEPS != 1";
  } else if (w == "AGGR_PROL") {
    need("SMOOTHED");
  } else if (w == "PAR_AGGR_ALG") {
    need("DEC");
  } else if (w == "AGGR_ORD") {
    need("NATURAL");
  } else if (w == "AGGR_FILTER") {
    need("NOFILTER");
  } else if (w == "AGGR_OMEGA_ALG") {
    need("EIG_EST");
  } else if (w == "AGGR_EIG") {
    need("MAX_NORM");
  } else if (w == "PRECISION") {  // extension: FP64 | FP32 | FP32_P16 | FP32_H16
    const std::string v = sv ? upper(sv->c_str()) : "";
    if (v == "FP64")
      p->precision = MLDG_PREC_FP64;
    else if (v == "FP32")
      p->precision = MLDG_PREC_FP32;
    else if (v == "FP32_P16")
      p->precision = MLDG_PREC_FP32_P16;
    else if (v == "FP32_H16")
      p->precision = MLDG_PREC_FP32_H16;
    else
      return fail(p, MLDG_ERR_ARG, "set PRECISION: unknown value " + v);
  } else if (w == "SETUP_DEVICE") {  // extension: HOST | GPU (sparse products and ILU(0) on the GPU)
    const std::string v = sv ? upper(sv->c_str()) : "";
    if (v == "HOST")
      p->parms.setup_device = -1;
    else if (v == "GPU")
      p->parms.setup_device = p->device;
    else
      return fail(p, MLDG_ERR_ARG, "set SETUP_DEVICE: unknown value " + v);
  } else {
    return fail(p, MLDG_ERR_ARG, "set: unknown keyword " + w);
  }
  return 0;
}

extern "C" int mldp_seti(mldp_prec *p, const char *what, int val, int ilev) {
  return set_common(p, upper(what), nullptr, &val, nullptr, ilev);
}
extern "C" int mldp_setr(mldp_prec *p, const char *what, double val, int ilev) {
  return set_common(p, upper(what), nullptr, nullptr, &val, ilev);
}
extern "C" int mldp_setc(mldp_prec *p, const char *what, const char *val, int ilev) {
  const std::string s = val ? val : "";
  return set_common(p, upper(what), &s, nullptr, nullptr, ilev);
}

extern "C" int mldp_hierarchy_build(mldp_prec *p, int n, const int32_t *irp, const int32_t *ja,
                                    const double *val) {
  if (!p) return MLDG_ERR_ARG;
  if (!p->inited) return fail(p, 3111, "hierarchy_build before init");
  if (n <= 0 || !irp || !ja || !val) return fail(p, MLDG_ERR_ARG, "hierarchy_build: bad matrix");
  if (!p->unsupported.empty())
    return fail(p, MLDG_ERR_ARG, "setting not supported by the GPU apply: " + p->unsupported);
  mld::CSR a = make_csr(n, irp, ja, val);
  p->hier_built = p->smoothers_built = false;
  std::string msg;
  int rc;
  if (p->parms.max_levs <= 1) {
    p->lv.assign(1, mld::Level());
    p->lv[0].A = std::move(a);
    rc = 0;
  } else {
    rc = mld::hierarchy_build(a, p->parms, p->lv, msg);
  }
  if (rc) return fail(p, rc, msg);
  p->hier_built = true;
  return 0;
}

static int upload_all(mldp_prec *p);

extern "C" int mldp_smoothers_build(mldp_prec *p) {
  if (!p) return MLDG_ERR_ARG;
  if (!p->hier_built) return fail(p, 3112, "smoothers_build before hierarchy_build");
  std::string msg;
  const auto t0 = std::chrono::steady_clock::now();
  int rc = mld::smoothers_build(p->lv, p->parms, msg);
  if (rc) return fail(p, rc, msg);
  const auto t1 = std::chrono::steady_clock::now();
  rc = upload_all(p);
  if (std::getenv("MLDG_TIMING"))
    std::fprintf(stderr, "mldg timing: host smoothers (ILU(0), GS split) %.3f s, upload + finalize %.3f s\n",
                 std::chrono::duration<double>(t1 - t0).count(),
                 std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count());
  return rc;
}

extern "C" int mldp_smoothers_build_host(mldp_prec *p) {
  if (!p) return MLDG_ERR_ARG;
  if (!p->hier_built) return fail(p, 3112, "smoothers_build before hierarchy_build");
  std::string msg;
  const int rc = mld::smoothers_build(p->lv, p->parms, msg);
  return rc ? fail(p, rc, msg) : 0;
}

// the finished host levels -> the GPU handle (mldg_upload_level + finalize)
static int upload_all(mldp_prec *p) {
  int rc = 0;
  if (!p->gpu) {
    mldg_opts o;
    o.device = p->device;
    o.index_base = 0;
    o.use_graphs = 1;
    o.autotune = 1;
    rc = mldg_create(&p->gpu, &o);
    if (rc) return fail(p, rc, "mldg_create failed");
  }
  const int nlev = (int)p->lv.size();
  for (int l = 0; l < nlev; ++l) {
    const mld::Level &L = p->lv[l];
    mldg_level_desc d;
    std::memset(&d, 0, sizeof d);
    d.A = view(L.A);
    d.P = view(L.P);
    d.R = view(L.R);
    d.ND = view(L.ND);
    d.L = view(L.L);
    d.U = view(L.U);
    d.d = L.d.data();
    d.smoother_kind = L.kind;
    d.sweeps_pre = L.sweeps_pre;
    d.sweeps_post = L.sweeps_post;
    d.damping = L.damping;
    rc = mldg_upload_level(p->gpu, l, &d);
    if (rc) return fail(p, rc, mldg_last_error(p->gpu));
  }
  rc = mldg_set_cycle(p->gpu, p->cycle);
  if (rc == 0) rc = mldg_finalize(p->gpu, nlev, p->precision);
  if (rc) return fail(p, rc, mldg_last_error(p->gpu));
  p->smoothers_built = true;
  return 0;
}

extern "C" int mldp_dump(const mldp_prec *p, const char *prefix) {
  if (!p || !prefix) return MLDG_ERR_ARG;
  if (!p->smoothers_built) return MLDG_ERR_NOT_BUILT;
  std::string msg;
  const int rc = mld::dump_hierarchy(p->lv, prefix, msg);
  if (rc) {
    const_cast<mldp_prec *>(p)->err = msg;
    return MLDG_ERR_ARG;
  }
  return 0;
}

extern "C" int mldp_load_dump(mldp_prec *p, const char *prefix, int nlev, int n, const int32_t *irp,
                              const int32_t *ja, const double *val) {
  if (!p || !prefix) return MLDG_ERR_ARG;
  if (!p->inited) return fail(p, 3111, "load_dump before init");
  if (n <= 0 || !irp || !ja || !val) return fail(p, MLDG_ERR_ARG, "load_dump: bad matrix");
  if (!p->unsupported.empty())
    return fail(p, MLDG_ERR_ARG, "setting not supported by the GPU apply: " + p->unsupported);
  mld::CSR a = make_csr(n, irp, ja, val);
  std::string msg;
  p->hier_built = p->smoothers_built = false;
  const int rc = mld::load_hierarchy(prefix, nlev, a, p->parms, p->lv, msg);
  if (rc) return fail(p, rc, msg);
  p->hier_built = true;
  return upload_all(p);
}

extern "C" int mldp_build(mldp_prec *p, int n, const int32_t *irp, const int32_t *ja,
                          const double *val) {
  int rc = mldp_hierarchy_build(p, n, irp, ja, val);
  if (rc) return rc;
  return mldp_smoothers_build(p);
}

extern "C" int mldp_apply(mldp_prec *p, const double *x, double *y, char trans, int mem_kind) {
  if (!p) return MLDG_ERR_ARG;
  if (!p->smoothers_built) return fail(p, MLDG_ERR_NOT_BUILT, "apply before build");
  const int rc = mldg_apply(p->gpu, x, y, trans, 1, p->lv[0].A.nr, mem_kind);
  if (rc) return fail(p, rc, mldg_last_error(p->gpu));
  return 0;
}

extern "C" int mldp_krylov(mldp_prec *p, const char *method, int n, const int32_t *irp,
                           const int32_t *ja, const double *val, const double *b, double *x,
                           double eps, int itmax, int *iters, double *err, int mem_kind) {
  if (!p) return MLDG_ERR_ARG;
  if (!p->smoothers_built) return fail(p, MLDG_ERR_NOT_BUILT, "krylov before build");
  const std::string m = upper(method);
  int mc;
  if (m == "CG")
    mc = 0;
  else if (m == "FCG")
    mc = 1;
  else
    return fail(p, MLDG_ERR_ARG, "krylov: method " + m + " not available (CG, FCG)");
  mldg_csr A;
  const mldg_csr *Ap = nullptr;
  if (irp) {
    A.nrows = A.ncols = n;
    A.irp = irp;
    A.ja = ja;
    A.val = val;
    Ap = &A;
  }
  const int rc = mldg_krylov(p->gpu, mc, Ap, b, x, eps, itmax, iters, err, mem_kind);
  if (rc) return fail(p, rc, mldg_last_error(p->gpu));
  return 0;
}

extern "C" int mldp_nlev(const mldp_prec *p) { return p ? (int)p->lv.size() : 0; }

extern "C" int mldp_level_info(const mldp_prec *p, int l, int64_t *info, double *dinfo) {
  if (!p || l < 0 || l >= (int)p->lv.size() || !info) return MLDG_ERR_ARG;
  const mld::Level &L = p->lv[l];
  info[0] = L.A.nr;
  info[1] = L.A.nnz();
  info[2] = L.P.nnz();
  info[3] = L.R.nnz();
  info[4] = L.L.nnz();
  info[5] = L.U.nnz();
  info[6] = L.ND.nnz();
  info[7] = L.naggr;
  info[8] = L.kind;
  info[9] = L.sweeps_pre;
  if (dinfo) {
    dinfo[0] = L.omega;
    dinfo[1] = L.damping;
  }
  return 0;
}

extern "C" int mldp_level_csr(const mldp_prec *p, int l, const char *which, int32_t *irp,
                              int32_t *ja, double *val) {
  if (!p || l < 0 || l >= (int)p->lv.size()) return MLDG_ERR_ARG;
  const mld::Level &L = p->lv[l];
  const std::string w = upper(which);
  const mld::CSR *c = w == "A" ? &L.A : w == "P" ? &L.P : w == "R" ? &L.R : w == "L" ? &L.L
                      : w == "U" ? &L.U : w == "ND" ? &L.ND : nullptr;
  if (!c || !c->present()) return MLDG_ERR_ARG;
  std::copy(c->irp.begin(), c->irp.end(), irp);
  std::copy(c->ja.begin(), c->ja.end(), ja);
  std::copy(c->val.begin(), c->val.end(), val);
  return 0;
}

extern "C" int mldp_level_vec(const mldp_prec *p, int l, const char *which, double *dv,
                              int32_t *iv) {
  if (!p || l < 0 || l >= (int)p->lv.size()) return MLDG_ERR_ARG;
  const mld::Level &L = p->lv[l];
  const std::string w = upper(which);
  if (w == "D") {
    if (L.d.empty()) return MLDG_ERR_ARG;
    std::copy(L.d.begin(), L.d.end(), dv);
  } else if (w == "ILAGGR") {
    if (L.ilaggr.empty()) return MLDG_ERR_ARG;
    std::copy(L.ilaggr.begin(), L.ilaggr.end(), iv);
  } else {
    return MLDG_ERR_ARG;
  }
  return 0;
}

extern "C" int mldp_descr(const mldp_prec *p, char *buf, int len) {
  if (!p || !buf || len <= 0) return MLDG_ERR_ARG;
  std::string s = "Multilevel preconditioner (GPU V-cycle apply)\n";
  char line[256];
  const char *prec = p->precision == MLDG_PREC_FP64 ? "FP64"
                     : p->precision == MLDG_PREC_FP32     ? "FP32"
                     : p->precision == MLDG_PREC_FP32_P16 ? "FP32 (FP16 prolongator)"
                                                          : "FP32 (FP16 operator values)";
  std::snprintf(line, sizeof line, "  levels: %zu   V-cycle precision: %s\n", p->lv.size(), prec);
  s += line;
  double opc = 0, nnz0 = p->lv.empty() ? 1 : (double)p->lv[0].A.nnz();
  for (size_t l = 0; l < p->lv.size(); ++l) {
    const mld::Level &L = p->lv[l];
    opc += (double)L.A.nnz();
    std::snprintf(line, sizeof line,
                  "  level %zu: rows %d nnz %lld  smoother %s sweeps %d/%d%s", l, L.A.nr,
                  (long long)L.A.nnz(), L.kind == mld::SM_BJAC ? "BJAC-ILU(0)" : (L.kind == mld::SM_FBGS ? "FBGS" : "JACOBI"),
                  L.sweeps_pre, L.sweeps_post, l ? "" : "\n");
    s += line;
    if (l) {
      std::snprintf(line, sizeof line, "  omega %.6g\n", L.omega);
      s += line;
    }
  }
  std::snprintf(line, sizeof line, "  operator complexity: %.4f\n", opc / nnz0);
  s += line;
  std::snprintf(buf, (size_t)len, "%s", s.c_str());
  return 0;
}

extern "C" mldg_handle *mldp_gpu(mldp_prec *p) { return p ? p->gpu : nullptr; }

extern "C" const char *mldp_last_error(const mldp_prec *p) { return p ? p->err.c_str() : "null"; }

extern "C" void mldp_destroy(mldp_prec *p) {
  if (!p) return;
  if (p->gpu) mldg_destroy(p->gpu);
  delete p;
}

extern "C" int64_t mldp_pde3d_nnz(int idim) {
  const int64_t n = (int64_t)idim * idim * idim;
  return 7 * n - 6LL * idim * idim;
}

extern "C" int mldp_gen_pde3d(int idim, int hden, const double *coef, int32_t *irp, int32_t *ja,
                              double *val) {
  if (idim <= 0 || !coef || !irp || !ja || !val) return MLDG_ERR_ARG;
  mld::CSR a;
  mld::gen_pde3d(idim, hden, coef, a);
  std::copy(a.irp.begin(), a.irp.end(), irp);
  std::copy(a.ja.begin(), a.ja.end(), ja);
  std::copy(a.val.begin(), a.val.end(), val);
  return 0;
}

extern "C" int mldp_gen_kappa3d(int idim, const double *kappa, int32_t *irp, int32_t *ja,
                                double *val) {
  if (idim <= 0 || !kappa || !irp || !ja || !val) return MLDG_ERR_ARG;
  mld::CSR a;
  mld::gen_kappa3d(idim, kappa, a);
  std::copy(a.irp.begin(), a.irp.end(), irp);
  std::copy(a.ja.begin(), a.ja.end(), ja);
  std::copy(a.val.begin(), a.val.end(), val);
  return 0;
}
