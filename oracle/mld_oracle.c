/*
 * mld_oracle.c -- TEST INFRASTRUCTURE ONLY (see mld_oracle.h).
 *
 * Plain-C restatement of the MLD2P4 2.1 algorithms on the preconditioner
 * apply path and of the host-side build that produces its inputs.  Every
 * function cites the reference file:line it follows.  Built with
 * -ffp-contract=off so that every a*b+c is two roundings, as written.
 */
#include "mld_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* PSBLAS 3.5 d_epstol (pivot threshold used by mld_dilu0_fact.f90:436) */
#define ORC_EPSTOL 1.1102230246251565e-16

typedef struct {
  int nr, nc;
  int *irp;
  int *ja;
  double *val;
} csr;

typedef struct {
  csr A;           /* level matrix (base_a) */
  csr P, R;        /* maps to the previous level (stored at this level, l >= 2) */
  int *ilaggr;     /* aggregate of each row of the previous level */
  int naggr;
  double omega;
  int smoother;    /* ORC_JACOBI / ORC_BJAC / ORC_FBGS */
  int sweeps_pre, sweeps_post;
  double damp;
  csr L, U;        /* ILU(0): unit lower / unit upper (U rows scaled by 1/pivot);
                      FBGS: the strict lower / strict upper triangles of A */
  double *d;       /* ILU(0): 1/pivot; FBGS: the diagonal a_ii */
  double *dinv;    /* diag solver: 1/a_ii (0 -> 1) */
  csr ND;          /* jac smoother off-(block-)diagonal part */
  long nnz_nd;
} level;

struct orc_prec {
  orc_params par;
  int nlev;
  level *lv;
  /* per-level work vectors for the cycle */
  double **x2l, **y2l, **ty, **tx, **w1, **wa, **wb;
};

/* ------------------------------------------------------------------------ */
static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s);
  if (!p) {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return p;
}

static void csr_alloc(csr *a, int nr, int nc, long nnz) {
  a->nr = nr;
  a->nc = nc;
  a->irp = (int *)xcalloc((size_t)nr + 1, sizeof(int));
  a->ja = (int *)xcalloc((size_t)nnz, sizeof(int));
  a->val = (double *)xcalloc((size_t)nnz, sizeof(double));
}

static void csr_free(csr *a) {
  free(a->irp);
  free(a->ja);
  free(a->val);
  memset(a, 0, sizeof(*a));
}

static long csr_nnz(const csr *a) { return a->irp ? a->irp[a->nr] : 0; }

static void csr_copy(csr *dst, int nr, int nc, const int *irp, const int *ja,
                     const double *val) {
  long nnz = irp[nr];
  csr_alloc(dst, nr, nc, nnz);
  memcpy(dst->irp, irp, sizeof(int) * ((size_t)nr + 1));
  memcpy(dst->ja, ja, sizeof(int) * (size_t)nnz);
  memcpy(dst->val, val, sizeof(double) * (size_t)nnz);
}

/* diagonal of a CSR matrix, 0 where absent (psb get_diag) */
static double *csr_diag(const csr *a) {
  double *d = (double *)xcalloc((size_t)a->nr, sizeof(double));
  for (int i = 0; i < a->nr; i++)
    for (int k = a->irp[i]; k < a->irp[i + 1]; k++)
      if (a->ja[k] == i) d[i] += a->val[k];
  return d;
}

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* C = A * B, Gustavson row-by-row with a dense accumulator; entries of row i
 * accumulate in the order of A's row i then B's rows; output columns sorted.
 * Stands in for psb_spspmm (PSBLAS 3.5), call sites
 * mlprec/impl/mld_daggrmat_smth_asb.f90:316,345,399. */
static void csr_spgemm(const csr *A, const csr *B, csr *C) {
  int nr = A->nr, nc = B->nc;
  int *mark = (int *)xcalloc((size_t)nc, sizeof(int));
  double *acc = (double *)xcalloc((size_t)nc, sizeof(double));
  int *cols = (int *)xcalloc((size_t)nc, sizeof(int));
  for (int j = 0; j < nc; j++) mark[j] = -1;
  /* symbolic */
  long nnz = 0;
  int *irp = (int *)xcalloc((size_t)nr + 1, sizeof(int));
  for (int i = 0; i < nr; i++) {
    int cnt = 0;
    for (int ka = A->irp[i]; ka < A->irp[i + 1]; ka++) {
      int k = A->ja[ka];
      for (int kb = B->irp[k]; kb < B->irp[k + 1]; kb++) {
        int j = B->ja[kb];
        if (mark[j] != i) {
          mark[j] = i;
          cnt++;
        }
      }
    }
    nnz += cnt;
    irp[i + 1] = (int)nnz;
  }
  C->nr = nr;
  C->nc = nc;
  C->irp = irp;
  C->ja = (int *)xcalloc((size_t)nnz, sizeof(int));
  C->val = (double *)xcalloc((size_t)nnz, sizeof(double));
  for (int j = 0; j < nc; j++) mark[j] = -1;
  for (int i = 0; i < nr; i++) {
    int cnt = 0;
    for (int ka = A->irp[i]; ka < A->irp[i + 1]; ka++) {
      int k = A->ja[ka];
      double a = A->val[ka];
      for (int kb = B->irp[k]; kb < B->irp[k + 1]; kb++) {
        int j = B->ja[kb];
        double p = a * B->val[kb];
        if (mark[j] != i) {
          mark[j] = i;
          acc[j] = p;
          cols[cnt++] = j;
        } else {
          acc[j] = acc[j] + p;
        }
      }
    }
    qsort(cols, (size_t)cnt, sizeof(int), cmp_int);
    int base = irp[i];
    for (int t = 0; t < cnt; t++) {
      C->ja[base + t] = cols[t];
      C->val[base + t] = acc[cols[t]];
    }
  }
  free(mark);
  free(acc);
  free(cols);
}

/* T = A^T with ascending columns in each row */
static void csr_transpose(const csr *A, csr *T) {
  long nnz = csr_nnz(A);
  csr_alloc(T, A->nc, A->nr, nnz);
  for (long k = 0; k < nnz; k++) T->irp[A->ja[k] + 1]++;
  for (int j = 0; j < A->nc; j++) T->irp[j + 1] += T->irp[j];
  int *fill = (int *)xcalloc((size_t)A->nc, sizeof(int));
  for (int i = 0; i < A->nr; i++)
    for (int k = A->irp[i]; k < A->irp[i + 1]; k++) {
      int j = A->ja[k];
      int pos = T->irp[j] + fill[j]++;
      T->ja[pos] = i;
      T->val[pos] = A->val[k];
    }
  free(fill);
}

/* ------------------------------------------------------------------------ */
/* y = alpha*A*x + beta*y ; row sum accumulated from 0 in stored order
 * (psb_spmm, PSBLAS 3.5; call sites mld_dmlprec_aply.f90:674,752) */
void orc_spmv(int nr, const int *irp, const int *ja, const double *val,
              double alpha, const double *x, double beta, double *y) {
#pragma omp parallel for schedule(static) if (nr > 20000)
  for (int i = 0; i < nr; i++) {
    double s = 0.0;
    for (int k = irp[i]; k < irp[i + 1]; k++) s = s + val[k] * x[ja[k]];
    if (beta == 0.0)
      y[i] = alpha * s;
    else
      y[i] = alpha * s + beta * y[i];
  }
}

/* y = alpha*A^T*x + beta*y (A is nr x nc) */
void orc_spmv_t(int nr, int nc, const int *irp, const int *ja,
                const double *val, double alpha, const double *x, double beta,
                double *y) {
  double *t = (double *)xcalloc((size_t)nc, sizeof(double));
  for (int i = 0; i < nr; i++)
    for (int k = irp[i]; k < irp[i + 1]; k++) t[ja[k]] = t[ja[k]] + val[k] * x[i];
  for (int j = 0; j < nc; j++)
    y[j] = (beta == 0.0) ? alpha * t[j] : alpha * t[j] + beta * y[j];
  free(t);
}

static void spmv_op(const csr *a, char trans, double alpha, const double *x,
                    double beta, double *y) {
  if (trans == 'N')
    orc_spmv(a->nr, a->irp, a->ja, a->val, alpha, x, beta, y);
  else
    orc_spmv_t(a->nr, a->nc, a->irp, a->ja, a->val, alpha, x, beta, y);
}

static void axpby(int n, double a, const double *x, double b, double *y) {
#pragma omp parallel for schedule(static) if (n > 20000)
  for (int i = 0; i < n; i++) y[i] = (b == 0.0) ? a * x[i] : a * x[i] + b * y[i];
}

/* Dot product summed in ORC_DOT_CHUNKS fixed chunks (each from zero in index
 * order), the chunk sums then added in chunk order: the same result for any
 * number of threads. */
#define ORC_DOT_CHUNKS 64
static double dot(int n, const double *x, const double *y) {
  double part[ORC_DOT_CHUNKS];
#pragma omp parallel for schedule(static) if (n > 20000)
  for (int c = 0; c < ORC_DOT_CHUNKS; c++) {
    const int lo = (int)((long)n * c / ORC_DOT_CHUNKS), hi = (int)((long)n * (c + 1) / ORC_DOT_CHUNKS);
    double s = 0.0;
    for (int i = lo; i < hi; i++) s = s + x[i] * y[i];
    part[c] = s;
  }
  double s = 0.0;
  for (int c = 0; c < ORC_DOT_CHUNKS; c++) s = s + part[c];
  return s;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* tests/pdegen/mld_d_pde3d.f90:98-412: row id = (ix-1)*idim^2+(iy-1)*idim+iz,
 * stencil order (x-1),(y-1),(z-1),C,(z+1),(y+1),(x+1); coefficients constant. */
long orc_pde3d_nnz(int idim) {
  long n = (long)idim * idim * idim;
  return 7 * n - 6L * idim * idim;
}

int orc_gen_pde3d(int idim, int hden, const double *coef, int *irp, int *ja,
                  double *val) {
  double a1 = coef[0], a2 = coef[1], a3 = coef[2];
  double b1 = coef[3], b2 = coef[4], b3 = coef[5], c = coef[6];
  double deltah = 1.0 / (double)(idim + hden);
  double sqdeltah = deltah * deltah;
  double deltah2 = 2.0 * deltah;
  long idim2 = (long)idim * idim;
  long n = idim2 * idim;
  long nz = 0;
  irp[0] = 0;
  for (long row = 0; row < n; row++) {
    int ix = (int)(row / idim2);
    int iy = (int)((row / idim) % idim);
    int iz = (int)(row % idim);
    if (ix > 0) {
      ja[nz] = (int)(row - idim2);
      val[nz++] = -a1 / sqdeltah - b1 / deltah2;
    }
    if (iy > 0) {
      ja[nz] = (int)(row - idim);
      val[nz++] = -a2 / sqdeltah - b2 / deltah2;
    }
    if (iz > 0) {
      ja[nz] = (int)(row - 1);
      val[nz++] = -a3 / sqdeltah - b3 / deltah2;
    }
    ja[nz] = (int)row;
    val[nz++] = 2.0 * (a1 + a2 + a3) / sqdeltah + c;
    if (iz < idim - 1) {
      ja[nz] = (int)(row + 1);
      val[nz++] = -a3 / sqdeltah + b3 / deltah2;
    }
    if (iy < idim - 1) {
      ja[nz] = (int)(row + idim);
      val[nz++] = -a2 / sqdeltah + b2 / deltah2;
    }
    if (ix < idim - 1) {
      ja[nz] = (int)(row + idim2);
      val[nz++] = -a1 / sqdeltah + b1 / deltah2;
    }
    irp[row + 1] = (int)nz;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Decoupled aggregation, natural ordering, one rank:
 * mlprec/impl/mld_d_dec_map_bld.f90:70-321 */
static int dec_map_bld(const csr *a, double theta, int *ilaggr, int *naggr_out) {
  int nr = a->nr;
  double *diag = csr_diag(a);
  int *icol = (int *)xcalloc((size_t)nr + 1, sizeof(int));
  int *tmpaggr = (int *)xcalloc((size_t)nr, sizeof(int));
  const int unset = -(nr + 1);
  int naggr = 0;
  for (int i = 0; i < nr; i++) ilaggr[i] = unset;

  /* phase one: disjoint strongly-coupled neighbourhoods (:148-189) */
  for (int i = 0; i < nr; i++) {
    if (ilaggr[i] != unset) continue;
    int ip = 0;
    for (int k = a->irp[i]; k < a->irp[i + 1]; k++) {
      int j = a->ja[k];
      if (j >= 0 && j < nr &&
          fabs(a->val[k]) > theta * sqrt(fabs(diag[i] * diag[j])))
        icol[ip++] = j;
    }
    int disjoint = 1;
    for (int t = 0; t < ip; t++)
      if (ilaggr[icol[t]] != unset) {
        disjoint = 0;
        break;
      }
    if (disjoint || ip == 0) {
      naggr++;
      for (int t = 0; t < ip; t++) ilaggr[icol[t]] = naggr;
      ilaggr[i] = naggr;
    }
  }

  /* phase two: join the most strongly coupled phase-one aggregate (:199-230) */
  memcpy(tmpaggr, ilaggr, sizeof(int) * (size_t)nr);
  for (int i = 0; i < nr; i++) {
    if (ilaggr[i] != unset) continue;
    double cpling = 0.0;
    int ip = -1;
    for (int k = a->irp[i]; k < a->irp[i + 1]; k++) {
      int j = a->ja[k];
      if (j >= 0 && j < nr) {
        double av = fabs(a->val[k]);
        if (av > theta * sqrt(fabs(diag[i] * diag[j])) && tmpaggr[j] > 0 &&
            av > cpling) {
          ip = k;
          cpling = av;
        }
      }
    }
    if (ip >= 0) ilaggr[i] = ilaggr[a->ja[ip]];
  }

  /* phase three: leftovers become new aggregates (:236-278) */
  for (int i = 0; i < nr; i++) {
    if (ilaggr[i] >= 0) continue;
    int ip = 0;
    for (int k = a->irp[i]; k < a->irp[i + 1]; k++) {
      int j = a->ja[k];
      if (j >= 0 && j < nr &&
          fabs(a->val[k]) > theta * sqrt(fabs(diag[i] * diag[j])) &&
          ilaggr[j] < 0)
        icol[ip++] = j;
    }
    naggr++;
    ilaggr[i] = naggr;
    for (int t = 0; t < ip; t++) ilaggr[icol[t]] = naggr;
  }
  int bad = 0;
  for (int i = 0; i < nr; i++) {
    if (ilaggr[i] < 0) bad = 1;
    ilaggr[i] -= 1; /* to 0-based aggregate ids */
  }
  free(diag);
  free(icol);
  free(tmpaggr);
  *naggr_out = naggr;
  return bad ? -1 : 0;
}

/* Smoothed prolongator, restriction and Galerkin product, no filtering:
 * mlprec/impl/mld_daggrmat_smth_asb.f90:174-401 (one rank). */
static int aggrmat_smth_asb(const csr *a, const int *ilaggr, int naggr,
                            double *omega_out, csr *P, csr *R, csr *Ac) {
  int nr = a->nr;
  double *adiag = csr_diag(a);
  for (int i = 0; i < nr; i++) adiag[i] = (adiag[i] != 0.0) ? 1.0 / adiag[i] : 1.0;
  /* acsr3 = D^{-1} A (:263-264), anorm = ||D^{-1}A||_inf (:270) */
  csr S;
  csr_copy(&S, nr, a->nc, a->irp, a->ja, a->val);
  double anorm = 0.0;
  for (int i = 0; i < nr; i++) {
    double rs = 0.0;
    for (int k = S.irp[i]; k < S.irp[i + 1]; k++) {
      S.val[k] = adiag[i] * S.val[k];
      rs = rs + fabs(S.val[k]);
    }
    if (rs > anorm) anorm = rs;
  }
  double omega = 4.0 / (3.0 * anorm);
  *omega_out = omega;
  /* I - omega D^{-1} A on the stored pattern (:298-306) */
  for (int i = 0; i < nr; i++)
    for (int k = S.irp[i]; k < S.irp[i + 1]; k++)
      S.val[k] = (S.ja[k] == i) ? 1.0 - omega * S.val[k] : -omega * S.val[k];
  /* tentative prolongator: row i has a single 1 in column ilaggr(i)
   * (mld_daggrmap_bld.f90:171-180) */
  csr Pt;
  csr_alloc(&Pt, nr, naggr, nr);
  for (int i = 0; i < nr; i++) {
    Pt.irp[i + 1] = i + 1;
    Pt.ja[i] = ilaggr[i];
    Pt.val[i] = 1.0;
  }
  csr_spgemm(&S, &Pt, P); /* (:316) */
  csr_free(&Pt);
  csr_free(&S);
  csr AP;
  csr_spgemm(a, P, &AP); /* (:345) */
  csr_transpose(P, R);   /* (:355-375) */
  csr_spgemm(R, &AP, Ac); /* (:399) */
  csr_free(&AP);
  free(adiag);
  return 0;
}

/* ILU(0): mlprec/impl/mld_dilu0_fact.f90:284-477 (ialg = ILU_N), with the
 * row split of ilu_copyin (:551-660). */
static int ilu0_fact(const csr *a, csr *L, csr *U, double *d) {
  int m = a->nr;
  long nz = csr_nnz(a);
  csr_alloc(L, m, m, nz);
  csr_alloc(U, m, m, nz);
  int l1 = 0, l2 = 0;
  L->irp[0] = 0;
  U->irp[0] = 0;
  for (int i = 0; i < m; i++) {
    double dia = 0.0;
    for (int k = a->irp[i]; k < a->irp[i + 1]; k++) {
      int j = a->ja[k];
      if (j < i) {
        L->ja[l1] = j;
        L->val[l1++] = a->val[k];
      } else if (j == i) {
        dia = a->val[k];
      } else if (j < m) {
        U->ja[l2] = j;
        U->val[l2++] = a->val[k];
      }
    }
    L->irp[i + 1] = l1;
    U->irp[i + 1] = l2;
    for (int kk = L->irp[i]; kk < L->irp[i + 1]; kk++) {
      double temp = L->val[kk];
      int k = L->ja[kk];
      L->val[kk] = temp * d[k];
      int low1 = kk + 1, low2 = U->irp[i];
      for (int jj = U->irp[k]; jj < U->irp[k + 1]; jj++) {
        int j = U->ja[jj];
        if (j < i) {
          for (int ll = low1; ll < L->irp[i + 1]; ll++) {
            int l = L->ja[ll];
            if (l > j) {
              low1 = ll;
              break;
            } else if (l == j) {
              L->val[ll] = L->val[ll] - temp * U->val[jj];
              low1 = ll + 1;
              break;
            }
          }
        } else if (j == i) {
          dia = dia - temp * U->val[jj];
        } else {
          for (int ll = low2; ll < U->irp[i + 1]; ll++) {
            int l = U->ja[ll];
            if (l > j) {
              low2 = ll;
              break;
            } else if (l == j) {
              U->val[ll] = U->val[ll] - temp * U->val[jj];
              low2 = ll + 1;
              break;
            }
          }
        }
      }
    }
    if (fabs(dia) < ORC_EPSTOL) return 2 + i; /* pivot too small (:436-445) */
    dia = 1.0 / dia;
    d[i] = dia;
    for (int kk = U->irp[i]; kk < U->irp[i + 1]; kk++) U->val[kk] = U->val[kk] * dia;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* unit lower solve t = L^{-1} x, row sum from 0 then subtract
 * (psb_spsm, call site mld_d_ilu_solver_apply_vect.f90:132) */
static void lsolve(const csr *L, const double *x, double *t) {
  for (int i = 0; i < L->nr; i++) {
    double s = 0.0;
    for (int k = L->irp[i]; k < L->irp[i + 1]; k++) s = s + L->val[k] * t[L->ja[k]];
    t[i] = x[i] - s;
  }
}
/* unit upper solve z = U^{-1} w */
static void usolve(const csr *U, const double *w, double *z) {
  for (int i = U->nr - 1; i >= 0; i--) {
    double s = 0.0;
    for (int k = U->irp[i]; k < U->irp[i + 1]; k++) s = s + U->val[k] * z[U->ja[k]];
    z[i] = w[i] - s;
  }
}
/* z = U^{-T} x (U^T unit lower), column-oriented */
static void usolve_t(const csr *U, const double *x, double *z) {
  int n = U->nr;
  memcpy(z, x, sizeof(double) * (size_t)n);
  for (int i = 0; i < n; i++)
    for (int k = U->irp[i]; k < U->irp[i + 1]; k++)
      z[U->ja[k]] = z[U->ja[k]] - U->val[k] * z[i];
}
/* z = L^{-T} x (L^T unit upper), column-oriented */
static void lsolve_t(const csr *L, const double *x, double *z) {
  int n = L->nr;
  memcpy(z, x, sizeof(double) * (size_t)n);
  for (int i = n - 1; i >= 0; i--)
    for (int k = L->irp[i]; k < L->irp[i + 1]; k++)
      z[L->ja[k]] = z[L->ja[k]] - L->val[k] * z[i];
}

/* ILU solver apply, y = alpha*U^{-1}(d o L^{-1}x) + beta*y ('N') or
 * y = alpha*L^{-T}(d o U^{-T}x) + beta*y ('T'):
 * mlprec/impl/solver/mld_d_ilu_solver_apply_vect.f90:130-142 */
static void ilu_apply(const level *lv, char trans, double alpha, const double *x,
                      double beta, double *y, double *w1, double *w2) {
  int n = lv->A.nr;
  if (trans == 'N') {
    lsolve(&lv->L, x, w1);
    for (int i = 0; i < n; i++) w1[i] = lv->d[i] * w1[i];
    usolve(&lv->U, w1, w2);
  } else {
    usolve_t(&lv->U, x, w1);
    for (int i = 0; i < n; i++) w1[i] = lv->d[i] * w1[i];
    lsolve_t(&lv->L, w1, w2);
  }
  axpby(n, alpha, w2, beta, y);
}

/* diag solver: y = alpha*d o x + beta*y
 * (mlprec/impl/solver/mld_d_diag_solver_apply_vect.f90:102) */
static void diag_apply(const level *lv, double alpha, const double *x,
                       double beta, double *y) {
  int n = lv->A.nr;
#pragma omp parallel for schedule(static) if (n > 20000)
  for (int i = 0; i < n; i++)
    y[i] = (beta == 0.0) ? alpha * (lv->dinv[i] * x[i])
                         : alpha * (lv->dinv[i] * x[i]) + beta * y[i];
}

/* One Gauss-Seidel sweep of the GS solver (forward: wv = x - U xit,
 * xit = (D+L)^{-1} wv; mlprec/impl/solver/mld_d_gs_solver_apply_vect.f90:143-158)
 * or of the BWGS solver (backward: wv = x - L xit, xit = (D+U)^{-1} wv;
 * mld_d_bwgs_solver_apply_vect.f90:150-156).  The triangular solve with a
 * non-unit diagonal sums the row from zero, subtracts, divides by a_ii. */
static void gs_sweep(const level *lv, int backward, const double *x, double *xit,
                     double *wv) {
  int n = lv->A.nr;
  const csr *off = backward ? &lv->L : &lv->U;
  const csr *tri = backward ? &lv->U : &lv->L;
  memcpy(wv, x, sizeof(double) * (size_t)n);
  spmv_op(off, 'N', -1.0, xit, 1.0, wv);
  if (!backward) {
    for (int i = 0; i < n; i++) {
      double s = 0.0;
      for (int k = tri->irp[i]; k < tri->irp[i + 1]; k++) s = s + tri->val[k] * xit[tri->ja[k]];
      xit[i] = (wv[i] - s) / lv->d[i];
    }
  } else {
    for (int i = n - 1; i >= 0; i--) {
      double s = 0.0;
      for (int k = tri->irp[i]; k < tri->irp[i + 1]; k++) s = s + tri->val[k] * xit[tri->ja[k]];
      xit[i] = (wv[i] - s) / lv->d[i];
    }
  }
}

static void solver_apply(const level *lv, char trans, double alpha,
                         const double *x, double beta, double *y, double *w1,
                         double *w2) {
  if (lv->smoother == ORC_BJAC)
    ilu_apply(lv, trans, alpha, x, beta, y, w1, w2);
  else
    diag_apply(lv, alpha, x, beta, y);
}

/* jac smoother apply with init='Z':
 * mlprec/impl/smoother/mld_d_jac_smoother_apply_vect.f90:107-177.
 * Damping (extension): ty <- (1-w) ty + w S(x - ND ty); w = 1 is the
 * reference iteration exactly. */
static void jac_smoother_apply(orc_prec *p, int l, char trans, double alpha,
                               const double *x, double beta, double *y,
                               int sweeps, int post) {
  level *lv = &p->lv[l];
  int n = lv->A.nr;
  double *tx = p->tx[l], *ty2 = p->w1[l];
  double *wa = p->wa[l], *wb = p->wb[l];
  if (lv->smoother == ORC_FBGS) {
    /* GS solvers are iterative: always the general branch (:117-177).
     * init Z, then sweeps-1 more sweeps from the previous iterate; the
     * off-block part ND is empty on one rank (tx = x).  Pre smoother sm:
     * forward GS; post smoother sm2: backward GS (onelev_cseti.F90:128-132). */
    memset(ty2, 0, sizeof(double) * (size_t)n);
    for (int s = 0; s < sweeps; s++) gs_sweep(lv, post, x, ty2, wa);
    axpby(n, alpha, ty2, beta, y);
    return;
  }
  if (sweeps == 1 || lv->nnz_nd == 0) {
    /* single solver application (:107-109); the diag solver is not iterative */
    if (lv->smoother == ORC_JACOBI && lv->damp != 1.0)
      solver_apply(lv, trans, alpha * lv->damp, x, beta, y, wa, wb);
    else
      solver_apply(lv, trans, alpha, x, beta, y, wa, wb);
  } else {
    double w = lv->damp;
    /* first sweep unrolled with init Z (:136) */
    solver_apply(lv, trans, (w == 1.0) ? 1.0 : w, x, 0.0, ty2, wa, wb);
    for (int s = 1; s < sweeps; s++) {
      memcpy(tx, x, sizeof(double) * (size_t)n);
      spmv_op(&lv->ND, trans, -1.0, ty2, 1.0, tx); /* (:161-162) */
      if (w == 1.0) {
        solver_apply(lv, trans, 1.0, tx, 0.0, ty2, wa, wb); /* (:166) */
      } else {
        solver_apply(lv, trans, w, tx, 1.0 - w, ty2, wa, wb);
      }
    }
    axpby(n, alpha, ty2, beta, y); /* (:177) */
  }
}

/* V-cycle body: mlprec/impl/mld_dmlprec_aply.f90:590-809 (ml_cycle=VCYCLE) */
static void inner_k_cycle(orc_prec *p, int l, char trans);

/* dispatch on ml_cycle (mld_dmlprec_aply.f90:418-460 inner_ml_aply) */
static void inner_ml_aply(orc_prec *p, int l, char trans);

static void inner_mult(orc_prec *p, int l, char trans) {
  level *lv = &p->lv[l];
  int nlev = p->nlev;
  int n = lv->A.nr;
  int spre = lv->sweeps_pre, spost = lv->sweeps_post;
  int pre = (spre > 0 && trans == 'N') || (spost > 0 && trans != 'N');
  int post = (spost > 0 && trans == 'N') || (spre > 0 && trans != 'N');
  double *x = p->x2l[l], *y = p->y2l[l], *ty = p->ty[l];
  if (l < nlev - 1) {
    level *lc = &p->lv[l + 1];
    if (pre) {
      /* (:644-664) sm (N) / sm2 (T); init Z, beta 0 */
      jac_smoother_apply(p, l, trans, 1.0, x, 0.0, y,
                         trans == 'N' ? spre : spost, trans == 'N' ? 0 : 1);
      /* residual (:669-676) and restriction (:682-684) */
      memcpy(ty, x, sizeof(double) * (size_t)n);
      spmv_op(&lv->A, trans, -1.0, y, 1.0, ty);
      orc_spmv(lc->R.nr, lc->R.irp, lc->R.ja, lc->R.val, 1.0, ty, 0.0,
               p->x2l[l + 1]);
    } else {
      memset(y, 0, sizeof(double) * (size_t)n);
      orc_spmv(lc->R.nr, lc->R.irp, lc->R.ja, lc->R.val, 1.0, x, 0.0,
               p->x2l[l + 1]);
    }
    inner_mult(p, l + 1, trans); /* (:702) */
    /* prolongation + correction y += P y_c (:707-709) */
    orc_spmv(lc->P.nr, lc->P.irp, lc->P.ja, lc->P.val, 1.0, p->y2l[l + 1], 1.0, y);
    if (p->par.ml_cycle == ORC_WCYCLE) {
      /* W-cycle: a second coarse correction from the new residual (:716-745) */
      memcpy(ty, x, sizeof(double) * (size_t)n);
      spmv_op(&lv->A, trans, -1.0, y, 1.0, ty);
      orc_spmv(lc->R.nr, lc->R.irp, lc->R.ja, lc->R.val, 1.0, ty, 0.0, p->x2l[l + 1]);
      inner_mult(p, l + 1, trans);
      orc_spmv(lc->P.nr, lc->P.irp, lc->P.ja, lc->P.val, 1.0, p->y2l[l + 1], 1.0, y);
    }
    if (post) {
      memcpy(ty, x, sizeof(double) * (size_t)n);
      spmv_op(&lv->A, trans, -1.0, y, 1.0, ty); /* (:748-755) */
      jac_smoother_apply(p, l, trans, 1.0, ty, 1.0, y,
                         trans == 'N' ? spost : spre, trans == 'N' ? 1 : 0); /* (:765-777) */
    }
  } else {
    /* coarsest level (:787-793) */
    jac_smoother_apply(p, l, trans, 1.0, x, 0.0, y, spre, 0);
  }
}

/* additive cycle (mld_d_inner_add, mld_dmlprec_aply.f90:464-588): smooth x
 * (FBGS: max(sweeps) times forward then backward GS, each from the previous
 * result), restrict x itself, recurse, add the prolongated correction */
static void inner_add(orc_prec *p, int l, char trans) {
  level *lv = &p->lv[l];
  int n = lv->A.nr;
  double *x = p->x2l[l], *y = p->y2l[l], *tx = p->tx[l];
  if (lv->smoother == ORC_FBGS) {
    memcpy(y, x, sizeof(double) * (size_t)n);
    int sw = lv->sweeps_pre > lv->sweeps_post ? lv->sweeps_pre : lv->sweeps_post;
    for (int k = 0; k < sw; k++) {
      jac_smoother_apply(p, l, trans, 1.0, y, 0.0, tx, 1, 0);
      jac_smoother_apply(p, l, trans, 1.0, tx, 0.0, y, 1, 1);
    }
  } else {
    jac_smoother_apply(p, l, trans, 1.0, x, 0.0, y, lv->sweeps_pre, 0);
  }
  if (l < p->nlev - 1) {
    level *lc = &p->lv[l + 1];
    orc_spmv(lc->R.nr, lc->R.irp, lc->R.ja, lc->R.val, 1.0, x, 0.0, p->x2l[l + 1]);
    inner_ml_aply(p, l + 1, trans);
    orc_spmv(lc->P.nr, lc->P.irp, lc->P.ja, lc->P.val, 1.0, p->y2l[l + 1], 1.0, y);
  }
}

static void inner_ml_aply(orc_prec *p, int l, char trans) {
  if (p->par.ml_cycle == ORC_KCYCLE || p->par.ml_cycle == ORC_KCYCLESYM)
    inner_k_cycle(p, l, trans);
  else if (p->par.ml_cycle == ORC_ADD)
    inner_add(p, l, trans);
  else
    inner_mult(p, l, trans);
}

/* K-cycle inner iteration at level l (mld_dinneritkcycle,
 * mld_dmlprec_aply.f90:1017-1184): at most two steps of flexible CG (FCG,
 * KCYCLESYM) or GCR (KCYCLE) on A_l with the level's own cycle as
 * preconditioner; the second step only when the first left
 * ||w|| > 0.25 ||rhs||.  The inner products use A_l (no transpose) for
 * either trans, as the reference does. */
static void inneritkcycle(orc_prec *p, int l, char trans, int gcr) {
  level *lv = &p->lv[l];
  int n = lv->A.nr;
  size_t nb = sizeof(double) * (size_t)n;
  double *w = (double *)xcalloc((size_t)n, sizeof(double));
  double *v = (double *)xcalloc((size_t)n, sizeof(double));
  double *v1 = (double *)xcalloc((size_t)n, sizeof(double));
  double *xk = (double *)xcalloc((size_t)n, sizeof(double));
  double *d0 = (double *)xcalloc((size_t)n, sizeof(double));
  double *d1 = (double *)xcalloc((size_t)n, sizeof(double));
  memcpy(w, p->x2l[l], nb);
  double delta0 = sqrt(dot(n, w, w));
  memset(p->y2l[l], 0, nb);
  inner_ml_aply(p, l, trans);
  memcpy(d0, p->y2l[l], nb);
  orc_spmv(n, lv->A.irp, lv->A.ja, lv->A.val, 1.0, d0, 0.0, v);
  double delta_old, tau;
  if (gcr) {
    delta_old = dot(n, v, w);
    tau = dot(n, v, v);
  } else {
    delta_old = dot(n, d0, w);
    tau = dot(n, d0, v);
  }
  double alpha = delta_old / tau;
  for (int i = 0; i < n; i++) w[i] = -alpha * v[i] + w[i];
  double l2 = sqrt(dot(n, w, w));
  if (l2 <= 0.25 * delta0) {
    for (int i = 0; i < n; i++) xk[i] = alpha * d0[i] + xk[i];
  } else {
    memcpy(p->x2l[l], w, nb);
    inner_ml_aply(p, l, trans);
    memcpy(d1, p->y2l[l], nb);
    orc_spmv(n, lv->A.irp, lv->A.ja, lv->A.val, 1.0, d1, 0.0, v1);
    double tau1, tau2, tau3;
    if (gcr) {
      tau1 = dot(n, v1, v);
      tau2 = dot(n, v1, v1);
      tau3 = dot(n, v1, w);
    } else {
      tau1 = dot(n, d1, v);
      tau2 = dot(n, d1, v1);
      tau3 = dot(n, d1, w);
    }
    double tau4 = tau2 - (tau1 * tau1) / tau;
    alpha = alpha - (tau1 * tau3) / (tau * tau4);
    for (int i = 0; i < n; i++) xk[i] = alpha * d0[i] + xk[i];
    alpha = tau3 / tau4;
    for (int i = 0; i < n; i++) xk[i] = alpha * d1[i] + xk[i];
  }
  memcpy(p->y2l[l], xk, nb);
  free(w);
  free(v);
  free(v1);
  free(xk);
  free(d0);
  free(d1);
}

/* K-cycle body (mld_d_inner_k_cycle, mld_dmlprec_aply.f90:811-1000): pre
 * smoothing, restriction, the inner Krylov iteration on the next level (a
 * plain cycle call on the coarsest two), prolongation, post smoothing. */
static void inner_k_cycle(orc_prec *p, int l, char trans) {
  level *lv = &p->lv[l];
  int nlev = p->nlev;
  int n = lv->A.nr;
  int spre = lv->sweeps_pre, spost = lv->sweeps_post;
  double *x = p->x2l[l], *y = p->y2l[l], *ty = p->ty[l];
  if (l == nlev - 1) {
    jac_smoother_apply(p, l, trans, 1.0, x, 0.0, y, spre, 0);
    return;
  }
  level *lc = &p->lv[l + 1];
  jac_smoother_apply(p, l, trans, 1.0, x, 0.0, y, trans == 'N' ? spre : spost, trans == 'N' ? 0 : 1);
  memcpy(ty, x, sizeof(double) * (size_t)n);
  spmv_op(&lv->A, trans, -1.0, y, 1.0, ty);
  orc_spmv(lc->R.nr, lc->R.irp, lc->R.ja, lc->R.val, 1.0, ty, 0.0, p->x2l[l + 1]);
  if (l + 1 <= nlev - 2)
    inneritkcycle(p, l + 1, trans, p->par.ml_cycle == ORC_KCYCLE);
  else
    inner_ml_aply(p, l + 1, trans);
  orc_spmv(lc->P.nr, lc->P.irp, lc->P.ja, lc->P.val, 1.0, p->y2l[l + 1], 1.0, y);
  memcpy(ty, x, sizeof(double) * (size_t)n);
  spmv_op(&lv->A, trans, -1.0, y, 1.0, ty);
  jac_smoother_apply(p, l, trans, 1.0, ty, 1.0, y, trans == 'N' ? spost : spre, trans == 'N' ? 1 : 0);
}

/* ------------------------------------------------------------------------ */
void orc_default_params(orc_params *p) {
  p->smoother = ORC_BJAC;
  p->sweeps_pre = 1;
  p->sweeps_post = 1;
  p->jac_damp = 1.0;
  p->coarse_solver = ORC_BJAC;
  p->coarse_sweeps = 4;
  p->min_coarse_size = -1;
  p->max_levs = 20;
  p->min_cr_ratio = 1.5;
  p->aggr_thresh = 0.01;
  p->ml_cycle = ORC_VCYCLE;
}

orc_prec *orc_prec_new(const orc_params *par) {
  orc_prec *p = (orc_prec *)xcalloc(1, sizeof(orc_prec));
  if (par)
    p->par = *par;
  else
    orc_default_params(&p->par);
  return p;
}

static void level_free(level *lv) {
  csr_free(&lv->A);
  csr_free(&lv->P);
  csr_free(&lv->R);
  csr_free(&lv->L);
  csr_free(&lv->U);
  csr_free(&lv->ND);
  free(lv->ilaggr);
  free(lv->d);
  free(lv->dinv);
  memset(lv, 0, sizeof(*lv));
}

void orc_prec_free(orc_prec *p) {
  if (!p) return;
  for (int l = 0; l < p->nlev; l++) {
    level_free(&p->lv[l]);
    free(p->x2l[l]);
    free(p->y2l[l]);
    free(p->ty[l]);
    free(p->tx[l]);
    free(p->w1[l]);
    free(p->wa[l]);
    free(p->wb[l]);
  }
  free(p->lv);
  free(p->x2l);
  free(p->y2l);
  free(p->ty);
  free(p->tx);
  free(p->w1);
  free(p->wa);
  free(p->wb);
  free(p);
}

/* jac smoother build (mld_d_jac_smoother_bld.f90:73-103) + solver build
 * (mld_d_diag_solver_bld.f90:74-92, mld_d_ilu_solver_bld.f90:126-175) */
static int smoother_build(level *lv, int kind, int spre, int spost, double damp) {
  const csr *a = &lv->A;
  int n = a->nr;
  lv->smoother = kind;
  lv->sweeps_pre = spre;
  lv->sweeps_post = spost;
  lv->damp = damp;
  if (kind == ORC_JACOBI) {
    /* ND = A without its diagonal (clip_diag) */
    long nnz = 0;
    for (int i = 0; i < n; i++)
      for (int k = a->irp[i]; k < a->irp[i + 1]; k++)
        if (a->ja[k] != i) nnz++;
    csr_alloc(&lv->ND, n, a->nc, nnz);
    long t = 0;
    for (int i = 0; i < n; i++) {
      for (int k = a->irp[i]; k < a->irp[i + 1]; k++)
        if (a->ja[k] != i) {
          lv->ND.ja[t] = a->ja[k];
          lv->ND.val[t++] = a->val[k];
        }
      lv->ND.irp[i + 1] = (int)t;
    }
    lv->nnz_nd = nnz;
    lv->dinv = csr_diag(a);
    for (int i = 0; i < n; i++)
      lv->dinv[i] = (lv->dinv[i] == 0.0) ? 1.0 : 1.0 / lv->dinv[i];
    return 0;
  }
  if (kind == ORC_FBGS) {
    /* GS / BWGS solvers (mld_d_gs_solver_bld.f90:73-81: tril with the
     * diagonal + the rest): kept here as strict lower L, strict upper U and
     * the diagonal d; ND is empty on one rank */
    long nl = 0, nu = 0;
    for (int i = 0; i < n; i++)
      for (int k = a->irp[i]; k < a->irp[i + 1]; k++) {
        if (a->ja[k] < i) nl++;
        if (a->ja[k] > i) nu++;
      }
    csr_alloc(&lv->L, n, n, nl);
    csr_alloc(&lv->U, n, n, nu);
    lv->d = (double *)xcalloc((size_t)n, sizeof(double));
    long tl = 0, tu = 0;
    for (int i = 0; i < n; i++) {
      for (int k = a->irp[i]; k < a->irp[i + 1]; k++) {
        int j = a->ja[k];
        if (j < i) {
          lv->L.ja[tl] = j;
          lv->L.val[tl++] = a->val[k];
        } else if (j > i) {
          lv->U.ja[tu] = j;
          lv->U.val[tu++] = a->val[k];
        } else {
          lv->d[i] = a->val[k];
        }
      }
      lv->L.irp[i + 1] = (int)tl;
      lv->U.irp[i + 1] = (int)tu;
      if (lv->d[i] == 0.0) return 1; /* zero diagonal: the GS solve divides by it */
    }
    csr_alloc(&lv->ND, n, a->nc, 0);
    lv->nnz_nd = 0;
    return 0;
  }
  /* BJAC + ILU(0): on one rank the off-block part (columns > nrow) is empty */
  csr_alloc(&lv->ND, n, a->nc, 0);
  lv->nnz_nd = 0;
  lv->d = (double *)xcalloc((size_t)n, sizeof(double));
  return ilu0_fact(a, &lv->L, &lv->U, lv->d);
}

/* hierarchy build: mlprec/impl/mld_d_hierarchy_bld.f90:187-413 */
int orc_prec_build(orc_prec *p, int n, const int *irp, const int *ja,
                   const double *val) {
  const orc_params *par = &p->par;
  int nplevs = par->max_levs < 2 ? 2 : par->max_levs;
  long casize = par->min_coarse_size;
  if (casize < 0) {
    casize = (long)pow((double)n, 1.0 / 3.0);
    if (casize < 1) casize = 1;
    casize *= 40;
  }
  level *lv = (level *)xcalloc((size_t)nplevs, sizeof(level));
  csr_copy(&lv[0].A, n, n, irp, ja, val);
  int nlev = 1;
  int newsz = 0;
  /* max_levs == 1: the one-level preconditioner of init('BJAC'/'JACOBI')
   * (mld_d_hierarchy_bld.f90:159-164 returns at once for one level) */
  for (int i = 1; i < (par->max_levs == 1 ? 1 : nplevs); i++) {
    const csr *af = &lv[i - 1].A;
    int *ilaggr = (int *)xcalloc((size_t)af->nr, sizeof(int));
    int naggr = 0;
    if (dec_map_bld(af, par->aggr_thresh, ilaggr, &naggr) != 0) {
      free(ilaggr);
      return 1;
    }
    double sizeratio = (double)af->nr / (double)naggr;
    if (naggr <= casize) newsz = i;
    if (i > 1) {
      if (sizeratio < par->min_cr_ratio) newsz = (sizeratio > 1) ? i : i - 1;
      if (naggr == lv[i - 1].naggr) newsz = i - 1;
    }
    if (newsz > 0) {
      if (newsz < i) {
        /* revisit the previous level as the coarsest: its own aggregation
         * and matrix are unchanged (same aggregation parameters) */
        free(ilaggr);
        nlev = newsz + 1;
      } else {
        lv[i].ilaggr = ilaggr;
        lv[i].naggr = naggr;
        aggrmat_smth_asb(af, ilaggr, naggr, &lv[i].omega, &lv[i].P, &lv[i].R,
                         &lv[i].A);
        nlev = i + 1;
      }
      break;
    }
    lv[i].ilaggr = ilaggr;
    lv[i].naggr = naggr;
    aggrmat_smth_asb(af, ilaggr, naggr, &lv[i].omega, &lv[i].P, &lv[i].R, &lv[i].A);
    nlev = i + 1;
  }
  for (int l = nlev; l < nplevs; l++) level_free(&lv[l]);
  p->nlev = nlev;
  p->lv = lv;
  /* smoothers (mld_d_smoothers_bld.f90:156-169) */
  for (int l = 0; l < nlev; l++) {
    int rc;
    if (l < nlev - 1 || nlev == 1)
      rc = smoother_build(&lv[l], par->smoother, par->sweeps_pre, par->sweeps_post,
                          par->jac_damp);
    else
      rc = smoother_build(&lv[l], par->coarse_solver, par->coarse_sweeps,
                          par->coarse_sweeps, par->jac_damp);
    if (rc) return 100 + l;
  }
  p->x2l = (double **)xcalloc((size_t)nlev, sizeof(double *));
  p->y2l = (double **)xcalloc((size_t)nlev, sizeof(double *));
  p->ty = (double **)xcalloc((size_t)nlev, sizeof(double *));
  p->tx = (double **)xcalloc((size_t)nlev, sizeof(double *));
  p->w1 = (double **)xcalloc((size_t)nlev, sizeof(double *));
  p->wa = (double **)xcalloc((size_t)nlev, sizeof(double *));
  p->wb = (double **)xcalloc((size_t)nlev, sizeof(double *));
  for (int l = 0; l < nlev; l++) {
    size_t nl = (size_t)lv[l].A.nr;
    p->x2l[l] = (double *)xcalloc(nl, sizeof(double));
    p->y2l[l] = (double *)xcalloc(nl, sizeof(double));
    p->ty[l] = (double *)xcalloc(nl, sizeof(double));
    p->tx[l] = (double *)xcalloc(nl, sizeof(double));
    p->w1[l] = (double *)xcalloc(nl, sizeof(double));
    p->wa[l] = (double *)xcalloc(nl, sizeof(double));
    p->wb[l] = (double *)xcalloc(nl, sizeof(double));
  }
  return 0;
}

int orc_prec_nlev(const orc_prec *p) { return p->nlev; }

int orc_prec_level_info(const orc_prec *p, int l, long *info, double *dinfo) {
  if (l < 0 || l >= p->nlev) return 1;
  const level *lv = &p->lv[l];
  info[0] = lv->A.nr;
  info[1] = csr_nnz(&lv->A);
  info[2] = csr_nnz(&lv->P);
  info[3] = csr_nnz(&lv->R);
  info[4] = csr_nnz(&lv->L);
  info[5] = csr_nnz(&lv->U);
  info[6] = csr_nnz(&lv->ND);
  info[7] = lv->naggr;
  info[8] = lv->smoother;
  info[9] = lv->sweeps_pre;
  if (dinfo) {
    dinfo[0] = lv->omega;
    dinfo[1] = lv->damp;
  }
  return 0;
}

int orc_prec_level_csr(const orc_prec *p, int l, int which, int *irp, int *ja,
                       double *val) {
  if (l < 0 || l >= p->nlev) return 1;
  const level *lv = &p->lv[l];
  const csr *m = which == 0 ? &lv->A
                 : which == 1 ? &lv->P
                 : which == 2 ? &lv->R
                 : which == 3 ? &lv->L
                 : which == 4 ? &lv->U
                              : &lv->ND;
  if (!m->irp) return 2;
  long nnz = csr_nnz(m);
  memcpy(irp, m->irp, sizeof(int) * ((size_t)m->nr + 1));
  memcpy(ja, m->ja, sizeof(int) * (size_t)nnz);
  memcpy(val, m->val, sizeof(double) * (size_t)nnz);
  return 0;
}

int orc_prec_level_vec(const orc_prec *p, int l, int which, double *dv, int *iv) {
  if (l < 0 || l >= p->nlev) return 1;
  const level *lv = &p->lv[l];
  int n = lv->A.nr;
  if (which == 0) {
    if (!lv->d) return 2;
    memcpy(dv, lv->d, sizeof(double) * (size_t)n);
  } else if (which == 1) {
    if (!lv->dinv) return 2;
    memcpy(dv, lv->dinv, sizeof(double) * (size_t)n);
  } else {
    if (!lv->ilaggr) return 2;
    memcpy(iv, lv->ilaggr, sizeof(int) * (size_t)p->lv[l - 1].A.nr);
  }
  return 0;
}

/* mld_dmlprec_aply_vect (mld_dmlprec_aply.f90:203-357) with outer_sweeps=1,
 * alpha=1, beta=0 */
int orc_prec_apply(orc_prec *p, const double *x, double *y, char trans) {
  if (!p || p->nlev < 1) return 3112; /* apply before build */
  if (trans != 'N' && trans != 'T') return 1;
  /* the GS solvers accept trans = 'N' only (mld_d_gs_solver_apply_vect.f90:68-75) */
  for (int l = 0; l < p->nlev; l++)
    if (p->lv[l].smoother == ORC_FBGS && trans != 'N') return 40;
  int n = p->lv[0].A.nr;
  memcpy(p->x2l[0], x, sizeof(double) * (size_t)n);
  if (p->nlev == 1 && p->lv[0].smoother == ORC_FBGS) {
    /* one-level symmetrized GS (mld_dprecaply.f90:374-409): nswps times
     * w2 = sm(w1), w1 = sm2(w2), one sweep each; y = w1 */
    level *lv = &p->lv[0];
    int nswps = lv->sweeps_pre > lv->sweeps_post ? lv->sweeps_pre : lv->sweeps_post;
    double *w1 = p->ty[0], *w2 = p->y2l[0];
    memcpy(w1, x, sizeof(double) * (size_t)n);
    for (int k = 0; k < nswps; k++) {
      jac_smoother_apply(p, 0, 'N', 1.0, w1, 0.0, w2, 1, 0);
      jac_smoother_apply(p, 0, 'N', 1.0, w2, 0.0, w1, 1, 1);
    }
    memcpy(p->y2l[0], w1, sizeof(double) * (size_t)n);
  } else if (p->nlev == 1) {
    jac_smoother_apply(p, 0, trans, 1.0, p->x2l[0], 0.0, p->y2l[0],
                       p->lv[0].sweeps_pre, 0);
  } else {
    inner_ml_aply(p, 0, trans);
  }
  memcpy(y, p->y2l[0], sizeof(double) * (size_t)n);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Preconditioned CG (method 0) and flexible CG with truncation 1 (method 1;
 * Y. Notay, SIAM J. Sci. Comput. 22 (2000) 1444-1460), stopping on
 * ||r||_2 / ||b||_2 <= eps (PSBLAS istop=2).  PSBLAS 3.5's psb_dcg/psb_dfcg
 * are not in the reference tree; this is the published algorithm. */
int orc_krylov(int method, int n, const int *irp, const int *ja,
               const double *val, orc_prec *prec, const double *b, double *x,
               double eps, int itmax, int *iters, double *relres,
               double *reshist) {
  double *r = (double *)xcalloc((size_t)n, sizeof(double));
  double *z = (double *)xcalloc((size_t)n, sizeof(double));
  double *d = (double *)xcalloc((size_t)n, sizeof(double));
  double *q = (double *)xcalloc((size_t)n, sizeof(double));
  memcpy(r, b, sizeof(double) * (size_t)n);
  orc_spmv(n, irp, ja, val, -1.0, x, 1.0, r);
  double bn2 = sqrt(dot(n, b, b));
  if (bn2 == 0.0) bn2 = 1.0;
  double rn2 = sqrt(dot(n, r, r));
  double err = rn2 / bn2;
  int it = 0;
  double rho = 0.0, dq_prev = 0.0;
  int rc = 0;
  while (err > eps && it < itmax) {
    it++;
    if (prec)
      rc = orc_prec_apply(prec, r, z, 'N');
    else
      memcpy(z, r, sizeof(double) * (size_t)n);
    if (rc) break;
    if (method == 0) {
      double rho_old = rho;
      rho = dot(n, r, z);
      if (it == 1)
        memcpy(d, z, sizeof(double) * (size_t)n);
      else {
        double beta = rho / rho_old;
#pragma omp parallel for schedule(static) if (n > 20000)
        for (int i = 0; i < n; i++) d[i] = z[i] + beta * d[i];
      }
      orc_spmv(n, irp, ja, val, 1.0, d, 0.0, q);
      double sigma = dot(n, d, q);
      double alpha = rho / sigma;
#pragma omp parallel for schedule(static) if (n > 20000)
      for (int i = 0; i < n; i++) {
        x[i] = x[i] + alpha * d[i];
        r[i] = r[i] - alpha * q[i];
      }
    } else {
      if (it == 1) {
        memcpy(d, z, sizeof(double) * (size_t)n);
      } else {
        double beta = dot(n, z, q) / dq_prev; /* (z, A d_prev)/(d_prev, A d_prev) */
#pragma omp parallel for schedule(static) if (n > 20000)
        for (int i = 0; i < n; i++) d[i] = z[i] - beta * d[i];
      }
      orc_spmv(n, irp, ja, val, 1.0, d, 0.0, q);
      double dq = dot(n, d, q);
      double alpha = dot(n, d, r) / dq;
#pragma omp parallel for schedule(static) if (n > 20000)
      for (int i = 0; i < n; i++) {
        x[i] = x[i] + alpha * d[i];
        r[i] = r[i] - alpha * q[i];
      }
      dq_prev = dq;
    }
    rn2 = sqrt(dot(n, r, r));
    err = rn2 / bn2;
    if (reshist) reshist[it - 1] = err;
  }
  *iters = it;
  *relres = err;
  free(r);
  free(z);
  free(d);
  free(q);
  return rc;
}
