/*
 * mld_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the MLD2P4 2.1 multilevel preconditioner (hierarchy
 * build + V-cycle application + CG/FCG) used as the checker for the CUDA
 * path.  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py may load this library; the product never links it.
 *
 * Parity status: the reference (Fortran 2003 + PSBLAS 3.5 + MPI) cannot be
 * compiled on this image (no Fortran compiler, no MPI, no PSBLAS).  The
 * oracle is pinned against the reference's only recorded numeric artefact,
 * tests/fileread/runs/{mld_mat,mld_rhs,mld_sol}.mtx (end-to-end solve), and
 * against analytic known answers.  Per-apply arithmetic of PSBLAS (summation
 * order inside psb_spmm / psb_spsm / psb_spspmm) is "parity unpinned".
 *
 * All indices are 0-based int32, values FP64, CSR rows with ascending
 * column indices.
 */
#ifndef MLD_ORACLE_H
#define MLD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* smoother / solver kinds (values follow mld_base_prec_type.F90 names) */
enum { ORC_JACOBI = 1, ORC_BJAC = 2, ORC_FBGS = 3 };

typedef struct {
  int smoother;        /* ORC_JACOBI: jac smoother + diag solver; ORC_BJAC: jac + ILU(0);
                          ORC_FBGS: jac + forward GS (pre) / backward GS (post) */
  int sweeps_pre;
  int sweeps_post;
  double jac_damp;     /* extension (not in the reference): 1.0 == reference Jacobi */
  int coarse_solver;   /* ORC_BJAC (ILU(0) subsolve) or ORC_JACOBI */
  int coarse_sweeps;
  int min_coarse_size; /* < 0: 40 * floor(n^(1/3)) as mld_d_hierarchy_bld.f90:187-197 */
  int max_levs;        /* default 20 (mld_d_prec_type.f90:92) */
  double min_cr_ratio; /* default 1.5 (mld_d_prec_type.f90:94) */
  double aggr_thresh;  /* default 0.01 (mld_d_onelev_mod.f90:445) */
  int ml_cycle;        /* ORC_VCYCLE (default) or ORC_WCYCLE */
} orc_params;

/* KCYCLE: inner GCR; KCYCLESYM: inner flexible CG (mld_base_prec_type.F90:220-221) */
enum { ORC_VCYCLE = 0, ORC_WCYCLE = 1, ORC_KCYCLE = 2, ORC_KCYCLESYM = 3, ORC_ADD = 4 };

typedef struct orc_prec orc_prec;

void orc_default_params(orc_params *p);

/* ---- problem generator (tests/pdegen/mld_d_pde3d.f90:98-412) ---------- */
/* constant-coefficient 3D convection-diffusion, 7-point centred FD.
 * coef = {a1,a2,a3,b1,b2,b3,c}; h = 1/(idim + hden) (reference: hden=2,
 * benchmark configs: hden=1).  Arrays sized by orc_pde3d_nnz. */
long orc_pde3d_nnz(int idim);
int orc_gen_pde3d(int idim, int hden, const double *coef,
                  int *irp, int *ja, double *val);

/* ---- preconditioner ---------------------------------------------------- */
orc_prec *orc_prec_new(const orc_params *p);
void orc_prec_free(orc_prec *p);
/* copies A; builds hierarchy + smoothers.  returns 0 or an error code. */
int orc_prec_build(orc_prec *p, int n, const int *irp, const int *ja,
                   const double *val);
int orc_prec_nlev(const orc_prec *p);
/* info[0..9]: n, nnzA, nnzP, nnzR, nnzL, nnzU, nnzND, naggr, smoother kind,
 * sweeps_pre ; dinfo[0..1]: omega, damping */
int orc_prec_level_info(const orc_prec *p, int lev, long *info, double *dinfo);
/* which: 0=A 1=P 2=R 3=L 4=U 5=ND ; copies CSR arrays (irp of length nr+1) */
int orc_prec_level_csr(const orc_prec *p, int lev, int which, int *irp,
                       int *ja, double *val);
/* which: 0 = ILU 1/pivot (d), 1 = diag-solver inverse diagonal, 2 = ilaggr */
int orc_prec_level_vec(const orc_prec *p, int lev, int which, double *dv,
                       int *iv);
/* y = M^{-1} x (trans 'N') or M^{-T} x (trans 'T') */
int orc_prec_apply(orc_prec *p, const double *x, double *y, char trans);

/* ---- Krylov (PSBLAS-style CG / flexible CG, istop=2: ||r||/||b||) ----- */
/* method: 0 = CG, 1 = FCG.  prec may be NULL (unpreconditioned). */
int orc_krylov(int method, int n, const int *irp, const int *ja,
               const double *val, orc_prec *prec, const double *b, double *x,
               double eps, int itmax, int *iters, double *relres,
               double *reshist);

/* ---- kernels on single operators (for per-kernel parity tests) -------- */
void orc_spmv(int nr, const int *irp, const int *ja, const double *val,
              double alpha, const double *x, double beta, double *y);
void orc_spmv_t(int nr, int nc, const int *irp, const int *ja,
                const double *val, double alpha, const double *x,
                double beta, double *y);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
