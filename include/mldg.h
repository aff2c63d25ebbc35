/*
 * mldg.h -- C ABI of the B200 multilevel preconditioner application.
 *
 * This is the drop-in boundary for MLD2P4 2.1's `prec%apply`: a Fortran
 * 2003 extension of mld_dprec_type overrides psb_d_apply2_vect and reaches
 * these entry points through ISO_C_BINDING (the module mldg_cbind in
 * mld2p4-2_b200/fortran/mldg_cbind.f90).  The level
 * hierarchy built on the host by mld_dprecbld (aggregation, smoothed
 * prolongators, Galerkin products, ILU(0)/diagonal factors) is uploaded
 * unchanged, level by level; the V-cycle then runs on the GPU.
 *
 * Conventions
 *  - int32 indices, FP64 values, CSR with ascending columns per row.
 *  - index_base 0 (C) or 1 (Fortran) for every uploaded CSR.
 *  - Levels are numbered from 0 (finest).  Level l >= 1 carries the maps
 *    between level l-1 and level l, as the reference stores them at level l
 *    (mlprec/impl/mld_dmlprec_aply.f90:376-379): P_l is n_{l-1} x n_l and
 *    R_l = P_l^T is n_l x n_{l-1}.
 *  - All calls on one handle are serialised by the caller; a handle is not
 *    reentrant across threads.  Nothing is allocated per apply.
 *  - Every entry point returns MLDG_SUCCESS (0) or an error code; the
 *    message is available from mldg_last_error().
 */
#ifndef MLDG_H
#define MLDG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes (values follow the reference's info codes) ------------ */
#define MLDG_SUCCESS 0
#define MLDG_ERR_ARG 30              /* invalid argument                     */
#define MLDG_ERR_SIZE 36             /* vector too short (psb info 36)       */
#define MLDG_ERR_NOT_BUILT 3112      /* apply before build (mld_dprecaply.f90:355-360) */
#define MLDG_ERR_NO_SOLVER 1121      /* smoother without solver (jac_smoother_apply_vect.f90:85-89) */
#define MLDG_ERR_NO_DIAG 1124        /* solver without D/DV (ilu_solver_apply_vect.f90:95-104) */
#define MLDG_ERR_TRANS 40            /* invalid trans                        */
#define MLDG_ERR_CUDA 4000           /* CUDA runtime error                   */
#define MLDG_ERR_ALLOC 4010          /* device allocation failed             */
#define MLDG_ERR_TIMEOUT 4020        /* a dependency wait exceeded its limit */
#define MLDG_ERR_NOT_CONVERGED 4030  /* Krylov hit itmax (result still returned) */
#define MLDG_ERR_INTERNAL 4999

/* ---- smoother / solver kinds (mld_base_prec_type.F90 names) ------------- */
#define MLDG_SMOOTHER_JACOBI 1   /* mld_jac_: jac smoother + diag solver      */
#define MLDG_SMOOTHER_BJAC 2     /* mld_bjac_: jac smoother + ILU(0) solver   */
#define MLDG_SMOOTHER_FBGS 3     /* mld_fbgs_: jac smoother + forward GS (pre),
                                    jac smoother + backward GS (post)         */

/* ---- precision forms chosen at finalize -------------------------------- */
#define MLDG_PREC_FP64 0         /* plain FP64 drop-in                        */
#define MLDG_PREC_FP32 1         /* FP32 hierarchy and V-cycle                */
#define MLDG_PREC_FP32_P16 2     /* FP32 V-cycle, FP16 prolongator values with
                                    an FP32 per-row scale                     */
#define MLDG_PREC_FP32_H16 3     /* FP32 V-cycle, FP16 values with an FP32
                                    per-row scale for every level's A, P, R
                                    and Jacobi off-diagonal part (the
                                    single-vector V-cycle; multi-RHS and the
                                    triangular factors read FP32 values)     */

/* ---- Krylov methods of mldg_krylov, mldg_krylov_multi, mldg_krylov_batch */
#define MLDG_METHOD_CG 0         /* psb_krylov('CG', ...)                     */
#define MLDG_METHOD_FCG 1        /* psb_krylov('FCG', ...)                    */

/* ---- memory kinds for vector arguments ---------------------------------- */
#define MLDG_MEM_HOST 0
#define MLDG_MEM_DEVICE 1

typedef struct mldg_handle mldg_handle;

typedef struct {
  int32_t nrows;
  int32_t ncols;
  const int32_t *irp; /* nrows + 1 */
  const int32_t *ja;  /* irp[nrows] - base */
  const double *val;
} mldg_csr;

typedef struct {
  int device;      /* CUDA device ordinal                                   */
  int index_base;  /* 0 or 1                                                 */
  int use_graphs;  /* capture the V-cycle in a CUDA graph (default 1)       */
  int autotune;    /* per-level launch-shape autotuner (default 1)          */
} mldg_opts;

/* One level as produced by the reference's build.  Unused members are
 * zero/NULL.  smoother_kind selects which of (L,U,d) or (ND,d) is used:
 *   MLDG_SMOOTHER_BJAC  : L (unit lower, strictly lower part stored), U
 *                         (unit upper, rows scaled by 1/pivot), d = 1/pivot
 *                         (mld_d_ilu_solver.f90:63-68, mld_dilu0_fact.f90:436-457)
 *   MLDG_SMOOTHER_JACOBI: ND = off-diagonal part, d = 1/a_ii with 0 -> 1
 *                         (mld_d_jac_smoother.f90:56-62, mld_d_diag_solver_bld.f90:86-92)
 *   MLDG_SMOOTHER_FBGS  : L = strictly lower, U = strictly upper triangle of
 *                         A, d = the diagonal a_ii (nonzero): the GS solver's
 *                         tril/triu split (mld_d_gs_solver_bld.f90:73-81);
 *                         pre-smoothing sweeps are forward GS, post-smoothing
 *                         sweeps backward GS (mld_d_base_onelev_cseti.F90:128-132).
 *                         trans 'T' is rejected like the reference's GS solver
 *                         (mld_d_gs_solver_apply_vect.f90:68-75, MLDG_ERR_TRANS).
 *                         A one-level hierarchy applies forward then backward GS
 *                         max(sweeps_pre, sweeps_post) times (mld_dprecaply.f90:374-409).
 * Level l >= 1 also carries P and R (mld_d_onelev_mod.f90:122-158, map).
 * sweeps_pre/sweeps_post: mld_dml_parms (the coarsest level uses
 * sweeps_pre, mld_dmlprec_aply.f90:787-793).  damping: extension, 1.0 is the
 * reference Jacobi iteration. */
typedef struct {
  mldg_csr A;
  mldg_csr P;
  mldg_csr R;
  mldg_csr ND;
  mldg_csr L;
  mldg_csr U;
  const double *d;
  int smoother_kind;
  int sweeps_pre;
  int sweeps_post;
  double damping;
} mldg_level_desc;

/* replaces: type(mld_dprec_type) allocation + prec%init
 * (mlprec/mld_d_prec_type.f90:84-110, impl/mld_dprecinit.F90:188-207) */
int mldg_create(mldg_handle **h, const mldg_opts *opts);

/* replaces: the per-level data left by prec%hierarchy_build +
 * prec%smoothers_build (impl/mld_d_hierarchy_bld.f90:66-490,
 * impl/mld_d_smoothers_bld.f90:156-169).  Copies the arrays to the device;
 * the library owns its copies.  Levels may be uploaded in any order. */
int mldg_upload_level(mldg_handle *h, int lev, const mldg_level_desc *desc);

/* Freezes the hierarchy of nlev levels: transposes, triangular-solve
 * schedules, precision conversion, work vectors, autotuning, graph capture.
 * precision: MLDG_PREC_*.  replaces: the end of mld_dprecbld
 * (impl/mld_dprecbld.f90:60-159). */
int mldg_finalize(mldg_handle *h, int nlev, int precision);

/* Multilevel cycle of every later apply: MLDG_CYCLE_V (default);
 * MLDG_CYCLE_W, which repeats the coarse correction once from the updated
 * residual before post-smoothing (mld_dmlprec_aply.f90:716-745);
 * MLDG_CYCLE_K / MLDG_CYCLE_KSYM, the K-cycle: on every level below the
 * second, at most two steps of GCR (K) or flexible CG (KSYM) with the next
 * level's cycle as preconditioner, the second step only if the first left
 * more than 0.25 of the level residual (mld_dmlprec_aply.f90:811-1184).  The
 * K-cycle decides on the host between its kernels, so its applies are not
 * replayed from CUDA graphs, a multi-column apply runs column by column, and
 * mldg_krylov_multi / mldg_krylov_batch reject it.  May be called before or
 * after mldg_finalize.  replaces: prec%set('ML_CYCLE', 'VCYCLE' | 'WCYCLE' |
 * 'KCYCLE' | 'KCYCLESYM') (mld_base_prec_type.F90:430-439). */
#define MLDG_CYCLE_V 0
#define MLDG_CYCLE_W 1
#define MLDG_CYCLE_K 2
#define MLDG_CYCLE_KSYM 3
/* MLDG_CYCLE_ADD: the additive cycle, smoothing and coarse corrections of the
 * restricted input summed (mld_dmlprec_aply.f90:464-588, ML_CYCLE='ADD') */
#define MLDG_CYCLE_ADD 4
int mldg_set_cycle(mldg_handle *h, int cycle);

/* y = M^{-1} x (trans 'N') or y = M^{-T} x (trans 'T'/'C') for nrhs vectors
 * stored column by column with leading dimension ld (ld >= n).
 * mem_kind: MLDG_MEM_HOST or MLDG_MEM_DEVICE for both x and y.
 * nrhs > 1 runs blocks of up to 32 columns through one multi-vector V-cycle
 * (every kernel works on all columns of the block at once); the result of
 * each column is that of nrhs = 1 up to rounding order.
 * replaces: prec%apply(x,y,desc_a,info,trans,work) ->
 *   mld_dprecaply2_vect (mlprec/impl/mld_dprecaply.f90:305-443) ->
 *   mld_dmlprec_aply_vect (mlprec/impl/mld_dmlprec_aply.f90:203-357). */
int mldg_apply(mldg_handle *h, const double *x, double *y, char trans,
               int nrhs, int ld, int mem_kind);

/* Flexible CG (truncation 1) in FP64 on the GPU with this preconditioner,
 * stopping on ||b - A x||_2 / ||b||_2 <= tol (PSBLAS istop = 2).  A may be
 * NULL to use the finest uploaded level matrix.  x holds the initial guess
 * on entry.  method: 0 = CG, 1 = FCG.
 * replaces: psb_krylov('FCG'|'CG', a, prec, b, x, eps, desc_a, info, itmax,
 * iter, err, istop=2) as called at tests/pdegen/mld_d_pde3d.f90:753-755. */
int mldg_krylov(mldg_handle *h, int method, const mldg_csr *A,
                const double *b, double *x, double tol, int itmax,
                int *iters, double *relres, int mem_kind);

/* nrhs independent CG/FCG solves A x_c = b_c sharing this preconditioner,
 * advanced together in blocks of up to 32 columns (one multi-vector V-cycle
 * and SpMM per iteration, per-column scalars).  b and x are column-major with
 * leading dimensions ldb, ldx >= n; x holds the initial guesses.  Each column
 * stops on its own ||b_c - A x_c||_2 / ||b_c||_2 <= tol and is frozen from
 * then on; iters[c] and relres[c] report it.  Returns MLDG_ERR_NOT_CONVERGED
 * if a column reached itmax above tol.  No counterpart in the reference (a
 * caller there loops psb_krylov over the right-hand sides). */
int mldg_krylov_multi(mldg_handle *h, int method, const mldg_csr *A, int nrhs,
                      const double *b, int ldb, double *x, int ldx, double tol,
                      int itmax, int *iters, double *relres, int mem_kind);

/* nsys independent systems, each with its own finalized handle (hierarchy
 * and finest-level matrix A_i, all on one device), solved together by CG/FCG
 * in FP64 in ONE graph launch: the systems' initial residuals, then a loop
 * whose every iteration runs, as concurrent branches, the V-cycle (in the
 * handle's precision) and the CG/FCG step of each unfinished system; the
 * stopping tests run on the device and the loop ends when the last system
 * has finished.  The graph is captured on the first call with these handles
 * (kept for later calls until one of them is finalized again or destroyed);
 * handles with a K-cycle, use_graphs = 0 or a probe set are rejected.  b[i],
 * x[i] are vectors of handle i's size (x[i] holds the initial guess); each
 * system stops on its own ||b_i - A_i x_i||_2 / ||b_i||_2 <= tol.  Results
 * equal mldg_krylov on each handle.  *ms (optional) receives the device time
 * of the whole batch.  No counterpart in the reference. */
int mldg_krylov_batch(int nsys, mldg_handle *const *h, int method, const double *const *b,
                      double *const *x, double tol, int itmax, int *iters, double *relres,
                      int mem_kind, double *ms);

/* Adjoint solve A^T lambda = g with flexible CG in FP64, preconditioned by
 * the transposed V-cycle M^{-T} (the reference's trans='T' apply,
 * mld_dmlprec_aply.f90:634-656,765-777: smoothers swapped, A^T residuals,
 * U^T/L^T triangular solves).  lambda holds the initial guess on entry;
 * stops on ||g - A^T lambda||_2 / ||g||_2 <= tol.  No counterpart as an entry
 * point in the reference (it composes psb_krylov with trans='T'). */
int mldg_adjoint(mldg_handle *h, const double *g, double *lambda, double tol, int itmax,
                 int *iters, double *relres, int mem_kind);

/* dL/dkappa for -div(kappa grad u) = f assembled by the harmonic-mean face
 * rule on idim^3 cells (h = 1/(idim+1), zero Dirichlet boundary faces taking
 * the cell's own kappa): given the forward solution x and the adjoint
 * lambda (A^T lambda = dL/dx),
 *   grad[c] = -(1/h^2) [ sum_{interior faces (c,s)} 2 kappa_s^2/(kappa_c+kappa_s)^2
 *                           (lambda_c - lambda_s)(x_c - x_s)
 *                        + (boundary faces of c) lambda_c x_c ].
 * One thread per cell, no atomics.  No counterpart in the reference. */
int mldg_kappa_grad(mldg_handle *h, int idim, const double *kappa, const double *x,
                    const double *lambda, double *grad, int mem_kind);

/* Per-level sizes of the finalized hierarchy:
 * info[0..4] = n, nnz(A), nnz(P), nnz(L)+nnz(U)+nnz(ND), number of levels. */
int mldg_level_info(const mldg_handle *h, int lev, int64_t *info);

/* Device time (ms) of the last mldg_apply / mldg_krylov, measured with CUDA
 * events on the handle's stream, and the number of kernel launches it made. */
int mldg_last_timing(const mldg_handle *h, double *ms, int64_t *launches);

/* Algorithmic bytes of one V-cycle apply (trans 'N') in the finalized
 * precision: every sparse operand of the reference's operation sequence
 * (mld_dmlprec_aply.f90:590-809) once, CSR bytes nnz*(value + index size) +
 * 4*(rows+1), plus every dense vector operand read once and every output
 * written once (the roofline numerator).  A level whose ILU(0) or GS solves
 * run as products with an explicit dense inverse counts the sparse factors
 * it stands for.  Valid after the first apply. */
int mldg_apply_bytes(const mldg_handle *h, int64_t *bytes);
/* Bytes the chosen kernels of one V-cycle apply move: as mldg_apply_bytes,
 * except that a dense-inverse product counts its n*n matrix.  No counterpart
 * in the reference. */
int mldg_apply_impl_bytes(const mldg_handle *h, int64_t *bytes);

/* ---- diagnostics: per-kernel device time ------------------------------- */
#define MLDG_KERNEL_TRSV 1    /* sparse unit-triangular solve (ILU factors)   */
#define MLDG_KERNEL_SPMV 2    /* CSR SpMV family: residual, R, P             */
#define MLDG_KERNEL_JACOBI 3  /* fused point-Jacobi sweep                    */
#define MLDG_KERNEL_VEC 4     /* vector kernels (diag, fill, cast, axpby)   */

typedef struct {
  int kind;       /* MLDG_KERNEL_*                                            */
  int level;      /* level the launch works on                               */
  int64_t bytes;  /* algorithmic bytes of the launch                         */
  double ms;      /* device time between CUDA events around the launch       */
} mldg_kernel_stat;

/* Brackets, in every later V-cycle (graph replays included), the index-th
 * launch of kernel class `kind` on level `lev` with two CUDA events on the
 * launching stream; kind 0 disables the probe.  Takes effect at the next
 * graph capture (the call drops captured graphs). */
int mldg_probe_set(mldg_handle *h, int kind, int lev, int index);
/* Accumulated device time of the probed launch since the last read, the
 * number of probed launches, and the algorithmic bytes of one of them. */
int mldg_probe_read(mldg_handle *h, double *total_ms, int64_t *count, int64_t *bytes);

/* Runs one V-cycle (trans 'N'/'T') on the current level-0 input without a
 * graph, with CUDA events around every launch; writes up to max entries. */
int mldg_profile(mldg_handle *h, char trans, int max, mldg_kernel_stat *stats, int *n);
/* The same for the multi-vector V-cycle of mldg_apply with nrhs (2..32)
 * columns (nrhs = 1 is mldg_profile). */
int mldg_profile_multi(mldg_handle *h, char trans, int nrhs, int max, mldg_kernel_stat *stats,
                       int *n);

/* ---- allocation-free relative residual --------------------------------- */
/* No counterpart in the reference.  For callers that must not allocate
 * device memory: applications whose memory pool or allocator owns every
 * device byte (a second allocator would fragment or overcommit it), and
 * convergence checks in tight host loops, where cudaMalloc / cudaFree would
 * synchronise the whole device on every call.
 *
 * Computes *relres = ||b - A x||_2 / ||b||_2 (1 when ||b|| = 0).  A's arrays
 * and x, b are DEVICE pointers, 0-based CSR, nrows == ncols == n.  The
 * residual vector and the reduction partials live in one file-scope device
 * array of MLDG_NOALLOC_MAX_N + 1024 doubles (about 4 MiB) that every GPU
 * loading the library keeps until exit; n > MLDG_NOALLOC_MAX_N is rejected
 * with MLDG_ERR_SIZE.  Nothing is allocated: the first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) once, so make that
 * first call before any stream capture.  All calls share the array and it
 * keeps the last call's contents; calls that overlap on the GPU (other
 * streams, other threads) race on it.  Runs on the handle's stream, copies
 * the result to the host and waits for it: the call returns with *relres
 * set. */
#define MLDG_NOALLOC_MAX_N 524288
int mldg_relres_noalloc(mldg_handle *h, const mldg_csr *A, const double *x, const double *b,
                        double *relres);

/* ---- hierarchy set-up on the GPU --------------------------------------- */
/* ILU(0) factorisation of A (0-based CSR, n x n, ascending columns) on the
 * GPU, bit for bit the reference's row-by-row factorisation
 * (mlprec/impl/mld_dilu0_fact.f90:284-477 with the row split of ilu_copyin
 * :551-660): L unit lower (strict part stored), U unit upper (strict part,
 * rows scaled by 1/pivot), d = 1/pivot -- the MLDG_SMOOTHER_BJAC data of
 * mldg_level_desc.  Rows of one dependency level are factorised together,
 * each in the host's operation order without fused multiply-adds.  Host
 * arrays: Lirp, Uirp n + 1; Lja, Lval, Uja, Uval room for nnz(A) entries; d
 * n.  Returns MLDG_SUCCESS, or 2 with *bad_row = the first row whose pivot
 * is below 1.11e-16 (the reference's "pivot too small", :436-445), or an
 * error code.  *ms (optional): device time.  Allocates its own device
 * scratch (freed before return) and does not need a handle. */
int mldg_ilu0_factor(int device, const mldg_csr *A, int32_t *Lirp, int32_t *Lja, double *Lval, int32_t *Uirp,
                     int32_t *Uja, double *Uval, double *d, int *bad_row, double *ms);

/* C = A B (0-based CSR, ascending columns; A m x k, B k x n) on the GPU, bit
 * for bit the host build's row-by-row (Gustavson) product that stands in for
 * psb_spspmm in the smoothed prolongator and the Galerkin product
 * (mlprec/impl/mld_daggrmat_smth_asb.f90:316,345,399): row i takes a_ik in
 * stored order and, for each, row k of B in stored order; a column's first
 * contribution is assigned, later ones added, every product and sum rounded
 * on its own; columns ascending.  One warp per row, lanes across the
 * distinct columns of a row of B; rows with more than 1,536 distinct
 * columns are formed on the host in the same order.  *Cirp (m + 1), *Cja,
 * *Cval (nnz) are allocated by the library (release each with mldg_free);
 * *ms (optional): device time.  Allocates and frees its own device scratch;
 * needs no handle. */
int mldg_spgemm(int device, const mldg_csr *A, const mldg_csr *B, int32_t **Cirp, int32_t **Cja, double **Cval,
                int *Cnrows, int *Cncols, double *ms);
void mldg_free(void *p);

const char *mldg_last_error(const mldg_handle *h);

/* replaces: prec%free (mlprec/mld_d_prec_type.f90:537-568) */
void mldg_destroy(mldg_handle *h);

#ifdef __cplusplus
}
#endif
#endif
