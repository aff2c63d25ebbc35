/*
 * mld_prec.h -- C API of the host-side mirror of MLD2P4's mld_dprec_type.
 *
 * Mirrors the reference's preconditioner object for callers that are not
 * Fortran (C, C++, Python): init / set / hierarchy_build / smoothers_build /
 * build / apply / free / descr, plus the Krylov driver.  The hierarchy is
 * built on the host (C++, the reference's algorithms), uploaded through the
 * mldg C ABI (mldg.h) and applied on the GPU.  Fortran callers keep the
 * reference's own build and call mldg.h directly.
 *
 * Every function returns 0 or an error code; mldp_last_error() gives the text.
 */
#ifndef MLD_PREC_H
#define MLD_PREC_H

#include <stdint.h>

#include "mldg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mldp_prec mldp_prec;

/* allocation of a type(mld_dprec_type) bound to one CUDA device */
int mldp_create(mldp_prec **p, int device);
/* prec%init(ptype): "ML" (multilevel, the reference defaults of
 * mlprec/impl/mld_dprecinit.F90:188-207 with the no-external-library coarse
 * solver), "BJAC" or "JACOBI" (one-level). */
int mldp_init(mldp_prec *p, const char *ptype);
/* prec%set(what, val [, ilev]) (mlprec/impl/mld_dcprecset.F90:78-453).
 * ilev < 0: the reference's default routing over levels.  Integer, real and
 * string forms, as mld_dprecseti / mld_dprecsetr / mld_dprecsetc. */
int mldp_seti(mldp_prec *p, const char *what, int val, int ilev);
int mldp_setr(mldp_prec *p, const char *what, double val, int ilev);
int mldp_setc(mldp_prec *p, const char *what, const char *val, int ilev);
/* prec%hierarchy_build(a, desc_a, info) (impl/mld_d_hierarchy_bld.f90) */
int mldp_hierarchy_build(mldp_prec *p, int n, const int32_t *irp, const int32_t *ja,
                         const double *val);
/* prec%smoothers_build(a, desc_a, info) (impl/mld_d_smoothers_bld.f90) and
 * upload of the hierarchy to the GPU (mldg_upload_level + mldg_finalize) */
int mldp_smoothers_build(mldp_prec *p);
/* The host half of mldp_smoothers_build: the smoother and solver data of
 * every level (ILU(0) factors L, U and pivots, the GS split, the Jacobi
 * off-diagonal part and inverse diagonal) without the upload to the GPU, so
 * that they can be read back (mldp_level_csr / mldp_level_vec) and compared
 * on a machine without a GPU.  No counterpart in the reference. */
int mldp_smoothers_build_host(mldp_prec *p);
/* prec%build = hierarchy_build + smoothers_build (impl/mld_dprecbld.f90) */
int mldp_build(mldp_prec *p, int n, const int32_t *irp, const int32_t *ja, const double *val);
/* prec%apply(x, y, desc_a, info, trans) */
int mldp_apply(mldp_prec *p, const double *x, double *y, char trans, int mem_kind);
/* psb_krylov(method, a, prec, b, x, eps, desc_a, info, itmax, iter, err,
 * istop=2); method "CG" or "FCG"; irp == NULL uses the level-0 matrix. */
int mldp_krylov(mldp_prec *p, const char *method, int n, const int32_t *irp, const int32_t *ja,
                const double *val, const double *b, double *x, double eps, int itmax,
                int *iters, double *err, int mem_kind);
/* hierarchy inspection (for tests and descr) */
int mldp_nlev(const mldp_prec *p);

/* MatrixMarket hierarchy I/O in the file layout of the reference's
 * prec%dump(info, istart=1, prefix=..., ac=.true., rp=.true., smoother=.true.,
 * solver=.true.) (mld_d_prec_type.f90:698-729, mld_d_base_onelev_dump.f90):
 * <prefix>_p000_l<LLL>_{ac,r,p}.mtx for levels >= 2, and the smoother /
 * solver files <prefix>_sm[2a]_p000_l<LLL>_{nd,lower,diag,upper}.mtx.
 * mldp_dump writes the built hierarchy.  mldp_load_dump replaces
 * hierarchy_build + smoothers_build: level 1 is the given matrix, levels
 * 2..nlev and every level's smoother data come from the files (the
 * smoother kind of a level follows from the files present: GS + BWGS ->
 * FBGS, lower/diag/upper -> ILU(0), diag only -> Jacobi), sweeps from set();
 * the hierarchy is then uploaded to the GPU like mldp_smoothers_build. */
int mldp_dump(const mldp_prec *p, const char *prefix);
int mldp_load_dump(mldp_prec *p, const char *prefix, int nlev, int n, const int32_t *irp,
                   const int32_t *ja, const double *val);
/* info[0..9] = n, nnzA, nnzP, nnzR, nnzL, nnzU, nnzND, naggr, smoother kind,
 * sweeps_pre ; dinfo[0..1] = omega, damping */
int mldp_level_info(const mldp_prec *p, int lev, int64_t *info, double *dinfo);
/* which: "A","P","R","L","U","ND"; arrays sized from mldp_level_info */
int mldp_level_csr(const mldp_prec *p, int lev, const char *which, int32_t *irp, int32_t *ja,
                   double *val);
/* which: "d" (ILU 1/pivot or diag inverse), "ilaggr" (level >= 1) */
int mldp_level_vec(const mldp_prec *p, int lev, const char *which, double *dv, int32_t *iv);
/* prec%descr: a text summary of the hierarchy (len includes the NUL) */
int mldp_descr(const mldp_prec *p, char *buf, int len);
/* the GPU handle behind the preconditioner (for timing queries) */
mldg_handle *mldp_gpu(mldp_prec *p);
const char *mldp_last_error(const mldp_prec *p);
/* prec%free */
void mldp_destroy(mldp_prec *p);

/* pdegen-style problem generators (tests/pdegen/mld_d_pde3d.f90:98-412):
 * constant coefficients coef = {a1,a2,a3,b1,b2,b3,c}, h = 1/(idim+hden).
 * nnz from mldp_pde3d_nnz.  Variable kappa: harmonic-mean faces, h=1/(idim+1). */
int64_t mldp_pde3d_nnz(int idim);
int mldp_gen_pde3d(int idim, int hden, const double *coef, int32_t *irp, int32_t *ja,
                   double *val);
int mldp_gen_kappa3d(int idim, const double *kappa, int32_t *irp, int32_t *ja, double *val);

#ifdef __cplusplus
}
#endif
#endif
