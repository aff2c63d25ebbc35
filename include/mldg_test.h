/*
 * mldg_test.h -- host-only test hook of libmldgpu.so.
 *
 * No counterpart in the reference: it checks the plans of the replicated-
 * window cluster solve (the kernel that runs the large ILU(0) levels) without
 * a GPU.  It builds the plans of an ILU(0) pair exactly as mldg_finalize
 * would and replays them through a host emulation of the kernel, in the
 * kernel's step order, checking every ring read against the position its
 * slot holds, every far read and reset, and every plan block against its
 * descriptor.
 */
#ifndef MLDG_TEST_H
#define MLDG_TEST_H

#include "mldg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* L, U: strict triangles of the ILU(0) factors (0-based CSR, n x n); d: the
 * diagonal scaling between them; x: right-hand side.  trans 'N': y =
 * U^{-1} diag(d) L^{-1} x; 'T': y = L^{-T} diag(d) U^{-T} x.  cluster: 8 or
 * 16 CTAs; fp32 != 0 plans the FP32 form.  stats[4]: plan violations, steps
 * of the first solve, far entries of both plans, plans usable (1) or not (0,
 * y untouched).  Returns MLDG_SUCCESS or MLDG_ERR_ARG. */
int mldg_rep_plan_check(const mldg_csr *L, const mldg_csr *U, const double *d, const double *x,
                        double *y, int cluster, int fp32, char trans, long long *stats);

#ifdef __cplusplus
}
#endif

#endif /* MLDG_TEST_H */
