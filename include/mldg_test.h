/*
 * mldg_test.h -- test hooks of libmldgpu.so (no counterparts in the reference).
 *
 * mldg_rep_plan_check checks the plans of the replicated-window cluster
 * solve (the kernel that runs the large ILU(0) levels) without a GPU: it
 * builds the plans of an ILU(0) pair exactly as mldg_finalize would and
 * replays them through a host emulation of the kernel, in the kernel's step
 * order, checking every ring read against the position its slot holds, every
 * far read and reset, and every plan block against its descriptor.
 * mldg_test_set_spin_limit makes dependency waits run out on purpose
 * (failure detection without a GPU fault).
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

/* Builds the partitioned-solve plan (k_trsv_blk) of the strictly triangular
 * factor T (0-based CSR, n x n; upper != 0: an upper factor, walked in
 * reverse) with nblocks blocks, exactly as mldg_finalize would, and replays
 * it through a host emulation of the kernel: blocks in ticket order, steps
 * in order, every plan access checked against its buffer, every ring read
 * against the row that slot holds, every remote read against a written
 * value, no slot overwritten while its step reads it.  t = scale o rhs -
 * T_strict t (scale may be NULL).  stats[6]: violations, steps, ring size,
 * plan usable (1) or not (0, t untouched), blocks, shared memory bytes.
 * Returns MLDG_SUCCESS or an error code. */
int mldg_blk_plan_check(const mldg_csr *T, int upper, const double *scale, const double *rhs, double *t,
                        int nblocks, int fp32, long long *stats);

/* Polls a sentinel wait of the sync-free and ELL triangular solves makes
 * before it gives up with MLDG_ERR_TIMEOUT, on `device`; polls < 0 restores
 * the default (2^22).  A test lowers it (0: give up at the first poll that
 * finds a dependency not yet written) to make a solve's waits run out on
 * purpose, then checks that the call returns MLDG_ERR_TIMEOUT, that the
 * kernel ends, and that the next apply on the same handle is correct.  The
 * mbarrier waits of the window and cluster solves keep their own limit.
 * Returns MLDG_SUCCESS or MLDG_ERR_CUDA. */
int mldg_test_set_spin_limit(int device, int polls);

#ifdef __cplusplus
}
#endif

#endif /* MLDG_TEST_H */
