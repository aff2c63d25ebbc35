"""CPU: plans of the partitioned triangular solve (k_trsv_blk), run through the
library's host emulation of the kernel (mldg_blk_plan_check).

The emulation takes the blocks in ticket order and the steps in order, and
checks every access the kernel makes: each plan block inside the plan and
within a shared-memory stage, each row's entry range, each ring read against
the row its slot holds (no slot overwritten while its step still reads it),
each remote read against a value already written, every row solved once.
The emulated solve must match a direct triangular solve of the same factor
(the ILU(0) factors of pdegen problems, lower and upper, in both precisions,
for several block counts, with the U solve's right-hand side scaled by the
ILU pivots as in the V-cycle)."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from conftest import ANISO, ISO, oracle_params


def _factors(orc, idim, coef, lev):
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=50))
    op.build(a)
    return op.level_csr(lev, "L"), op.level_csr(lev, "U"), op.level_vec(lev, "d")


def _check(mld, M, upper, scale, P, fp32):
    lib = mld.lib()
    f = lib.mldg_blk_plan_check
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    n = M.nrows
    Mc = mld.CSR(M.irp, M.ja, M.val, ncols=n).c()
    x = np.random.default_rng(n + P).uniform(-1, 1, n)
    t = np.zeros(n)
    st = np.zeros(6, np.int64)
    rc = f(C.byref(Mc), 1 if upper else 0, scale.ctypes.data if scale is not None else None, x.ctypes.data,
           t.ctypes.data, P, fp32, st.ctypes.data)
    assert rc == 0
    Ms = (sp.csr_matrix((M.val, M.ja, M.irp), shape=(n, n)) + sp.identity(n)).tocsr()
    rhs = x * scale if scale is not None else x
    ref = sla.spsolve_triangular(Ms, rhs, lower=not upper)
    return st, np.linalg.norm(t - ref) / np.linalg.norm(ref)


@pytest.mark.parametrize("idim,coef,lev", [(24, ISO, 0), (40, ISO, 1), (36, ANISO, 0), (48, ANISO, 1)])
@pytest.mark.parametrize("P", [1, 7, 64, 148])
def test_blk_plan_emulation(mld, orc, idim, coef, lev, P):
    Lm, Um, d = _factors(orc, idim, coef, lev)
    for fp32, tol in ((0, 1e-13), (1, 1e-5)):
        for M, upper, scale in ((Lm, False, None), (Um, True, d)):
            st, err = _check(mld, M, upper, scale, P, fp32)
            assert st[3] == 1, "plan not usable"
            assert st[0] == 0, f"{st[0]} violations"
            assert st[4] == min(P, M.nrows)
            assert st[5] <= 220 * 1024
            assert err <= tol, (fp32, upper, err)


def test_blk_plan_transposed_factors(mld, orc):
    """The trans 'T' solves run on U^T (lower) and L^T (upper)."""
    Lm, Um, d = _factors(orc, 30, ISO, 0)
    n = Lm.nrows
    for M, upper in ((Um, True), (Lm, False)):
        S = sp.csr_matrix((M.val, M.ja, M.irp), shape=(n, n)).T.tocsr()
        S.sort_indices()
        T = type(M)(S.indptr, S.indices, S.data, ncols=n)
        st, err = _check(mld, T, not upper, d if not upper else None, 37, 0)
        assert st[3] == 1 and st[0] == 0 and err <= 1e-13
