"""CPU: the slow convergence of FCG with the BJAC-ILU(0) V-cycle on the
anisotropic convection-diffusion problem is a property of the method, not
of the oracle's (or the product's) ILU(0) or V-cycle.

Everything here is independent of the oracle's C code except the
hierarchy's integer structure and Galerkin matrices (A, P, R of every
level):

* an ILU(0) factorisation written here (textbook IKJ elimination restricted
  to the pattern of A, mlprec/impl/mld_dilu0_fact.f90:364-457 is the
  reference's) reproduces the oracle's L, U and pivots of every level;
* a V-cycle written here with numpy/scipy triangular solves on those
  factors (mlprec/impl/mld_dmlprec_aply.f90:590-809, one BJAC sweep per
  side, one ILU(0) solve on the coarsest level) reproduces the oracle's
  apply;
* with that V-cycle, scipy's own (standard) CG does not reach 1e-10 on the
  anisotropic problem in 300 iterations, while it needs ~10 on the
  isotropic one; the oracle's flexible CG still converges at this small
  size but needs several times its isotropic count and more than the
  point-Jacobi V-cycle.  The BJAC-ILU(0) V-cycle is not symmetric, and on
  this convection-dominated anisotropic problem a CG-type method preconditioned
  by it degrades whoever implements it -- at idim=160 the flexible CG of the
  oracle and of the GPU path stall alike.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from conftest import ANISO, ISO, oracle_params

IDIM = 32


def to_scipy(m):
    return sp.csr_matrix((np.asarray(m.val), np.asarray(m.ja), np.asarray(m.irp)), shape=(m.nrows, m.ncols))


def ilu0(a):
    """ILU(0) of a CSR matrix with sorted columns: L strict lower (unit
    diagonal implied), U strict upper scaled by 1/pivot (unit diagonal
    implied), d = 1/pivot -- the layout of the reference's ILU solver."""
    a = a.tocsr().copy()
    a.sort_indices()
    n = a.shape[0]
    irp, ja, val = a.indptr, a.indices, a.data.astype(np.float64).copy()
    diag = np.full(n, -1, dtype=np.int64)
    pos = [dict() for _ in range(n)]
    for i in range(n):
        for k in range(irp[i], irp[i + 1]):
            pos[i][ja[k]] = k
            if ja[k] == i:
                diag[i] = k
    for i in range(n):
        for kk in range(irp[i], irp[i + 1]):
            k = ja[kk]
            if k >= i:
                break
            val[kk] /= val[diag[k]]
            lik = val[kk]
            for jj in range(diag[k] + 1, irp[k + 1]):
                p = pos[i].get(ja[jj])
                if p is not None:
                    val[p] -= lik * val[jj]
    piv = val[diag]
    row = np.repeat(np.arange(n), np.diff(irp))
    lo = sp.csr_matrix((np.where(ja < row, val, 0.0), ja.copy(), irp.copy()), shape=(n, n))
    up = sp.csr_matrix((np.where(ja > row, val, 0.0), ja.copy(), irp.copy()), shape=(n, n))
    lo.eliminate_zeros()
    up.eliminate_zeros()
    d = 1.0 / piv
    up = sp.diags(d) @ up
    return lo.tocsr(), up.tocsr(), d


def build(orc, coef, smoother):
    a = orc.gen_pde3d(IDIM, 1, coef)
    op = orc.Prec(oracle_params(orc, smoother, 1 if smoother == "BJAC" else 2,
                                1.0 if smoother == "BJAC" else 0.8, coarse_sweeps=4, mcs=300))
    op.build(a)
    return a, op


class NumpyBjacVcycle:
    """The V-cycle of the reference with BJAC-ILU(0) smoothers, written with
    scipy triangular solves on independently computed factors."""

    def __init__(self, orc, op):
        self.nlev = op.nlev
        self.A = [to_scipy(op.level_csr(l, "A")) for l in range(self.nlev)]
        self.P = [None] + [to_scipy(op.level_csr(l, "P")) for l in range(1, self.nlev)]
        self.R = [None] + [to_scipy(op.level_csr(l, "R")) for l in range(1, self.nlev)]
        self.f = [ilu0(self.A[l]) for l in range(self.nlev)]
        n = self.A[0].shape[0]
        self.eye = [sp.identity(self.A[l].shape[0], format="csr") for l in range(self.nlev)]
        self.n = n

    def ilu_solve(self, l, x):
        lo, up, d = self.f[l]
        w = spla.spsolve_triangular(lo + self.eye[l], x, lower=True, unit_diagonal=True)
        return spla.spsolve_triangular(up + self.eye[l], d * w, lower=False, unit_diagonal=True)

    def apply(self, x, l=0):
        if l == self.nlev - 1:
            return self.ilu_solve(l, x)
        y = self.ilu_solve(l, x)
        yc = self.apply(self.R[l + 1] @ (x - self.A[l] @ y), l + 1)
        y = y + self.P[l + 1] @ yc
        return y + self.ilu_solve(l, x - self.A[l] @ y)


@pytest.fixture(scope="module")
def aniso_bjac(orc):
    a, op = build(orc, ANISO, "BJAC")
    return a, op, NumpyBjacVcycle(orc, op)


def test_independent_ilu0_matches_oracle(orc, aniso_bjac):
    _, op, v = aniso_bjac
    for l in range(op.nlev):
        lo, up, d = v.f[l]
        Lo, Uo = to_scipy(op.level_csr(l, "L")), to_scipy(op.level_csr(l, "U"))
        do = op.level_vec(l, "d")
        assert np.max(np.abs(d - do)) <= 1e-13 * np.max(np.abs(do))
        for m, mo in ((lo, Lo), (up, Uo)):
            diff = abs(m - mo)
            assert (diff.max() if diff.nnz else 0.0) <= 1e-13 * abs(mo).max()


def test_independent_vcycle_matches_oracle(orc, aniso_bjac):
    a, op, v = aniso_bjac
    x = np.random.default_rng(0).uniform(-1, 1, a.nrows)
    y, y_ref = v.apply(x), op.apply(x)
    assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref)


def _scipy_cg_iterations(A, b, M, maxiter):
    its = [0]

    def cb(_):
        its[0] += 1
    _, info = spla.cg(A, b, rtol=1e-10, atol=0.0, maxiter=maxiter, M=M, callback=cb)
    return its[0], info


def test_bjac_slow_on_anisotropic_problem_independently(orc, aniso_bjac):
    a, op, v = aniso_bjac
    b = np.random.default_rng(0).uniform(-1, 1, a.nrows)
    A = to_scipy(a)
    it_cg_aniso, info_aniso = _scipy_cg_iterations(A, b, spla.LinearOperator(A.shape, matvec=v.apply), 300)
    _, it_fcg_aniso, rr_aniso, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    # the same method on the isotropic problem
    ai, opi = build(orc, ISO, "BJAC")
    vi = NumpyBjacVcycle(orc, opi)
    Ai = to_scipy(ai)
    bi = np.random.default_rng(0).uniform(-1, 1, ai.nrows)
    it_cg_iso, info_iso = _scipy_cg_iterations(Ai, bi, spla.LinearOperator(Ai.shape, matvec=vi.apply), 300)
    _, it_fcg_iso, _, _ = orc.krylov("FCG", ai, opi, bi, eps=1e-10)
    # the point-Jacobi V-cycle on the anisotropic problem (oracle FCG)
    aj, opj = build(orc, ANISO, "JACOBI")
    _, it_fcg_jac, _, _ = orc.krylov("FCG", aj, opj, b, eps=1e-10)
    # independent standard CG: converges on the isotropic problem, stalls on
    # the anisotropic one
    assert info_iso == 0 and it_cg_iso <= 15, it_cg_iso
    assert info_aniso != 0 and it_cg_aniso == 300
    # the oracle's flexible CG: converges here, but degraded
    assert rr_aniso <= 1e-10
    assert it_fcg_aniso >= 3 * it_fcg_iso and it_fcg_aniso > it_fcg_jac, (it_fcg_aniso, it_fcg_iso, it_fcg_jac)
