"""CPU: the oracle against the reference's recorded fixture and known answers."""
import os

import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params

GOLD = os.path.join(os.path.dirname(__file__), "golden", "fileread_fixture.npz")


def test_fixture_solution(orc):
    """tests/fileread/runs: 4096-row 2D Laplacian, recorded rhs and solution."""
    f = np.load(GOLD)
    a = orc.CSR(f["irp"], f["ja"], f["val"])
    # the fixture is the 64x64 five-point Laplacian with h = 1/66
    assert a.nrows == 4096 and a.nnz == 20224
    assert np.allclose(a.to_scipy().diagonal(), 4 * 66.0 ** 2)
    for sm in (orc.BJAC, orc.JACOBI):
        p = orc.Prec(orc.default_params(smoother=sm))
        p.build(a)
        x, it, rr, _ = orc.krylov("CG", a, p, f["rhs"], eps=1e-12)
        assert rr <= 1e-12
        # the recorded solution has residual 1.36e-10, so agreement is bounded by it
        assert np.linalg.norm(x - f["sol"]) / np.linalg.norm(f["sol"]) < 1e-9


def test_ilu0_exact_on_tridiagonal(orc):
    """ILU(0) of a tridiagonal matrix is its exact LU: one-level BJAC gives A^{-1}."""
    n = 50
    rng = np.random.default_rng(0)
    main = 4 + rng.uniform(0, 1, n)
    off = -rng.uniform(0.5, 1.5, n - 1)
    import scipy.sparse as sp
    m = sp.diags([off, main, off * 0.7], [-1, 0, 1], format="csr")
    m.sort_indices()
    a = orc.CSR(m.indptr, m.indices, m.data)
    p = orc.Prec(orc.default_params(smoother=orc.BJAC, max_levs=1))
    p.build(a)
    assert p.nlev == 1
    x = rng.uniform(-1, 1, n)
    y = p.apply(x)
    assert np.allclose(m @ y, x, rtol=0, atol=1e-12 * np.abs(x).max())


@pytest.mark.parametrize("smoother", ["BJAC", "JACOBI"])
def test_transpose_consistency(orc, smoother):
    """<M^{-1} x, z> = <x, M^{-T} z> (the reference's own trans='T' branch)."""
    a = orc.gen_pde3d(12, 1, ANISO)
    p = orc.Prec(oracle_params(orc, smoother, 2 if smoother == "JACOBI" else 1, mcs=100))
    p.build(a)
    rng = np.random.default_rng(1)
    x, z = rng.uniform(-1, 1, a.nrows), rng.uniform(-1, 1, a.nrows)
    lhs = p.apply(x, "N") @ z
    rhs = x @ p.apply(z, "T")
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_symmetric_operator_gives_symmetric_preconditioner(orc):
    """Symmetric A, Jacobi smoother, R = P^T: M^{-1} is symmetric."""
    a = orc.gen_pde3d(10, 1, (1, 1, 1, 0, 0, 0, 0))
    p = orc.Prec(oracle_params(orc, "JACOBI", 1, coarse_sweeps=1, mcs=60))
    p.build(a)
    rng = np.random.default_rng(2)
    x, z = rng.uniform(-1, 1, a.nrows), rng.uniform(-1, 1, a.nrows)
    assert abs(p.apply(x) @ z - x @ p.apply(z)) <= 1e-12 * abs(p.apply(x) @ z)


def test_fbgs_symmetric_and_forward_only(orc):
    """FBGS (forward GS pre, backward GS post) with R = P^T on a symmetric
    operator gives a symmetric V-cycle; the GS solvers reject trans 'T'
    (mld_d_gs_solver_apply_vect.f90:68-75)."""
    a = orc.gen_pde3d(10, 1, (1, 1, 1, 0, 0, 0, 0))
    for sweeps in (1, 2):
        p = orc.Prec(oracle_params(orc, "FBGS", sweeps, coarse_sweeps=1, mcs=60))
        p.build(a)
        assert p.nlev >= 2 and p.level_info(0)["smoother"] == orc.FBGS
        rng = np.random.default_rng(3)
        x, z = rng.uniform(-1, 1, a.nrows), rng.uniform(-1, 1, a.nrows)
        assert abs(p.apply(x) @ z - x @ p.apply(z)) <= 1e-12 * abs(p.apply(x) @ z)
        with pytest.raises(RuntimeError):
            p.apply(x, "T")


def test_gauss_seidel_exact_on_triangular(orc):
    """One-level FBGS on a lower-triangular matrix: the forward sweep is an
    exact solve (U = 0), and the backward sweep of the exact solution of a
    diagonal-only system returns D^{-1} x."""
    n = 30
    rng = np.random.default_rng(5)
    rows, cols, vals = [], [], []
    for i in range(n):
        for j in range(max(0, i - 2), i + 1):
            rows.append(i)
            cols.append(j)
            vals.append(4.0 + i if j == i else rng.uniform(-1, 1))
    import scipy.sparse as sp
    m = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    m.sort_indices()
    a = orc.CSR(m.indptr.astype(np.int32), m.indices.astype(np.int32), m.data)
    p = orc.Prec(orc.default_params(smoother=orc.FBGS, max_levs=1))
    p.build(a)
    x = rng.uniform(-1, 1, n)
    y = p.apply(x)
    # y = (D+U)^{-1} (D+L)^{-1} x with U = 0: y = D^{-1} A^{-1} x
    ref = np.linalg.solve(np.diag(m.diagonal()), np.linalg.solve(m.toarray(), x))
    assert np.linalg.norm(y - ref) <= 1e-13 * np.linalg.norm(ref)


def test_wcycle_symmetric_and_not_weaker(orc):
    """W-cycle on a symmetric operator with a symmetric smoother pair stays
    symmetric, and converges in no more FCG iterations than the V-cycle."""
    a = orc.gen_pde3d(14, 1, (1, 1, 1, 0, 0, 0, 0))
    b = orc.spmv(a, np.ones(a.nrows))
    its = {}
    for cyc in (orc.VCYCLE, orc.WCYCLE):
        par = oracle_params(orc, "FBGS", 1, coarse_sweeps=1, mcs=40)
        par.ml_cycle = cyc
        p = orc.Prec(par)
        p.build(a)
        assert p.nlev >= 3
        rng = np.random.default_rng(4)
        x, z = rng.uniform(-1, 1, a.nrows), rng.uniform(-1, 1, a.nrows)
        assert abs(p.apply(x) @ z - x @ p.apply(z)) <= 1e-12 * abs(p.apply(x) @ z)
        _, its[cyc], rr, _ = orc.krylov("FCG", a, p, b, eps=1e-10)
        assert rr <= 1e-10
    assert its[orc.WCYCLE] <= its[orc.VCYCLE]


@pytest.mark.parametrize("cycle", ["KCYCLE", "KCYCLESYM"])
def test_kcycle_converges(orc, cycle):
    """K-cycle with inner GCR / flexible CG (a nonlinear preconditioner, so
    FCG is the outer method): converges to the same solution as the V-cycle."""
    a = orc.gen_pde3d(16, 1, ISO)
    b = orc.spmv(a, np.ones(a.nrows))
    par = oracle_params(orc, "BJAC", 1, coarse_sweeps=4, mcs=40)
    par.ml_cycle = getattr(orc, cycle)
    p = orc.Prec(par)
    p.build(a)
    assert p.nlev >= 3
    x, it, rr, _ = orc.krylov("FCG", a, p, b, eps=1e-10)
    assert rr <= 1e-10 and np.abs(x - 1.0).max() <= 1e-7


def test_hierarchy_invariants(orc):
    a = orc.gen_pde3d(16, 1, ISO)
    p = orc.Prec(oracle_params(orc, "BJAC", mcs=150))
    p.build(a)
    assert p.nlev >= 2
    for l in range(1, p.nlev):
        il = p.level_vec(l, "ilaggr")
        info = p.level_info(l)
        prev = p.level_info(l - 1)["n"]
        assert il.shape == (prev,)
        assert il.min() == 0 and il.max() == info["n"] - 1
        assert len(np.unique(il)) == info["n"]  # every aggregate non-empty
        P = p.level_csr(l, "P").to_scipy()
        R = p.level_csr(l, "R").to_scipy()
        assert (abs(P.T - R) > 0).nnz == 0
        # Galerkin: A_c = R A P
        A = p.level_csr(l - 1, "A").to_scipy()
        Ac = p.level_csr(l, "A").to_scipy()
        assert abs(Ac - R @ A @ P).max() <= 1e-9 * abs(Ac).max()
        assert 0 < info["omega"] < 2


def test_linearity(orc):
    a = orc.gen_pde3d(10, 1, ISO)
    p = orc.Prec(oracle_params(orc, "BJAC", mcs=60))
    p.build(a)
    rng = np.random.default_rng(3)
    x, z = rng.uniform(-1, 1, a.nrows), rng.uniform(-1, 1, a.nrows)
    lhs = p.apply(2.5 * x - 0.75 * z)
    rhs = 2.5 * p.apply(x) - 0.75 * p.apply(z)
    assert np.linalg.norm(lhs - rhs) <= 1e-12 * np.linalg.norm(rhs)


def test_cg_fcg_agree_for_fixed_preconditioner(orc):
    a = orc.gen_pde3d(16, 1, ISO)
    p = orc.Prec(oracle_params(orc, "BJAC", mcs=150))
    p.build(a)
    b = orc.spmv(a, np.ones(a.nrows))
    _, it_cg, _, _ = orc.krylov("CG", a, p, b, eps=1e-10)
    x, it_fcg, rr, _ = orc.krylov("FCG", a, p, b, eps=1e-10)
    assert rr <= 1e-10 and abs(it_cg - it_fcg) <= 1
    assert np.abs(x - 1).max() < 1e-7
