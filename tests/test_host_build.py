"""CPU: the product's host-side hierarchy build (C++, libmldgpu.so) against
the oracle's restatement of the reference build.  Integer structure
(aggregates, sparsity patterns, level sizes) must be identical; values too,
since both follow the reference's operation order with the same rounding."""
import numpy as np
import pytest

from conftest import ANISO, ISO

CASES = [(6, ISO, "BJAC", 50), (10, ISO, "BJAC", 100), (16, ANISO, "BJAC", 200),
         (20, ISO, "JACOBI", 300), (24, ANISO, "JACOBI", -1)]


def _product(mld, a, smoother, mcs, sweeps=1):
    p = mld.MldPrec()
    p.init("ML")
    p.set("SMOOTHER_TYPE", smoother)
    p.set("SMOOTHER_SWEEPS", sweeps)
    p.set("COARSE_SOLVE", "BJAC")
    p.set("COARSE_SUBSOLVE", "ILU")
    p.set("COARSE_SWEEPS", 4)
    p.set("MIN_COARSE_SIZE", mcs)
    p.hierarchy_build(a)
    return p


@pytest.mark.parametrize("idim,coef,smoother,mcs", CASES)
def test_hierarchy_identical(mld, orc, idim, coef, smoother, mcs):
    ao = orc.gen_pde3d(idim, 1, coef)
    ap = mld.gen_pde3d(idim, 1, coef)
    assert np.array_equal(ao.irp, ap.irp) and np.array_equal(ao.ja, ap.ja)
    assert np.array_equal(ao.val, ap.val)
    sm = orc.BJAC if smoother == "BJAC" else orc.JACOBI
    op = orc.Prec(orc.default_params(smoother=sm, coarse_solver=orc.BJAC, coarse_sweeps=4,
                                     min_coarse_size=mcs))
    op.build(ao)
    pp = _product(mld, ap, smoother, mcs)
    assert pp.nlev == op.nlev
    for l in range(op.nlev):
        io, ip = op.level_info(l), pp.level_info(l)
        for k in ("n", "nnzA", "nnzP", "nnzR", "naggr"):
            assert io[k] == ip[k], (l, k)
        if l:
            assert io["omega"] == ip["omega"]
            assert np.array_equal(op.level_vec(l, "ilaggr"), pp.level_vec(l, "ilaggr"))
        for w in (["A", "P", "R"] if l else ["A"]):
            mo, mp = op.level_csr(l, w), pp.level_csr(l, w)
            assert np.array_equal(mo.irp, mp.irp), (l, w)
            assert np.array_equal(mo.ja, mp.ja), (l, w)
            assert np.array_equal(mo.val, mp.val), (l, w)


@pytest.mark.parametrize("idim,coef,smoother,mcs", [(14, ISO, "BJAC", 150), (16, ANISO, "BJAC", 200),
                                                    (14, ISO, "JACOBI", 150), (12, ISO, "FBGS", 100)])
def test_smoother_data_identical(mld, orc, idim, coef, smoother, mcs):
    """The smoother/solver data of every level -- ILU(0) factors L, U and
    pivots (mld_dilu0_fact.f90), the Jacobi off-diagonal part and inverse
    diagonal, the GS split -- bit for bit between the product's host build
    and the oracle."""
    ao = orc.gen_pde3d(idim, 1, coef)
    sm = {"BJAC": orc.BJAC, "JACOBI": orc.JACOBI, "FBGS": orc.FBGS}[smoother]
    op = orc.Prec(orc.default_params(smoother=sm, coarse_solver=orc.BJAC, coarse_sweeps=4,
                                     min_coarse_size=mcs))
    op.build(ao)
    pp = _product(mld, mld.gen_pde3d(idim, 1, coef), smoother, mcs)
    pp.smoothers_build_host()
    assert pp.nlev == op.nlev
    compared = 0
    for l in range(op.nlev):
        io = op.level_info(l)
        names = {orc.BJAC: ["L", "U"], orc.FBGS: ["L", "U"], orc.JACOBI: ["ND"]}[io["smoother"]]
        for w in names:
            mo, mp = op.level_csr(l, w), pp.level_csr(l, w)
            assert mo is not None and mp is not None, (l, w)
            assert np.array_equal(mo.irp, mp.irp), (l, w)
            assert np.array_equal(mo.ja, mp.ja), (l, w)
            assert np.array_equal(mo.val, mp.val), (l, w)
            compared += mo.nnz
        vo = op.level_vec(l, "dinv" if io["smoother"] == orc.JACOBI else "d")
        assert np.array_equal(vo, pp.level_vec(l, "d")), l
    assert compared > 0
