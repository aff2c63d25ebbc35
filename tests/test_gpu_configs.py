"""GPU parity at the benchmarked configurations themselves.

The oracle's hierarchy (the reference's build algorithm restated in C) is
uploaded unchanged through the C ABI at the exact settings of each
configuration, and one preconditioner apply (trans 'N' and 'T') and the
Krylov iteration counts are compared with the oracle's:

  C1  isotropic pdegen problem, idim=40, BJAC-ILU(0) 1+1 sweeps, coarsening to
      <= 2000 rows, coarsest 4 sweeps of BJAC-ILU(0); CG to 1e-9
  C2  isotropic, idim=160 (4,096,000 rows): BJAC-ILU(0) 1 sweep, and point
      Jacobi 2 sweeps with damping 0.8; FCG to 1e-10
  C3  anisotropic (0.01 u_zz), idim=160, b uniform[-1,1] (seed 0): the FP32,
      FP32+FP16-prolongator and FP16-operator V-cycles inside FP64 FCG to 1e-10

Bars: an FP64 apply within 1e-12 relative of the oracle's apply
(mld_dmlprec_aply.f90:590-809); iteration counts within +-1; the reduced
precision applies within 2e-5 (FP32), 5e-3 (FP16 prolongators) and 2e-2 (FP16
operator values) of the FP64 oracle apply; the reduced precision solves reach
1e-10 with at most 2 extra iterations, and their solutions agree with the
oracle's FP64 solution.
"""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FP32 = 2e-5
TOL_P16 = 5e-3
TOL_H16 = 2e-2


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _check_applies(h, op, n, seed, tol):
    rng = np.random.default_rng(seed)
    for trans in ("N", "T"):
        x = rng.uniform(-1, 1, n)
        y_ref = op.apply(x, trans)
        y = h.apply(x, trans=trans)
        assert _rel(y, y_ref) <= tol, (trans, _rel(y, y_ref))


@pytest.mark.parametrize("method,eps", [("CG", 1e-9), ("FCG", 1e-10)])
def test_c1_idim40(mld, orc, method, eps):
    a = orc.gen_pde3d(40, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", 1, 1.0, coarse_sweeps=4, mcs=2000))
    op.build(a)
    assert op.level_info(op.nlev - 1)["n"] <= 2000
    h = upload_oracle_hierarchy(mld, orc, op)
    _check_applies(h, op, a.nrows, 40, TOL_FP64)
    b = orc.spmv(a, np.ones(a.nrows))
    _, it_ref, _, _ = orc.krylov(method, a, op, b, eps=eps)
    x, it, rr = h.krylov(method, b.copy(), eps=eps)
    assert abs(it - it_ref) <= 1, (it, it_ref)
    assert rr <= eps and np.max(np.abs(x - 1)) < 1e-5


@pytest.fixture(scope="module")
def iso160(orc):
    return orc.gen_pde3d(160, 1, ISO)


@pytest.mark.parametrize("smoother,sweeps,damp", [("BJAC", 1, 1.0), ("JACOBI", 2, 0.8)])
def test_c2_idim160(mld, orc, iso160, smoother, sweeps, damp):
    a = iso160
    op = orc.Prec(oracle_params(orc, smoother, sweeps, damp, coarse_sweeps=4, mcs=2000))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    _check_applies(h, op, a.nrows, 160, TOL_FP64)
    b = orc.spmv(a, np.ones(a.nrows))
    _, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert abs(it - it_ref) <= 1, (it, it_ref)
    assert rr <= 1e-10 and np.max(np.abs(x - 1)) < 1e-6


def test_c3_idim160_reduced_precision(mld, orc):
    a = orc.gen_pde3d(160, 1, ANISO)
    op = orc.Prec(oracle_params(orc, "JACOBI", 2, 0.8, coarse_sweeps=4, mcs=2000))
    op.build(a)
    b = np.random.default_rng(0).uniform(-1.0, 1.0, a.nrows)
    x_ref, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    for prec, tol in ((mld.PREC_FP32, TOL_FP32), (mld.PREC_FP32_P16, TOL_P16), (mld.PREC_FP32_H16, TOL_H16)):
        h = upload_oracle_hierarchy(mld, orc, op, precision=prec)
        _check_applies(h, op, a.nrows, 3, tol)
        x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
        assert rr <= 1e-10
        assert it <= it_ref + 2, (prec, it, it_ref)
        assert _rel(x, x_ref) < 1e-8, (prec, _rel(x, x_ref))
        h.close()
