"""GPU parity of the FBGS smoother, the reference's default for init('ML').

Pre-smoothing runs forward Gauss-Seidel sweeps (jac smoother + GS solver),
post-smoothing backward sweeps (jac smoother + BWGS solver); the GPU solves
(D+L)^{-1} and (D+U)^{-1} with the sync-free triangular kernels on rows
scaled by 1/a_ii.  Bars as for the other smoothers: one FP64 apply within
1e-12 of the oracle, Krylov iteration counts within one.
"""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("idim,coef", [(8, ISO), (14, ANISO), (28, ISO), (40, ISO)])
@pytest.mark.parametrize("sweeps", [1, 2])
def test_fbgs_apply_matches_oracle(mld, orc, idim, coef, sweeps):
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, "FBGS", sweeps, mcs=200))
    op.build(a)
    assert op.level_info(0)["smoother"] == orc.FBGS
    h = upload_oracle_hierarchy(mld, orc, op)
    rng = np.random.default_rng(idim + sweeps)
    for _ in range(3):  # repeated applies: the exchange buffers return to their start state
        x = rng.uniform(-1, 1, a.nrows)
        y = h.apply(x)
        assert _rel(y, op.apply(x)) <= TOL_FP64
    X = rng.uniform(-1, 1, (5, a.nrows))
    Y = h.apply_block(X)
    for c in range(5):
        assert _rel(Y[c], op.apply(X[c])) <= TOL_FP64


def test_fbgs_rejects_transpose(mld, orc):
    a = orc.gen_pde3d(10, 1, ISO)
    op = orc.Prec(oracle_params(orc, "FBGS", mcs=100))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    with pytest.raises(mld.MldError) as e:
        h.apply(np.ones(a.nrows), trans="T")
    assert e.value.code == 40
    with pytest.raises(mld.MldError) as e:
        h.adjoint(np.ones(a.nrows))
    assert e.value.code == 40


def test_fbgs_krylov_matches_oracle(mld, orc):
    a = orc.gen_pde3d(24, 1, ISO)
    op = orc.Prec(oracle_params(orc, "FBGS", mcs=300))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    b = orc.spmv(a, np.ones(a.nrows))
    _, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert abs(it - it_ref) <= 1 and rr <= 1e-10
    assert np.abs(x - 1.0).max() <= 1e-8


def test_ml_default_is_fbgs_and_solves(mld, orc):
    """prec%init('ML') with no further settings: FBGS levels, ILU coarse
    solve; the product's host build + GPU apply against the oracle."""
    am = mld.gen_pde3d(20, 1, ISO)
    p = mld.MldPrec()
    p.init("ML")
    p.set("MIN_COARSE_SIZE", 200)
    p.build(am)
    assert "FBGS" in p.descr()
    ao = orc.gen_pde3d(20, 1, ISO)
    par = oracle_params(orc, "FBGS", mcs=200, coarse_sweeps=1)
    op = orc.Prec(par)
    op.build(ao)
    x = np.random.default_rng(8).uniform(-1, 1, ao.nrows)
    assert _rel(p.apply(x), op.apply(x)) <= TOL_FP64
    b = am.matvec(np.ones(am.nrows))
    xs, it, rr = mld.krylov("FCG", am, p, b, eps=1e-10, use_prec_matrix=True)
    assert rr <= 1e-10 and np.abs(xs - 1.0).max() <= 1e-8


def test_one_level_fbgs(mld, orc):
    a = orc.gen_pde3d(12, 1, ANISO)
    for sweeps in (1, 3):
        op = orc.Prec(orc.default_params(smoother=orc.FBGS, max_levs=1, sweeps_pre=sweeps,
                                         sweeps_post=sweeps))
        op.build(a)
        h = upload_oracle_hierarchy(mld, orc, op)
        x = np.random.default_rng(sweeps).uniform(-1, 1, a.nrows)
        assert _rel(h.apply(x), op.apply(x)) <= TOL_FP64
        X = np.stack([x, 2 * x + 1])
        Y = h.apply_block(X)
        assert _rel(Y[1], op.apply(X[1])) <= TOL_FP64
    am = mld.gen_pde3d(12, 1, ANISO)
    p = mld.MldPrec()
    p.init("FBGS")
    p.build(am)
    op = orc.Prec(orc.default_params(smoother=orc.FBGS, max_levs=1))
    op.build(a)
    assert _rel(p.apply(x), op.apply(x)) <= TOL_FP64


def test_fbgs_fp32(mld, orc):
    a = orc.gen_pde3d(20, 1, ISO)
    op = orc.Prec(oracle_params(orc, "FBGS", mcs=200))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op, precision=1)
    x = np.random.default_rng(1).uniform(-1, 1, a.nrows)
    assert _rel(h.apply(x), op.apply(x)) <= 2e-5
