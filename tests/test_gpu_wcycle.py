"""W-cycle (ML_CYCLE='WCYCLE'): the coarse correction is repeated once from
the updated residual before post-smoothing (mld_dmlprec_aply.f90:716-745).
GPU parity against the oracle for every smoother, single and multi-column,
and through the host mirror's set('ML_CYCLE', 'WCYCLE')."""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("idim,coef,smoother,sweeps", [(16, ISO, "BJAC", 1), (24, ANISO, "JACOBI", 2),
                                                       (20, ISO, "FBGS", 1), (40, ISO, "BJAC", 1)])
def test_wcycle_matches_oracle(mld, orc, idim, coef, smoother, sweeps):
    a = orc.gen_pde3d(idim, 1, coef)
    par = oracle_params(orc, smoother, sweeps, 0.8 if smoother == "JACOBI" else 1.0, mcs=100)
    par.ml_cycle = orc.WCYCLE
    op = orc.Prec(par)
    op.build(a)
    assert op.nlev >= 3
    h = upload_oracle_hierarchy(mld, orc, op)
    h.set_cycle(mld.CYCLE_W)
    rng = np.random.default_rng(idim)
    x = rng.uniform(-1, 1, a.nrows)
    assert _rel(h.apply(x), op.apply(x)) <= 1e-12
    if smoother != "FBGS":
        assert _rel(h.apply(x, trans="T"), op.apply(x, "T")) <= 1e-12
    X = rng.uniform(-1, 1, (4, a.nrows))
    Y = h.apply_block(X)
    assert max(_rel(Y[c], op.apply(X[c])) for c in range(4)) <= 1e-12
    # back to the V-cycle on the same handle
    h.set_cycle(mld.CYCLE_V)
    par.ml_cycle = orc.VCYCLE
    opv = orc.Prec(par)
    opv.build(a)
    assert _rel(h.apply(x), opv.apply(x)) <= 1e-12


def test_wcycle_through_host_mirror(mld, orc):
    am = mld.gen_pde3d(20, 1, ISO)
    p = mld.MldPrec()
    p.init("ML")
    p.set("SMOOTHER_TYPE", "BJAC")
    p.set("ML_CYCLE", "WCYCLE")
    p.set("COARSE_SOLVE", "BJAC")
    p.set("COARSE_SWEEPS", 4)
    p.set("MIN_COARSE_SIZE", 100)
    p.build(am)
    par = oracle_params(orc, "BJAC", mcs=100)
    par.ml_cycle = orc.WCYCLE
    op = orc.Prec(par)
    op.build(orc.gen_pde3d(20, 1, ISO))
    x = np.random.default_rng(2).uniform(-1, 1, am.nrows)
    assert _rel(p.apply(x), op.apply(x)) <= 1e-12
    b = am.matvec(np.ones(am.nrows))
    _, it, rr = mld.krylov("FCG", am, p, b, eps=1e-10, use_prec_matrix=True)
    assert rr <= 1e-10


@pytest.mark.parametrize("smoother,sweeps", [("BJAC", 1), ("JACOBI", 2), ("FBGS", 2)])
def test_additive_cycle_matches_oracle(mld, orc, smoother, sweeps):
    """ML_CYCLE='ADD' (mld_dmlprec_aply.f90:464-588): single and multi-column."""
    a = orc.gen_pde3d(20, 1, ISO)
    par = oracle_params(orc, smoother, sweeps, 0.8 if smoother == "JACOBI" else 1.0, mcs=60)
    par.ml_cycle = orc.ADD
    op = orc.Prec(par)
    op.build(a)
    assert op.nlev >= 3
    h = upload_oracle_hierarchy(mld, orc, op)
    h.set_cycle(mld.CYCLE_ADD)
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, a.nrows)
    assert _rel(h.apply(x), op.apply(x)) <= 1e-12
    X = rng.uniform(-1, 1, (4, a.nrows))
    Y = h.apply_block(X)
    assert max(_rel(Y[c], op.apply(X[c])) for c in range(4)) <= 1e-12
