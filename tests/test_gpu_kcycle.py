"""K-cycle (ML_CYCLE='KCYCLE' with inner GCR, 'KCYCLESYM' with inner flexible
CG; mld_dmlprec_aply.f90:811-1184): GPU parity against the oracle's
restatement, for every smoother, through the C ABI and the host mirror."""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _oracle(orc, a, smoother, cycle, sweeps=1):
    par = oracle_params(orc, smoother, sweeps, 0.8 if smoother == "JACOBI" else 1.0, mcs=60)
    par.ml_cycle = cycle
    op = orc.Prec(par)
    op.build(a)
    return op


@pytest.mark.parametrize("cyc", ["K", "KSYM"])
@pytest.mark.parametrize("idim,coef,smoother,sweeps", [(20, ISO, "BJAC", 1), (24, ANISO, "JACOBI", 2),
                                                       (18, ISO, "FBGS", 1)])
def test_kcycle_matches_oracle(mld, orc, cyc, idim, coef, smoother, sweeps):
    a = orc.gen_pde3d(idim, 1, coef)
    op = _oracle(orc, a, smoother, orc.KCYCLE if cyc == "K" else orc.KCYCLESYM, sweeps)
    assert op.nlev >= 3  # an inner Krylov step runs on level 1
    h = upload_oracle_hierarchy(mld, orc, op)
    h.set_cycle(mld.CYCLE_K if cyc == "K" else mld.CYCLE_KSYM)
    rng = np.random.default_rng(idim)
    for trans in (("N", "T") if smoother != "FBGS" else ("N",)):
        for _ in range(2):
            x = rng.uniform(-1, 1, a.nrows)
            assert _rel(h.apply(x, trans=trans), op.apply(x, trans)) <= 1e-12, trans
    # a block of columns is applied column by column
    X = rng.uniform(-1, 1, (3, a.nrows))
    Y = h.apply_block(X)
    assert max(_rel(Y[c], op.apply(X[c])) for c in range(3)) <= 1e-12
    b = orc.spmv(a, np.ones(a.nrows))
    _, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert abs(it - it_ref) <= 1 and rr <= 1e-10


def test_kcycle_host_mirror_and_limits(mld, orc):
    am = mld.gen_pde3d(20, 1, ISO)
    p = mld.MldPrec()
    p.init("ML")
    p.set("SMOOTHER_TYPE", "BJAC")
    p.set("ML_CYCLE", "KCYCLESYM")
    p.set("COARSE_SOLVE", "BJAC")
    p.set("COARSE_SWEEPS", 4)
    p.set("MIN_COARSE_SIZE", 60)
    p.build(am)
    op = _oracle(orc, orc.gen_pde3d(20, 1, ISO), "BJAC", orc.KCYCLESYM)
    x = np.random.default_rng(3).uniform(-1, 1, am.nrows)
    assert _rel(p.apply(x), op.apply(x)) <= 1e-12
    with pytest.raises(mld.MldError) as e:
        p.krylov_multi("FCG", np.ones((2, am.nrows)))
    assert e.value.code == 30
