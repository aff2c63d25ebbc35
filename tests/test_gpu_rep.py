"""GPU parity of the replicated-window cluster solve (k_trsv_rep).

The ILU(0) solves of every eligible level are forced onto the kernel (the
autotuner picks it only where it is fastest, normally the large coarse
levels of big problems); one V-cycle apply must agree with the oracle's
apply, and a Krylov solve must take the oracle's iteration count.  A small
ring (MLDG_REP_R) sends the older dependencies through the far path; both
cluster sizes are covered, and the finest level of idim=56 has levels wider
than one step.
"""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FP32 = 2e-5


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _force(monkeypatch, ring=None, cluster=16):
    monkeypatch.setenv("MLDG_NO_WIN", "1")
    monkeypatch.setenv("MLDG_NO_DENSE_INV", "1")
    monkeypatch.setenv("MLDG_REP_MIN", "0")
    monkeypatch.setenv("MLDG_REP_FORCE", "1")
    monkeypatch.setenv("MLDG_REP_C", str(cluster))
    monkeypatch.setenv("MLDG_VERBOSE", "1")
    if ring:
        monkeypatch.setenv("MLDG_REP_R", ring)


@pytest.mark.parametrize("idim,coef,ring,cluster", [(40, ISO, None, 8), (48, ANISO, "4096", 8),
                                                    (60, ISO, "2048", 16), (56, ISO, None, 16)])
def test_rep_apply_matches_oracle(mld, orc, monkeypatch, capfd, idim, coef, ring, cluster):
    _force(monkeypatch, ring, cluster)
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=50))
    op.build(a)
    rng = np.random.default_rng(idim)
    for precision, tol in ((0, TOL_FP64), (1, TOL_FP32)):
        h = upload_oracle_hierarchy(mld, orc, op, precision=precision)
        assert "uses rep" in capfd.readouterr().err
        for trans in ("N", "T"):
            x = rng.uniform(-1, 1, a.nrows)
            y1 = h.apply(x, trans=trans)
            assert _rel(y1, op.apply(x, trans)) <= tol, (precision, trans)
            # a second launch over the same plans gives the same bits
            assert np.array_equal(h.apply(x, trans=trans), y1)
        h.close()


def test_rep_krylov_iterations_match(mld, orc, monkeypatch, capfd):
    _force(monkeypatch, "2048")
    a = orc.gen_pde3d(60, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=400))
    op.build(a)
    b = orc.spmv(a, np.ones(a.nrows))
    _, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    h = upload_oracle_hierarchy(mld, orc, op)
    assert "uses rep" in capfd.readouterr().err
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert abs(it - it_ref) <= 1, (it, it_ref)
    assert rr <= 1e-10
    assert np.linalg.norm(x - 1) / np.sqrt(a.nrows) < 1e-6


@pytest.mark.parametrize("idim,cluster", [(3, 16), (12, 8), (12, 16)])
def test_rep_few_steps(mld, orc, monkeypatch, capfd, idim, cluster):
    """Levels of 7 to 74 steps: fewer steps than the step groups, the stage
    lookahead or one 32-step descriptor chunk of the producer."""
    _force(monkeypatch, None, cluster)
    a = orc.gen_pde3d(idim, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=20))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    assert "uses rep" in capfd.readouterr().err
    x = np.random.default_rng(idim).uniform(-1, 1, a.nrows)
    for trans in ("N", "T"):
        assert _rel(h.apply(x, trans=trans), op.apply(x, trans)) <= TOL_FP64
