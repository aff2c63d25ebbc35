"""GPU parity of the partitioned triangular solve (k_trsv_blk) and of the
SELL-32 SpMV / Jacobi / Krylov kernels, forced on every level where they
exist (normally the autotuner picks them per operator by timing).

The oracle's hierarchy is uploaded unchanged; one apply (trans 'N' and 'T')
must agree with the oracle's apply to 1e-12 relative in FP64 (2e-5 in FP32),
with several block counts, including blocks small enough that most
dependencies cross blocks, and two applies of one plan must give the same
bits.  The plans themselves are checked on the CPU by the host emulation
(tests/test_blk_plan.py)."""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("idim,coef", [(24, ISO), (36, ANISO), (48, ISO)])
@pytest.mark.parametrize("P", ["1", "16", "148"])
def test_blk_apply_matches_oracle(mld, orc, monkeypatch, idim, coef, P):
    monkeypatch.setenv("MLDG_BLK_FORCE", "1")
    monkeypatch.setenv("MLDG_BLK_MIN", "0")
    monkeypatch.setenv("MLDG_BLK_P", P)
    monkeypatch.setenv("MLDG_NO_DENSE_INV", "1")
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=200))
    op.build(a)
    rng = np.random.default_rng(idim)
    for prec, tol in ((0, 1e-12), (1, 2e-5)):
        h = upload_oracle_hierarchy(mld, orc, op, precision=prec)
        for trans in ("N", "T"):
            x = rng.uniform(-1, 1, a.nrows)
            y_ref = op.apply(x, trans)
            y = h.apply(x, trans=trans)
            assert _rel(y, y_ref) <= tol, (prec, trans, _rel(y, y_ref))
            assert np.array_equal(h.apply(x, trans=trans), y)
        h.close()


def test_blk_krylov_iterations(mld, orc, monkeypatch):
    monkeypatch.setenv("MLDG_BLK_FORCE", "1")
    monkeypatch.setenv("MLDG_BLK_MIN", "0")
    a = orc.gen_pde3d(40, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=2000))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    b = orc.spmv(a, np.ones(a.nrows))
    _, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert abs(it - it_ref) <= 1 and rr <= 1e-10


@pytest.mark.parametrize("smoother,sweeps,damp", [("JACOBI", 2, 0.8), ("BJAC", 1, 1.0)])
@pytest.mark.parametrize("coef", [ISO, ANISO])
@pytest.mark.parametrize("form", ["1", "2", "3"])
def test_sell_kernels_match_oracle(mld, orc, monkeypatch, smoother, sweeps, damp, coef, form):
    """SELL forms: 1 and 2 slices per warp iteration, and the software-pipelined SpMV."""
    monkeypatch.setenv("MLDG_SELL_FORCE", form)
    a = orc.gen_pde3d(30, 1, coef)
    op = orc.Prec(oracle_params(orc, smoother, sweeps, damp, mcs=300))
    op.build(a)
    rng = np.random.default_rng(3)
    b = rng.uniform(-1, 1, a.nrows)
    x_ref, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    for prec, tol in ((0, 1e-12), (1, 2e-5)):
        h = upload_oracle_hierarchy(mld, orc, op, precision=prec)
        for trans in ("N", "T"):
            x = rng.uniform(-1, 1, a.nrows)
            y_ref = op.apply(x, trans)
            assert _rel(h.apply(x, trans=trans), y_ref) <= tol
        x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
        assert rr <= 1e-10 and it <= it_ref + (1 if prec == 0 else 2)
        h.close()
