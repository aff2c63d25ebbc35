"""GPU parity of one preconditioner apply against the oracle.

The oracle's hierarchy (the reference's build algorithm, restated in C) is
uploaded unchanged through the C ABI; one V-cycle apply on the GPU must agree
with the oracle's apply on the same vector to 1e-12 relative (FP64 form).
"""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12   # north-star tolerance for one FP64 apply
TOL_FP32 = 2e-5    # FP32 V-cycle vs FP64 oracle apply


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("idim,coef", [(8, ISO), (12, ISO), (16, ANISO), (28, ISO)])
@pytest.mark.parametrize("smoother,sweeps,damp", [("BJAC", 1, 1.0), ("JACOBI", 2, 0.8),
                                                  ("JACOBI", 1, 1.0), ("JACOBI", 3, 1.0),
                                                  ("JACOBI", 4, 0.9)])
def test_apply_matches_oracle(mld, orc, idim, coef, smoother, sweeps, damp):
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, smoother, sweeps, damp, mcs=200))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    rng = np.random.default_rng(idim)
    for trans in ("N", "T"):
        for _ in range(2):
            x = rng.uniform(-1, 1, a.nrows)
            y_ref = op.apply(x, trans)
            y = h.apply(x, trans=trans)
            assert _rel(y, y_ref) <= TOL_FP64, (trans, _rel(y, y_ref))


def test_apply_without_graphs_identical(mld, orc):
    a = orc.gen_pde3d(14, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=300))
    op.build(a)
    # launch shapes pinned (no autotuning): graph replay and direct launches
    # run the same kernels with the same schedules -> identical bits
    h1 = upload_oracle_hierarchy(mld, orc, op, use_graphs=True, autotune=False)
    h2 = upload_oracle_hierarchy(mld, orc, op, use_graphs=False, autotune=False)
    x = np.random.default_rng(3).uniform(-1, 1, a.nrows)
    y1, y2 = h1.apply(x), h2.apply(x)
    assert np.array_equal(y1, y2)
    assert np.array_equal(h1.apply(x), y1)
    # an autotuned handle may pick other lanes-per-row (summation order), so
    # it agrees to rounding, and is bitwise repeatable on its own
    h3 = upload_oracle_hierarchy(mld, orc, op)
    y3 = h3.apply(x)
    assert np.linalg.norm(y3 - y1) <= 1e-14 * np.linalg.norm(y1)
    assert np.array_equal(h3.apply(x), y3)


def test_fp32_apply(mld, orc):
    a = orc.gen_pde3d(16, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=300))
    op.build(a)
    x = np.random.default_rng(5).uniform(-1, 1, a.nrows)
    y_ref = op.apply(x)
    for prec in (mld.PREC_FP32, mld.PREC_FP32_P16, mld.PREC_FP32_H16):
        h = upload_oracle_hierarchy(mld, orc, op, precision=prec)
        y = h.apply(x)
        tol = {mld.PREC_FP32: TOL_FP32, mld.PREC_FP32_P16: 5e-3}.get(prec, 2e-2)
        assert _rel(y, y_ref) <= tol, (prec, _rel(y, y_ref))


def test_host_mirror_apply_matches_oracle(mld, orc):
    a = orc.gen_pde3d(20, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=500))
    op.build(a)
    p = mld.MldPrec()
    p.init("ML")
    p.set("SMOOTHER_TYPE", "BJAC")
    p.set("SUB_SOLVE", "ILU")
    p.set("SMOOTHER_SWEEPS", 1)
    p.set("COARSE_SOLVE", "BJAC")
    p.set("COARSE_SUBSOLVE", "ILU")
    p.set("COARSE_SWEEPS", 4)
    p.set("MIN_COARSE_SIZE", 500)
    p.build(mld.CSR(a.irp, a.ja, a.val))
    assert p.nlev == op.nlev
    x = np.random.default_rng(7).uniform(-1, 1, a.nrows)
    for trans in ("N", "T"):
        assert _rel(p.apply(x, trans=trans), op.apply(x, trans)) <= TOL_FP64


def test_errors(mld, orc):
    h = mld.Hierarchy()
    x = np.zeros(10)
    with pytest.raises(mld.MldError) as e:
        h.apply(x)
    assert e.value.code == mld.ERR_NOT_BUILT
    a = orc.gen_pde3d(6, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=50))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    with pytest.raises(mld.MldError) as e:
        h.apply(np.zeros(a.nrows), trans="X")
    assert e.value.code == 40


def test_apply_large_coarse_level(mld, orc):
    """idim=60: level 1 has ~27k rows and ~15 entries per triangular row, so
    its solves run the multi-CTA sync-free kernel with several lanes per row
    (warp blocks aligned to dependency levels)."""
    a = orc.gen_pde3d(60, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=2000))
    op.build(a)
    assert op.level_info(1)["n"] > 16384
    h = upload_oracle_hierarchy(mld, orc, op)
    rng = np.random.default_rng(60)
    for trans in ("N", "T"):
        x = rng.uniform(-1, 1, a.nrows)
        assert _rel(h.apply(x, trans=trans), op.apply(x, trans)) <= TOL_FP64


@pytest.mark.parametrize("idim,coef,smoother", [(20, ISO, "BJAC"), (28, ANISO, "BJAC"), (20, ANISO, "FBGS")])
def test_dense_inverse_levels_match_oracle(mld, orc, monkeypatch, idim, coef, smoother):
    """Every level below the finest applied through explicit inverses (of its
    ILU(0), or of D+L and D+U for FBGS), computed on the GPU column block by
    column block."""
    monkeypatch.setenv("MLDG_DENSE_INV", "1")
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, smoother, mcs=60))
    op.build(a)
    assert op.nlev >= 3
    for precision, tol in ((0, TOL_FP64), (1, TOL_FP32)):
        h = upload_oracle_hierarchy(mld, orc, op, precision=precision)
        rng = np.random.default_rng(idim)
        for trans in (("N", "T") if smoother == "BJAC" else ("N",)):
            x = rng.uniform(-1, 1, a.nrows)
            assert _rel(h.apply(x, trans=trans), op.apply(x, trans)) <= tol
        X = rng.uniform(-1, 1, (3, a.nrows))
        Y = h.apply_block(X)
        assert max(_rel(Y[c], op.apply(X[c])) for c in range(3)) <= tol


@pytest.mark.parametrize("idim,smoother,max_levs", [(1, "BJAC", 20), (2, "BJAC", 20), (2, "JACOBI", 1),
                                                    (3, "FBGS", 20), (5, "BJAC", 1)])
def test_degenerate_sizes(mld, orc, idim, smoother, max_levs):
    """One-row and few-row systems, one-level and multilevel: same results as
    the oracle; a zero right-hand side gives zero; nrhs = 0 is a no-op."""
    a = orc.gen_pde3d(idim, 1, ISO)
    par = oracle_params(orc, smoother, mcs=1)
    par.max_levs = max_levs
    op = orc.Prec(par)
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    x = np.random.default_rng(idim).uniform(-1, 1, a.nrows)
    assert _rel(h.apply(x), op.apply(x)) <= TOL_FP64
    assert np.all(h.apply(np.zeros(a.nrows)) == 0.0)
    Y = np.full((0, a.nrows), 5.0)
    h.apply_block(np.zeros((0, a.nrows)), Y)
    X2 = np.stack([x, -x])
    Y2 = h.apply_block(X2)
    assert _rel(Y2[1], -op.apply(x)) <= TOL_FP64
