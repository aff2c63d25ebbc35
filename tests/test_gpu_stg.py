"""GPU: the staged SELL kernels (k_spmv_stg, k_jacobi_stg: one TMA bulk copy
of a packed tile of SELL-32 slices per stage of a per-warp shared-memory
ring, mldg_spmv_stg.cuh).

A staged kernel sums each row exactly like the SELL kernel (slots in stored
order from zero, padding included), so with launch shapes pinned (no
autotuning) a hierarchy whose operators take the staged kernels
(MLDG_STG_FORCE) must apply bit for bit like the one whose operators take
the SELL kernel (MLDG_SELL_FORCE=1) -- in every precision form, for trans 'N'
and 'T', with the two-stage ring the tiles are sized for and with the
deepest ring that fits.  The staged applies also meet the FP64 bar against
the oracle."""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu

CASES = [{}, {"MLDG_STG_S": "4"}]


@pytest.fixture(scope="module")
def hier(orc):
    a = orc.gen_pde3d(40, 1, ANISO)
    op = orc.Prec(oracle_params(orc, "JACOBI", 2, 0.8, coarse_sweeps=4, mcs=300))
    op.build(a)
    assert op.nlev >= 3
    return a, op


@pytest.mark.parametrize("env", CASES)
@pytest.mark.parametrize("prec", [0, 1, 3])
def test_staged_apply_bitwise_equal_to_sell(mld, orc, hier, monkeypatch, prec, env):
    a, op = hier
    monkeypatch.setenv("MLDG_NO_AUTOTUNE", "1")
    monkeypatch.setenv("MLDG_NO_DENSE_INV", "1")
    monkeypatch.setenv("MLDG_SELL_FORCE", "1")
    h_sell = upload_oracle_hierarchy(mld, orc, op, precision=prec)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    monkeypatch.setenv("MLDG_STG_FORCE", "1")
    h_stg = upload_oracle_hierarchy(mld, orc, op, precision=prec)
    rng = np.random.default_rng(3)
    for trans in ("N", "T"):
        x = rng.uniform(-1, 1, a.nrows)
        y_sell, y_stg = h_sell.apply(x, trans=trans), h_stg.apply(x, trans=trans)
        assert np.array_equal(y_sell, y_stg), (trans, np.abs(y_sell - y_stg).max())
        if prec == 0:
            y_ref = op.apply(x, trans)
            assert np.linalg.norm(y_stg - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    h_sell.close()
    h_stg.close()


@pytest.mark.parametrize("smoother,coef", [("BJAC", ISO), ("FBGS", ANISO)])
def test_staged_other_smoothers(mld, orc, monkeypatch, smoother, coef):
    # residual, restriction and prolongation staged under the triangular smoothers
    a = orc.gen_pde3d(28, 1, coef)
    op = orc.Prec(oracle_params(orc, smoother, 1, 1.0, coarse_sweeps=4, mcs=300))
    op.build(a)
    monkeypatch.setenv("MLDG_STG_FORCE", "1")
    h = upload_oracle_hierarchy(mld, orc, op)
    x = np.random.default_rng(4).uniform(-1, 1, a.nrows)
    y_ref = op.apply(x)
    assert np.linalg.norm(h.apply(x) - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    h.close()


def test_staged_fcg_iterations(mld, orc, hier, monkeypatch):
    a, op = hier
    monkeypatch.setenv("MLDG_STG_FORCE", "1")
    b = np.random.default_rng(0).uniform(-1.0, 1.0, a.nrows)
    x_ref, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    h = upload_oracle_hierarchy(mld, orc, op)
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert rr <= 1e-10 and abs(it - it_ref) <= 1
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    h.close()
