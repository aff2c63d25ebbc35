"""GPU: failure detection of the dependency-bound triangular solves, without
a GPU fault.

Every sentinel wait of the sync-free and ELL solves is bounded.  The test
hook mldg_test_set_spin_limit lowers the bound to zero polls, so a wait that
finds a dependency not yet written gives up at once: the kernel records
MLDG_ERR_TIMEOUT (4020), every other waiter leaves, and the kernel ends.  The
host reads the error word after the call and returns the code, as the
reference returns its info code (mld_dprecaply.f90:355-360 pushes its errors
the same way).  The handle must stay usable: with the bound restored the
next apply and the next solve on the same handle agree with the oracle, which
requires the library to put the exchange buffers and ticket counters back
into their start state after the failed call.

The levels are kept below the size that selects the cluster solves (whose
mbarrier waits keep their own bound), so only plain global-memory polls give
up here; nothing is left in flight when a kernel ends.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu


def _set_limit(mld, polls):
    f = mld.lib().mldg_test_set_spin_limit
    f.argtypes = [C.c_int, C.c_int]
    assert f(0, polls) == 0


@pytest.mark.parametrize("ell", ["1", "0"])
def test_wait_timeout_is_reported_and_handle_recovers(mld, orc, monkeypatch, ell):
    # ell "1": single-vector solves on the ELL kernel; "0": the sync-free kernel
    monkeypatch.setenv("MLDG_ELL1", ell)
    monkeypatch.setenv("MLDG_NO_DENSE_INV", "1")
    monkeypatch.setenv("MLDG_NO_WIN", "1")
    monkeypatch.setenv("MLDG_NO_REP", "1")
    a = orc.gen_pde3d(36, 1, ISO)       # 46,656 rows, 106 dependency levels on level 0
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=300))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    x = np.random.default_rng(7).uniform(-1, 1, a.nrows)
    y_ref = op.apply(x)
    assert np.linalg.norm(h.apply(x) - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    _set_limit(mld, 0)
    try:
        codes = []
        for _ in range(3):
            try:
                h.apply(x)
                codes.append(0)
            except mld.MldError as e:
                codes.append(e.code)
    finally:
        _set_limit(mld, -1)
    assert mld.ERR_TIMEOUT in codes, codes
    assert set(codes) <= {0, mld.ERR_TIMEOUT}, codes
    assert b"limit" in mld.lib().mldg_last_error(h._h)
    # the same handle, bound restored: applies and a solve are right again
    for trans in ("N", "T"):
        y_ref = op.apply(x, trans)
        y = h.apply(x, trans=trans)
        assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref), trans
    b = orc.spmv(a, np.ones(a.nrows))
    _, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    xs, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert rr <= 1e-10 and abs(it - it_ref) <= 1


def test_timeout_inside_a_graph_solve(mld, orc):
    """A solve that is one graph launch: the failed waits leave the device
    loop running to itmax or a NaN residual, the call returns 4020, and the
    handle solves correctly afterwards."""
    a = orc.gen_pde3d(30, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=300))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    b = orc.spmv(a, np.ones(a.nrows))
    _, it0, _ = h.krylov("FCG", b.copy(), eps=1e-10)  # captures the solve graph
    _set_limit(mld, 0)
    try:
        with pytest.raises(mld.MldError) as e:
            for _ in range(3):
                h.krylov("FCG", b.copy(), eps=1e-10, itmax=20)
    finally:
        _set_limit(mld, -1)
    assert e.value.code == mld.ERR_TIMEOUT
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert it == it0 and rr <= 1e-10 and np.max(np.abs(x - 1)) < 1e-6
