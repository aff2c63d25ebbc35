"""GPU: the hacked-diagonal kernels (k_spmv_hdia, k_jacobi_hdia,
k_kry_spmv_hdia: per slice of 32 rows the ascending column offsets of its
rows and one value per (offset, row), no column index per entry).

An HDIA kernel sums a row in ascending column order from zero, with zero
values on the offsets the row lacks; the SELL kernel sums the same row in
its stored (ascending) order with zero padding at its end.  Adding an exact
zero product leaves a sum unchanged, so with launch shapes pinned (no
autotuning) a hierarchy whose square operators take the HDIA kernels
(MLDG_HDIA_FORCE, with 4 or 16 diagonals' loads per pass; the other
operators the SELL kernel) applies bit for bit
like the one whose operators all take the SELL kernel (MLDG_SELL_FORCE=1),
in every precision form, for trans 'N' and 'T'; the FP64 applies also meet
the oracle bar, and whole FCG solves (the fused Krylov SpMV on the HDIA copy
of A) are bitwise the SELL solves.  The HDIA hierarchy moves fewer bytes per
apply (no column indices on the stencil level)."""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hier(orc):
    a = orc.gen_pde3d(40, 1, ANISO)
    op = orc.Prec(oracle_params(orc, "JACOBI", 2, 0.8, coarse_sweeps=4, mcs=300))
    op.build(a)
    assert op.nlev >= 3
    return a, op


@pytest.mark.parametrize("passes", ["1", "16"])
@pytest.mark.parametrize("prec", [0, 1, 3])
def test_hdia_apply_bitwise_equal_to_sell(mld, orc, hier, monkeypatch, prec, passes):
    a, op = hier
    monkeypatch.setenv("MLDG_NO_AUTOTUNE", "1")
    monkeypatch.setenv("MLDG_NO_DENSE_INV", "1")
    monkeypatch.setenv("MLDG_SELL_FORCE", "1")
    h_sell = upload_oracle_hierarchy(mld, orc, op, precision=prec)
    # operators without an HDIA copy stay on the SELL kernel
    monkeypatch.setenv("MLDG_HDIA_FORCE", passes)
    h_hd = upload_oracle_hierarchy(mld, orc, op, precision=prec)
    rng = np.random.default_rng(3)
    for trans in ("N", "T"):
        x = rng.uniform(-1, 1, a.nrows)
        y_sell, y_hd = h_sell.apply(x, trans=trans), h_hd.apply(x, trans=trans)
        assert np.array_equal(y_sell, y_hd), (trans, np.abs(y_sell - y_hd).max())
        if prec == 0:
            y_ref = op.apply(x, trans)
            assert np.linalg.norm(y_hd - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    # the stencil level's operators really ran on the HDIA copy: fewer bytes
    # per apply (counted when the apply is first recorded)
    assert 0 < h_hd.apply_impl_bytes() < h_sell.apply_impl_bytes()
    h_sell.close()
    h_hd.close()


@pytest.mark.parametrize("smoother,coef", [("BJAC", ISO), ("FBGS", ANISO)])
def test_hdia_other_smoothers(mld, orc, monkeypatch, smoother, coef):
    # residual (A, A^T) on the HDIA copy under the triangular smoothers
    a = orc.gen_pde3d(28, 1, coef)
    op = orc.Prec(oracle_params(orc, smoother, 1, 1.0, coarse_sweeps=4, mcs=300))
    op.build(a)
    monkeypatch.setenv("MLDG_HDIA_FORCE", "1")
    h = upload_oracle_hierarchy(mld, orc, op)
    x = np.random.default_rng(4).uniform(-1, 1, a.nrows)
    for trans in (("N",) if smoother == "FBGS" else ("N", "T")):
        y_ref = op.apply(x, trans)
        assert np.linalg.norm(h.apply(x, trans=trans) - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    h.close()


def test_hdia_fcg_bitwise_equal_to_sell(mld, orc, hier, monkeypatch):
    a, op = hier
    b = np.random.default_rng(0).uniform(-1.0, 1.0, a.nrows)
    monkeypatch.setenv("MLDG_NO_AUTOTUNE", "1")
    monkeypatch.setenv("MLDG_NO_DENSE_INV", "1")
    monkeypatch.setenv("MLDG_SELL_FORCE", "1")
    h_sell = upload_oracle_hierarchy(mld, orc, op)
    x_s, it_s, rr_s = h_sell.krylov("FCG", b.copy(), eps=1e-10)
    # operators without an HDIA copy stay on the SELL kernel
    monkeypatch.setenv("MLDG_HDIA_FORCE", "1")
    h_hd = upload_oracle_hierarchy(mld, orc, op)
    x_h, it_h, rr_h = h_hd.krylov("FCG", b.copy(), eps=1e-10)
    assert it_h == it_s and rr_h == rr_s
    assert np.array_equal(x_h, x_s)
    x_ref, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    assert rr_h <= 1e-10 and abs(it_h - it_ref) <= 1
    assert np.linalg.norm(x_h - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    h_sell.close()
    h_hd.close()


def test_hdia_ragged_and_unsorted(mld, orc, monkeypatch):
    """Rows beyond a multiple of 32 (a partial last slice) and boundary rows
    with missing diagonals; then the same hierarchy uploaded with the entries
    of some level-0 rows of A and ND stored in reverse order (no HDIA copy is
    built for an unsorted matrix: the apply still matches the oracle through
    the other kernels)."""
    a = orc.gen_pde3d(13, 1, ISO)  # 2197 rows: the last slice holds 21
    op = orc.Prec(oracle_params(orc, "JACOBI", 2, 1.0, coarse_sweeps=4, mcs=100))
    op.build(a)
    monkeypatch.setenv("MLDG_HDIA_FORCE", "1")
    x = np.random.default_rng(5).uniform(-1, 1, a.nrows)
    for mangle in (False, True):
        h = mld.Hierarchy()
        for l in range(op.nlev):
            info = op.level_info(l)

            def conv(m, rev=False):
                if m is None:
                    return None
                irp, ja, val = np.array(m.irp), np.array(m.ja), np.array(m.val)
                if rev:
                    for i in range(0, len(irp) - 1, 97):
                        k0, k1 = irp[i], irp[i + 1]
                        ja[k0:k1] = ja[k0:k1][::-1].copy()
                        val[k0:k1] = val[k0:k1][::-1].copy()
                return mld.CSR(irp, ja, val, ncols=m.ncols)
            rev = mangle and l == 0
            h.upload_level(l, conv(op.level_csr(l, "A"), rev),
                           P=conv(op.level_csr(l, "P")) if l else None,
                           R=conv(op.level_csr(l, "R")) if l else None,
                           ND=conv(op.level_csr(l, "ND"), rev) if info["nnzND"] else None,
                           L=conv(op.level_csr(l, "L")) if info["smoother"] == orc.BJAC else None,
                           U=conv(op.level_csr(l, "U")) if info["smoother"] == orc.BJAC else None,
                           d=op.level_vec(l, "d") if info["smoother"] == orc.BJAC else op.level_vec(l, "dinv"),
                           smoother=info["smoother"], sweeps_pre=info["sweeps_pre"],
                           sweeps_post=info["sweeps_pre"], damping=info["damp"])
        h.finalize(op.nlev, mld.PREC_FP64)
        for trans in ("N", "T"):
            y_ref = op.apply(x, trans)
            assert np.linalg.norm(h.apply(x, trans=trans) - y_ref) <= 1e-12 * np.linalg.norm(y_ref), (mangle, trans)
        h.close()


def test_tune_file_round_trip(mld, orc, hier, monkeypatch, tmp_path):
    """MLDG_TUNE_FILE: the first finalize times every operator and appends its
    choice; a second finalize reads the choices instead of timing (adds no
    line) and launches the same kernels (the same bits)."""
    a, op = hier
    fn = tmp_path / "tune.txt"
    monkeypatch.setenv("MLDG_TUNE_FILE", str(fn))
    h1 = upload_oracle_hierarchy(mld, orc, op, precision=3)
    lines = fn.read_text().splitlines()
    assert any(s.startswith("spmv 4 1 0 0 ") for s in lines)  # level-0 A of the FP16 operator form
    h2 = upload_oracle_hierarchy(mld, orc, op, precision=3)
    assert fn.read_text().splitlines() == lines
    x = np.random.default_rng(7).uniform(-1, 1, a.nrows)
    assert np.array_equal(h1.apply(x), h2.apply(x))
    h1.close()
    h2.close()
