"""MatrixMarket hierarchy I/O in the layout of the reference's prec%dump
(mld_d_prec_type.f90:698-729, mld_d_base_onelev_dump.f90:112-129 and the
smoother/solver dump routines): a hierarchy written by one build and read by
another applies identically, and files written independently from the
oracle's hierarchy (coordinate/array MatrixMarket, 1-based, as PSBLAS prints
them) load into the GPU apply with oracle parity."""
import os

import numpy as np
import pytest

from conftest import ISO, ANISO, oracle_params

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _set(p, smoother):
    p.init("ML")
    p.set("SMOOTHER_TYPE", smoother)
    if smoother == "JACOBI":
        p.set("SMOOTHER_SWEEPS", 2)
    p.set("COARSE_SOLVE", "BJAC")
    p.set("COARSE_SWEEPS", 4)
    p.set("MIN_COARSE_SIZE", 150)


@pytest.mark.parametrize("smoother", ["BJAC", "JACOBI", "FBGS"])
def test_dump_load_round_trip(mld, tmp_path, smoother):
    a = mld.gen_pde3d(18, 1, ANISO)
    p = mld.MldPrec()
    _set(p, smoother)
    p.build(a)
    prefix = str(tmp_path / "hier")
    p.dump(prefix)
    assert os.path.exists(prefix + "_p000_l002_ac.mtx")
    assert os.path.exists(prefix + "_sm_p000_l001_" + ("diag" if smoother == "JACOBI" else "lower") + ".mtx")
    q = mld.MldPrec()
    _set(q, smoother)
    q.load_dump(prefix, p.nlev, a)
    assert q.nlev == p.nlev
    x = np.random.default_rng(0).uniform(-1, 1, a.nrows)
    assert _rel(q.apply(x), p.apply(x)) <= 1e-14


def _write_csr(fname, m):
    with open(fname, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n% oracle level\n%\n")
        f.write(f"{m.nrows} {m.ncols} {len(m.val)}\n")
        for i in range(m.nrows):
            for k in range(m.irp[i], m.irp[i + 1]):
                f.write(f"{i + 1} {int(m.ja[k]) + 1} {float(m.val[k])!r}\n")


def _write_vec(fname, v):
    with open(fname, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n% oracle vector\n%\n")
        f.write(f"{len(v)} 1\n")
        for x in v:
            f.write(f"{float(x)!r}\n")


def test_load_files_written_from_the_oracle(mld, orc, tmp_path):
    """BJAC levels with an ILU coarse level, files written by this test in
    the reference's naming from the oracle's (reference-algorithm) data."""
    ao = orc.gen_pde3d(16, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=150))
    op.build(ao)
    prefix = str(tmp_path / "ref")
    for l in range(op.nlev):
        lev = l + 1
        if lev >= 2:
            _write_csr(f"{prefix}_p000_l{lev:03d}_ac.mtx", op.level_csr(l, "A"))
            _write_csr(f"{prefix}_p000_l{lev:03d}_r.mtx", op.level_csr(l, "R"))
            _write_csr(f"{prefix}_p000_l{lev:03d}_p.mtx", op.level_csr(l, "P"))
        _write_csr(f"{prefix}_sm_p000_l{lev:03d}_lower.mtx", op.level_csr(l, "L"))
        _write_csr(f"{prefix}_sm_p000_l{lev:03d}_upper.mtx", op.level_csr(l, "U"))
        _write_vec(f"{prefix}_sm_p000_l{lev:03d}_diag.mtx", op.level_vec(l, "d"))
    am = mld.gen_pde3d(16, 1, ISO)
    q = mld.MldPrec()
    _set(q, "BJAC")
    q.load_dump(prefix, op.nlev, am)
    x = np.random.default_rng(1).uniform(-1, 1, am.nrows)
    assert _rel(q.apply(x), op.apply(x)) <= 1e-12
    with pytest.raises(mld.MldError):
        r = mld.MldPrec()
        _set(r, "BJAC")
        r.load_dump(str(tmp_path / "missing"), op.nlev, am)
