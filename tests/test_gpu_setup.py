"""GPU: hierarchy set-up on the GPU -- the ILU(0) factorisation
(mldg_ilu0_factor) -- against the host build, bit for bit.

The reference factorises row by row (mld_dilu0_fact.f90:284-477); the GPU
factorises all rows of one dependency level at once, each row in the host's
operation order without fused multiply-adds, so L, U and the inverse pivots
must be identical to the oracle's (and the product host build's) on every
level of pdegen hierarchies, isotropic and anisotropic, idim 10..40.  The
host mirror's SETUP_DEVICE=GPU build must give the same hierarchy and the
same applies as the host build, and a zero pivot is reported with its row."""
import ctypes as C

import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params

pytestmark = pytest.mark.gpu


def _ilu_gpu(mld, A):
    lib = mld.lib()
    f = lib.mldg_ilu0_factor
    f.argtypes = [C.c_int, C.c_void_p] + [C.c_void_p] * 7 + [C.POINTER(C.c_int), C.POINTER(C.c_double)]
    n, nz = A.nrows, max(A.nnz, 1)
    Lirp, Uirp = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
    Lja, Uja = np.zeros(nz, np.int32), np.zeros(nz, np.int32)
    Lval, Uval, d = np.zeros(nz), np.zeros(nz), np.zeros(n)
    c = mld.CSR(A.irp, A.ja, A.val, ncols=A.ncols).c()
    bad, ms = C.c_int(0), C.c_double(0)
    rc = f(0, C.byref(c), Lirp.ctypes.data, Lja.ctypes.data, Lval.ctypes.data, Uirp.ctypes.data,
           Uja.ctypes.data, Uval.ctypes.data, d.ctypes.data, C.byref(bad), C.byref(ms))
    return rc, bad.value, (Lirp, Lja[:Lirp[-1]], Lval[:Lirp[-1]]), (Uirp, Uja[:Uirp[-1]], Uval[:Uirp[-1]]), d


@pytest.mark.parametrize("idim,coef", [(10, ISO), (20, ANISO), (32, ISO), (40, ANISO)])
def test_ilu0_gpu_bitwise_equal_to_oracle(mld, orc, idim, coef):
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=100))
    op.build(a)
    for l in range(op.nlev):
        A = op.level_csr(l, "A")
        rc, bad, L, U, d = _ilu_gpu(mld, A)
        assert rc == 0 and bad == -1
        Lo, Uo, do = op.level_csr(l, "L"), op.level_csr(l, "U"), op.level_vec(l, "d")
        assert np.array_equal(L[0], Lo.irp) and np.array_equal(L[1], Lo.ja), l
        assert np.array_equal(U[0], Uo.irp) and np.array_equal(U[1], Uo.ja), l
        assert np.array_equal(L[2], Lo.val), l
        assert np.array_equal(U[2], Uo.val), l
        assert np.array_equal(d, do), l


def test_setup_device_gpu_hierarchy_and_apply(mld, orc):
    a = mld.gen_pde3d(24, 1, ANISO)
    preps = []
    for dev in ("HOST", "GPU"):
        p = mld.MldPrec()
        p.init("ML")
        p.set("SMOOTHER_TYPE", "BJAC")
        p.set("COARSE_SOLVE", "BJAC")
        p.set("COARSE_SWEEPS", 4)
        p.set("MIN_COARSE_SIZE", 300)
        p.set("SETUP_DEVICE", dev)
        p.build(a)
        preps.append(p)
    ph, pg = preps
    assert ph.nlev == pg.nlev
    for l in range(ph.nlev):
        for w in ("L", "U"):
            mh, mg = ph.level_csr(l, w), pg.level_csr(l, w)
            assert np.array_equal(mh.irp, mg.irp) and np.array_equal(mh.ja, mg.ja)
            assert np.array_equal(mh.val, mg.val), (l, w)
        assert np.array_equal(ph.level_vec(l, "d"), pg.level_vec(l, "d"))
    x = np.random.default_rng(1).uniform(-1, 1, a.nrows)
    assert np.array_equal(ph.apply(x), pg.apply(x))


def test_ilu0_gpu_reports_zero_pivot(mld, orc):
    # 3x3 with a zero first pivot: [[0, 1, 0], [1, 2, 0], [0, 0, 1]]
    A = orc.CSR(np.array([0, 1, 3, 4]), np.array([1, 0, 1, 2]), np.array([1.0, 1.0, 2.0, 1.0]))
    rc, bad, _, _, _ = _ilu_gpu(mld, A)
    assert rc == 2 and bad == 0
