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


def test_setup_device_gpu_hierarchy_and_apply(mld, orc, monkeypatch):
    # launch shapes and kernel choices pinned (no timing-based choices), so
    # equal hierarchies give equal bits
    monkeypatch.setenv("MLDG_NO_AUTOTUNE", "1")
    monkeypatch.setenv("MLDG_NO_DENSE_INV", "1")
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


def _spgemm_gpu(mld, A, B):
    lib = mld.lib()
    f = lib.mldg_spgemm
    pp = C.POINTER(C.c_int32)
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.POINTER(pp), C.POINTER(pp),
                  C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_int), C.POINTER(C.c_int),
                  C.POINTER(C.c_double)]
    lib.mldg_free.argtypes = [C.c_void_p]
    a = mld.CSR(A.indptr, A.indices, A.data, ncols=A.shape[1]).c()
    b = mld.CSR(B.indptr, B.indices, B.data, ncols=B.shape[1]).c()
    irp, ja, val = pp(), pp(), C.POINTER(C.c_double)()
    nr, nc, ms = C.c_int(0), C.c_int(0), C.c_double(0)
    rc = f(0, C.byref(a), C.byref(b), C.byref(irp), C.byref(ja), C.byref(val), C.byref(nr), C.byref(nc),
           C.byref(ms))
    assert rc == 0
    n = nr.value
    ci = np.ctypeslib.as_array(irp, (n + 1,)).copy()
    nnz = int(ci[-1])
    cj = np.ctypeslib.as_array(ja, (max(nnz, 1),))[:nnz].copy()
    cv = np.ctypeslib.as_array(val, (max(nnz, 1),))[:nnz].copy()
    for p in (irp, ja, val):
        lib.mldg_free(C.cast(p, C.c_void_p))
    return ci, cj, cv, nc.value


def _spgemm_ref(A, B):
    """The host build's Gustavson order: a_ik in stored order, row k of B in
    stored order, first contribution assigned, later ones added."""
    irp, ja, val = [0], [], []
    for i in range(A.shape[0]):
        acc = {}
        for ka in range(A.indptr[i], A.indptr[i + 1]):
            k, av = A.indices[ka], A.data[ka]
            for kb in range(B.indptr[k], B.indptr[k + 1]):
                j, p = B.indices[kb], av * B.data[kb]
                acc[j] = p if j not in acc else acc[j] + p
        for j in sorted(acc):
            ja.append(j)
            val.append(acc[j])
        irp.append(len(ja))
    return np.array(irp), np.array(ja), np.array(val)


@pytest.mark.parametrize("m,k,n,dens,seed", [(300, 200, 250, 0.05, 0), (64, 2000, 2000, 0.0, 1),
                                             (500, 500, 40, 0.2, 2)])
def test_spgemm_gpu_bitwise_equal_to_host_order(mld, m, k, n, dens, seed):
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    if dens == 0.0:
        # rows with more distinct columns than a warp's table: the host fallback
        A = sp.csr_matrix(rng.uniform(-1, 1, (m, k)) * (rng.uniform(size=(m, k)) < 0.9))
        B = sp.identity(k, format="csr") * 3.0 + sp.random(k, n, density=0.01, random_state=seed, format="csr")
    else:
        A = sp.random(m, k, density=dens, random_state=seed, format="csr")
        B = sp.random(k, n, density=dens, random_state=seed + 7, format="csr")
    A.sort_indices()
    B = B.tocsr()
    B.sort_indices()
    ci, cj, cv, nc = _spgemm_gpu(mld, A, B)
    ri, rj, rv = _spgemm_ref(A, B)
    assert nc == n
    assert np.array_equal(ci, ri) and np.array_equal(cj, rj)
    assert np.array_equal(cv, rv)


@pytest.mark.parametrize("coef", [ISO, ANISO])
def test_setup_device_gpu_level_matrices(mld, orc, coef):
    """SETUP_DEVICE=GPU: P, R and the Galerkin products A_l of every level
    (GPU sparse products) and the ILU(0) factors equal the host build's."""
    a = mld.gen_pde3d(28, 1, coef)
    preps = []
    for dev in ("HOST", "GPU"):
        p = mld.MldPrec()
        p.init("ML")
        p.set("SMOOTHER_TYPE", "BJAC")
        p.set("COARSE_SOLVE", "BJAC")
        p.set("MIN_COARSE_SIZE", 200)
        p.set("SETUP_DEVICE", dev)
        p.hierarchy_build(a)
        p.smoothers_build_host()
        preps.append(p)
    ph, pg = preps
    assert ph.nlev == pg.nlev and ph.nlev >= 3
    for l in range(ph.nlev):
        for w in (["A", "P", "R", "L", "U"] if l else ["A", "L", "U"]):
            mh, mg = ph.level_csr(l, w), pg.level_csr(l, w)
            assert np.array_equal(mh.irp, mg.irp) and np.array_equal(mh.ja, mg.ja), (l, w)
            assert np.array_equal(mh.val, mg.val), (l, w)
