"""CPU: plans of the replicated-window cluster solve (k_trsv_rep), run through
the library's host emulation of the kernel (mldg_rep_plan_check).  The
emulation follows the kernel's step order and checks every ring read against
the position the schedule says the slot holds, every ring read against the
window bound of its step, every far read against its four-step distance and
every block against its descriptor and the stage capacity; the emulated ILU(0)
pair must match a direct triangular solve."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from conftest import ANISO, ISO, oracle_params


def _pair(orc, idim, coef, lev):
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=50))
    op.build(a)
    return op.level_csr(lev, "L"), op.level_csr(lev, "U"), op.level_vec(lev, "d")


def _check(mld, Lm, Um, d, cluster, fp32, trans):
    lib = mld.lib()
    f = lib.mldg_rep_plan_check
    f.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_int, C.c_char, C.c_void_p]
    n = len(d)
    Lc = mld.CSR(Lm.irp, Lm.ja, Lm.val, ncols=n).c()
    Uc = mld.CSR(Um.irp, Um.ja, Um.val, ncols=n).c()
    x = np.random.default_rng(n).uniform(-1, 1, n)
    y = np.zeros(n)
    st = np.zeros(4, np.int64)
    rc = f(C.byref(Lc), C.byref(Uc), d.ctypes.data, x.ctypes.data, y.ctypes.data, cluster, fp32,
           trans.encode(), st.ctypes.data)
    assert rc == 0
    Ls = (sp.csr_matrix((Lm.val, Lm.ja, Lm.irp), shape=(n, n)) + sp.identity(n)).tocsr()
    Us = (sp.csr_matrix((Um.val, Um.ja, Um.irp), shape=(n, n)) + sp.identity(n)).tocsr()
    if trans == "N":
        ref = sla.spsolve_triangular(Us, d * sla.spsolve_triangular(Ls, x, lower=True), lower=False)
    else:
        ref = sla.spsolve_triangular(Ls.T.tocsr(), d * sla.spsolve_triangular(Us.T.tocsr(), x, lower=True),
                                     lower=False)
    err = np.linalg.norm(y - ref) / np.linalg.norm(ref) if st[3] else None
    return st, err


@pytest.mark.parametrize("idim,coef,lev,ring", [(40, ISO, 1, None), (48, ANISO, 1, "4096"),
                                               (60, ISO, 1, "2048"), (56, ISO, 0, None)])
@pytest.mark.parametrize("cluster", [8, 16])
def test_rep_plan_emulation(mld, orc, monkeypatch, idim, coef, lev, ring, cluster):
    """Plans for both cluster sizes, both triangle orders and both precisions;
    a small ring sends the older dependencies of the coarse levels through the
    far path; the finest level of idim=56 has levels wider than one step."""
    if ring:
        monkeypatch.setenv("MLDG_REP_R", ring)
    Lm, Um, d = _pair(orc, idim, coef, lev)
    usable = False
    for fp32, tol in ((0, 1e-13), (1, 1e-6)):
        for trans in ("N", "T"):
            st, err = _check(mld, Lm, Um, d, cluster, fp32, trans)
            assert st[0] == 0, "plan violations"
            if st[3]:
                usable = True
                assert err <= tol, (fp32, trans, err)
    assert usable


def test_rep_plan_far_path_and_split_steps(mld, orc, monkeypatch):
    """A far dependency too few steps back (a 1024-slot ring) makes the plan
    unusable; the far path is taken (dependencies beyond a 2048-slot ring),
    every far copy is reset by the end of the solve, and a level wider than
    the cluster's row slots is split into several steps."""
    monkeypatch.setenv("MLDG_REP_R", "1024")
    Lm, Um, d = _pair(orc, 48, ANISO, 1)
    st, _ = _check(mld, Lm, Um, d, 8, 0, "N")
    assert st[3] == 0 and st[0] == 0
    monkeypatch.setenv("MLDG_REP_R", "2048")
    Lm, Um, d = _pair(orc, 60, ISO, 1)
    st, err = _check(mld, Lm, Um, d, 8, 0, "N")
    assert st[3] == 1 and st[2] > 0 and st[0] == 0 and err <= 1e-13
    monkeypatch.delenv("MLDG_REP_R")
    Lm, Um, d = _pair(orc, 40, ISO, 0)
    st, err = _check(mld, Lm, Um, d, 8, 0, "N")
    nlev = 3 * 40 - 2  # dependency levels of the 7-point lower triangle
    assert st[3] == 1 and st[1] > nlev and st[0] == 0 and err <= 1e-13


def _random_pair(seed, n, reach, per_row):
    """Random strict triangles with a mix of short and long dependencies."""
    rng = np.random.default_rng(seed)

    def tri(lower):
        irp, ja, val = [0], [], []
        for i in range(n):
            cand = []
            for _ in range(rng.integers(0, per_row + 1)):
                back = int(rng.integers(1, reach)) if rng.random() < 0.8 else int(rng.integers(1, n))
                j = i - back if lower else i + back
                if 0 <= j < n:
                    cand.append(j)
            cols = sorted(set(cand))
            ja += cols
            val += list(rng.uniform(-0.3, 0.3, len(cols)))
            irp.append(len(ja))
        return (np.array(irp, np.int32), np.array(ja if ja else [0], np.int32)[:len(ja)],
                np.array(val if val else [0.0])[:len(val)])

    class M:
        pass
    Lm, Um = M(), M()
    Lm.irp, Lm.ja, Lm.val = tri(True)
    Um.irp, Um.ja, Um.val = tri(False)
    d = rng.uniform(0.5, 1.5, n)
    return Lm, Um, d


@pytest.mark.parametrize("seed,n,reach,per_row,ring", [(1, 3000, 40, 6, None), (2, 5000, 400, 4, "2048"),
                                                      (3, 2000, 8, 30, None), (4, 6000, 3000, 3, "1024")])
def test_rep_plan_random_structures(mld, monkeypatch, seed, n, reach, per_row, ring):
    """Irregular triangles: plans are either rejected or replay without a
    single violation and match a direct solve, for both cluster sizes, both
    precisions and both triangle orders."""
    if ring:
        monkeypatch.setenv("MLDG_REP_R", ring)
    Lm, Um, d = _random_pair(seed, n, reach, per_row)
    for cluster in (8, 16):
        for fp32, tol in ((0, 1e-12), (1, 1e-5)):
            for trans in ("N", "T"):
                st, err = _check(mld, Lm, Um, d, cluster, fp32, trans)
                assert st[0] == 0, "plan violations"
                if st[3]:
                    assert err <= tol, (cluster, fp32, trans, err)
