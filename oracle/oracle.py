"""ctypes binding of the C test oracle (oracle/mld_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by ``bench.py``'s cpu_baseline / reference arm.  The
product package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

JACOBI = 1
BJAC = 2
VCYCLE, WCYCLE, KCYCLE, KCYCLESYM, ADD = 0, 1, 2, 3, 4  # ml_cycle
FBGS = 3  # forward GS pre / backward GS post (jac smoother + GS / BWGS solvers)


class Params(C.Structure):
    _fields_ = [
        ("smoother", C.c_int),
        ("sweeps_pre", C.c_int),
        ("sweeps_post", C.c_int),
        ("jac_damp", C.c_double),
        ("coarse_solver", C.c_int),
        ("coarse_sweeps", C.c_int),
        ("min_coarse_size", C.c_int),
        ("max_levs", C.c_int),
        ("min_cr_ratio", C.c_double),
        ("aggr_thresh", C.c_double),
        ("ml_cycle", C.c_int),
    ]


def build_lib() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, no GPU)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "mld_oracle.c")
        ):
            build_lib()
        L = C.CDLL(_LIB_PATH)
        ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        lp = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
        L.orc_default_params.argtypes = [C.POINTER(Params)]
        L.orc_pde3d_nnz.argtypes = [C.c_int]
        L.orc_pde3d_nnz.restype = C.c_long
        L.orc_gen_pde3d.argtypes = [C.c_int, C.c_int, dp, ip, ip, dp]
        L.orc_prec_new.argtypes = [C.POINTER(Params)]
        L.orc_prec_new.restype = C.c_void_p
        L.orc_prec_free.argtypes = [C.c_void_p]
        L.orc_prec_build.argtypes = [C.c_void_p, C.c_int, ip, ip, dp]
        L.orc_prec_nlev.argtypes = [C.c_void_p]
        L.orc_prec_level_info.argtypes = [C.c_void_p, C.c_int, lp, dp]
        L.orc_prec_level_csr.argtypes = [C.c_void_p, C.c_int, C.c_int, ip, ip, dp]
        L.orc_prec_level_vec.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, ip]
        L.orc_prec_apply.argtypes = [C.c_void_p, dp, dp, C.c_char]
        L.orc_krylov.argtypes = [C.c_int, C.c_int, ip, ip, dp, C.c_void_p, dp, dp,
                                 C.c_double, C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_double), dp]
        L.orc_spmv.argtypes = [C.c_int, ip, ip, dp, C.c_double, dp, C.c_double, dp]
        L.orc_spmv_t.argtypes = [C.c_int, C.c_int, ip, ip, dp, C.c_double, dp,
                                 C.c_double, dp]
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def default_params(**kw) -> Params:
    p = Params()
    lib().orc_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class CSR:
    """Plain 0-based CSR triple (int32 indices, float64 values)."""

    def __init__(self, irp, ja, val, ncols=None):
        self.irp = np.ascontiguousarray(irp, dtype=np.int32)
        self.ja = np.ascontiguousarray(ja, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        self.nrows = len(self.irp) - 1
        self.ncols = self.nrows if ncols is None else ncols

    @property
    def nnz(self):
        return int(self.irp[-1])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.ja, self.irp), shape=(self.nrows, self.ncols))


def gen_pde3d(idim: int, hden: int = 1, coef=(1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0)) -> CSR:
    """3D 7-point convection-diffusion matrix (tests/pdegen/mld_d_pde3d.f90)."""
    L = lib()
    n = idim ** 3
    nnz = L.orc_pde3d_nnz(idim)
    irp = np.zeros(n + 1, np.int32)
    ja = np.zeros(nnz, np.int32)
    val = np.zeros(nnz, np.float64)
    L.orc_gen_pde3d(idim, hden, np.asarray(coef, np.float64), irp, ja, val)
    return CSR(irp, ja, val)


class Prec:
    """Oracle multilevel preconditioner (build + apply)."""

    def __init__(self, params: Params | None = None):
        self._p = lib().orc_prec_new(C.byref(params) if params is not None else None)

    def __del__(self):
        if getattr(self, "_p", None):
            lib().orc_prec_free(self._p)
            self._p = None

    def build(self, a: CSR) -> None:
        rc = lib().orc_prec_build(self._p, a.nrows, a.irp, a.ja, a.val)
        if rc != 0:
            raise RuntimeError(f"oracle build failed: {rc}")

    @property
    def nlev(self) -> int:
        return lib().orc_prec_nlev(self._p)

    def level_info(self, lev: int) -> dict:
        info = np.zeros(10, np.int64)
        dinfo = np.zeros(2, np.float64)
        lib().orc_prec_level_info(self._p, lev, info, dinfo)
        keys = ["n", "nnzA", "nnzP", "nnzR", "nnzL", "nnzU", "nnzND", "naggr",
                "smoother", "sweeps_pre"]
        d = {k: int(v) for k, v in zip(keys, info)}
        d["omega"] = float(dinfo[0])
        d["damp"] = float(dinfo[1])
        return d

    def level_csr(self, lev: int, which: str) -> CSR | None:
        w = {"A": 0, "P": 1, "R": 2, "L": 3, "U": 4, "ND": 5}[which]
        info = self.level_info(lev)
        n = info["n"]
        if which == "P":
            nr = self.level_info(lev - 1)["n"] if lev > 0 else 0
            nc, nnz = n, info["nnzP"]
        elif which == "R":
            nr, nnz = n, info["nnzR"]
            nc = self.level_info(lev - 1)["n"] if lev > 0 else 0
        else:
            nr, nc = n, n
            nnz = info[{"A": "nnzA", "L": "nnzL", "U": "nnzU", "ND": "nnzND"}[which]]
        if lev == 0 and which in ("P", "R"):
            return None
        irp = np.zeros(nr + 1, np.int32)
        ja = np.zeros(max(nnz, 1), np.int32)
        val = np.zeros(max(nnz, 1), np.float64)
        rc = lib().orc_prec_level_csr(self._p, lev, w, irp, ja, val)
        if rc != 0:
            return None
        return CSR(irp, ja[:nnz], val[:nnz], ncols=nc)

    def level_vec(self, lev: int, which: str):
        w = {"d": 0, "dinv": 1, "ilaggr": 2}[which]
        n = self.level_info(lev)["n"]
        if which == "ilaggr":
            nf = self.level_info(lev - 1)["n"]
            iv = np.zeros(nf, np.int32)
            rc = lib().orc_prec_level_vec(self._p, lev, w, np.zeros(1), iv)
            return None if rc else iv
        dv = np.zeros(n, np.float64)
        rc = lib().orc_prec_level_vec(self._p, lev, w, dv, np.zeros(1, np.int32))
        return None if rc else dv

    def apply(self, x: np.ndarray, trans: str = "N") -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        rc = lib().orc_prec_apply(self._p, x, y, trans.encode())
        if rc != 0:
            raise RuntimeError(f"oracle apply failed: {rc}")
        return y


def krylov(method: str, a: CSR, prec: Prec | None, b: np.ndarray, x0=None,
           eps: float = 1e-10, itmax: int = 1000):
    """CG / FCG (istop 2). Returns (x, iters, relres, history)."""
    m = {"CG": 0, "FCG": 1}[method.upper()]
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    it = C.c_int(0)
    rr = C.c_double(0)
    hist = np.zeros(itmax + 1, np.float64)
    rc = lib().orc_krylov(m, a.nrows, a.irp, a.ja, a.val, prec._p if prec else None,
                          b, x, eps, itmax, C.byref(it), C.byref(rr), hist)
    if rc != 0:
        raise RuntimeError(f"oracle krylov failed: {rc}")
    return x, it.value, rr.value, hist[: it.value].copy()


def spmv(a: CSR, x, alpha=1.0, beta=0.0, y=None, trans="N"):
    x = np.ascontiguousarray(x, dtype=np.float64)
    if trans == "N":
        y = np.zeros(a.nrows) if y is None else np.array(y, dtype=np.float64)
        lib().orc_spmv(a.nrows, a.irp, a.ja, a.val, alpha, x, beta, y)
    else:
        y = np.zeros(a.ncols) if y is None else np.array(y, dtype=np.float64)
        lib().orc_spmv_t(a.nrows, a.ncols, a.irp, a.ja, a.val, alpha, x, beta, y)
    return y


def num_threads() -> int:
    return lib().orc_num_threads()
