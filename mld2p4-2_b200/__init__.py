"""mld2p4-2_b200 -- B200-native multilevel preconditioner application.

Python view of the product library ``libmldgpu.so``:

* ``Hierarchy`` -- the drop-in C ABI (include/mldg.h): upload a level
  hierarchy built elsewhere (the reference's host build), finalize, apply the
  V-cycle on the GPU, run FCG/CG on the GPU.
* ``MldPrec`` -- the host-side mirror of MLD2P4's ``mld_dprec_type``
  (include/mld_prec.h): ``init / set / hierarchy_build / smoothers_build /
  build / apply / descr / free`` with the same keywords and error codes.
* ``krylov`` -- ``psb_krylov('CG'|'FCG', ...)`` with ``istop=2``.
* ``gen_pde3d`` / ``gen_kappa3d`` -- pdegen-style test problems.

There is no CPU fallback: every entry point runs the CUDA library, and the
library raises when it cannot reach a GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmldgpu.so")
_lib = None

# smoother kinds / precision forms / memory kinds (include/mldg.h)
SMOOTHER_JACOBI = 1
SMOOTHER_BJAC = 2
SMOOTHER_FBGS = 3
CYCLE_V, CYCLE_W, CYCLE_K, CYCLE_KSYM, CYCLE_ADD = 0, 1, 2, 3, 4
PREC_FP64, PREC_FP32, PREC_FP32_P16, PREC_FP32_H16 = 0, 1, 2, 3
MEM_HOST, MEM_DEVICE = 0, 1

ERR_NOT_BUILT = 3112
ERR_TIMEOUT = 4020
ERR_NOT_CONVERGED = 4030


class MldError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _CSR(C.Structure):
    _fields_ = [("nrows", C.c_int32), ("ncols", C.c_int32),
                ("irp", C.POINTER(C.c_int32)), ("ja", C.POINTER(C.c_int32)),
                ("val", C.POINTER(C.c_double))]


class _Opts(C.Structure):
    _fields_ = [("device", C.c_int), ("index_base", C.c_int),
                ("use_graphs", C.c_int), ("autotune", C.c_int)]


class _LevelDesc(C.Structure):
    _fields_ = [("A", _CSR), ("P", _CSR), ("R", _CSR), ("ND", _CSR), ("L", _CSR),
                ("U", _CSR), ("d", C.POINTER(C.c_double)), ("smoother_kind", C.c_int),
                ("sweeps_pre", C.c_int), ("sweeps_post", C.c_int), ("damping", C.c_double)]


class _KStat(C.Structure):
    _fields_ = [("kind", C.c_int), ("level", C.c_int), ("bytes", C.c_int64),
                ("ms", C.c_double)]


KERNEL_TRSV, KERNEL_SPMV, KERNEL_JACOBI, KERNEL_VEC = 1, 2, 3, 4
KERNEL_NAMES = {1: "trsv", 2: "spmv", 3: "jacobi", 4: "vec"}


class _GpuDiag:
    """Timing diagnostics shared by Hierarchy and MldPrec (needs self._gpu())."""

    def probe_set(self, kind: int, lev: int, index: int = 0):
        rc = lib().mldg_probe_set(self._gpu(), kind, lev, index)
        if rc:
            raise MldError(rc, "probe_set")

    def probe_read(self):
        ms = C.c_double(0)
        cnt = C.c_int64(0)
        b = C.c_int64(0)
        lib().mldg_probe_read(self._gpu(), C.byref(ms), C.byref(cnt), C.byref(b))
        return ms.value, cnt.value, b.value

    def profile(self, trans: str = "N", nrhs: int = 1):
        """One un-graphed V-cycle (nrhs columns) with events around every launch."""
        stats = (_KStat * 4096)()
        n = C.c_int(0)
        rc = lib().mldg_profile_multi(self._gpu(), trans.encode(), nrhs, 4096, stats, C.byref(n))
        if rc:
            raise MldError(rc, "profile")
        return [{"kind": KERNEL_NAMES.get(s.kind, "?"), "kind_id": s.kind, "level": s.level,
                 "bytes": s.bytes, "ms": s.ms} for s in stats[: min(n.value, 4096)]]

    def last_timing(self):
        ms = C.c_double(0)
        nl = C.c_int64(0)
        lib().mldg_last_timing(self._gpu(), C.byref(ms), C.byref(nl))
        return ms.value, nl.value

    def adjoint(self, g, lam=None, eps: float = 1e-10, itmax: int = 500):
        """Solve A^T lam = g (FCG with the transposed V-cycle). Returns (lam, iters, relres)."""
        if lam is None:
            lam = np.zeros_like(g) if isinstance(g, np.ndarray) else g.new_zeros(g.shape)
        lp, gp, mem = _vec_args(lam, g)
        it = C.c_int(0)
        rr = C.c_double(0)
        rc = lib().mldg_adjoint(self._gpu(), gp, lp, eps, itmax, C.byref(it), C.byref(rr), mem)
        if rc and rc != ERR_NOT_CONVERGED:
            raise MldError(rc, lib().mldg_last_error(self._gpu()).decode())
        return lam, it.value, rr.value

    def kappa_grad(self, idim: int, kappa, x, lam, grad=None):
        """dL/dkappa from the forward solution x and the adjoint lam (harmonic-mean faces)."""
        if grad is None:
            grad = np.zeros_like(x) if isinstance(x, np.ndarray) else x.new_zeros(x.shape)
        kp, xp, mem = _vec_args(kappa, x)
        lp, gp, _ = _vec_args(lam, grad)
        rc = lib().mldg_kappa_grad(self._gpu(), idim, kp, xp, lp, gp, mem)
        if rc:
            raise MldError(rc, lib().mldg_last_error(self._gpu()).decode())
        return grad

    def apply_block(self, X, Y=None, trans: str = "N"):
        """Y = M^{-1} X for a block of right-hand sides: X has shape (nrhs, n),
        contiguous (column c of the C-ABI block is X[c]); numpy or torch."""
        if Y is None:
            Y = np.zeros_like(X) if isinstance(X, np.ndarray) else X.new_zeros(X.shape)
        nrhs, ld = X.shape
        xp, yp, mem = _vec_args(X, Y)
        rc = lib().mldg_apply(self._gpu(), xp, yp, trans.encode(), nrhs, ld, mem)
        if rc:
            raise MldError(rc, lib().mldg_last_error(self._gpu()).decode())
        return Y

    def krylov_multi(self, method: str, B, X=None, eps: float = 1e-10, itmax: int = 500,
                     A: "CSR | None" = None):
        """nrhs independent CG/FCG solves advanced together (mldg_krylov_multi).
        B has shape (nrhs, n).  Returns (X, iters[nrhs], relres[nrhs])."""
        m = {"CG": 0, "FCG": 1}[method.upper()]
        if X is None:
            X = np.zeros_like(B) if isinstance(B, np.ndarray) else B.new_zeros(B.shape)
        nrhs, ld = B.shape
        xp, bp, mem = _vec_args(X, B)
        it = (C.c_int * max(nrhs, 1))()
        rr = (C.c_double * max(nrhs, 1))()
        Ac = A.c() if A is not None else None
        rc = lib().mldg_krylov_multi(self._gpu(), m, C.byref(Ac) if Ac is not None else None, nrhs,
                                     bp, ld, xp, X.shape[1], eps, itmax, it, rr, mem)
        if rc and rc != ERR_NOT_CONVERGED:
            raise MldError(rc, lib().mldg_last_error(self._gpu()).decode())
        return X, np.array(it[:nrhs]), np.array(rr[:nrhs])

    def apply_bytes(self) -> int:
        """Algorithmic bytes of one V-cycle apply (mldg_apply_bytes)."""
        b = C.c_int64(0)
        lib().mldg_apply_bytes(self._gpu(), C.byref(b))
        return b.value

    def apply_impl_bytes(self) -> int:
        """Bytes the chosen kernels of one V-cycle apply move (dense inverses at full size)."""
        b = C.c_int64(0)
        lib().mldg_apply_impl_bytes(self._gpu(), C.byref(b))
        return b.value


def lib():
    """Load libmldgpu.so (built by build.py); raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built: run python mld2p4-2_b200/build.py")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)
        L.mldg_create.argtypes = [C.POINTER(vp), C.POINTER(_Opts)]
        L.mldg_upload_level.argtypes = [vp, C.c_int, C.POINTER(_LevelDesc)]
        L.mldg_finalize.argtypes = [vp, C.c_int, C.c_int]
        L.mldg_apply.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_char, C.c_int, C.c_int, C.c_int]
        L.mldg_krylov.argtypes = [vp, C.c_int, C.POINTER(_CSR), C.c_void_p, C.c_void_p,
                                  C.c_double, C.c_int, C.POINTER(C.c_int),
                                  C.POINTER(C.c_double), C.c_int]
        L.mldg_krylov_multi.argtypes = [vp, C.c_int, C.POINTER(_CSR), C.c_int, C.c_void_p, C.c_int,
                                        C.c_void_p, C.c_int, C.c_double, C.c_int,
                                        C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int]
        L.mldg_krylov_batch.argtypes = [C.c_int, C.POINTER(vp), C.c_int, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p), C.c_double, C.c_int,
                                        C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int,
                                        C.POINTER(C.c_double)]
        L.mldg_set_cycle.argtypes = [vp, C.c_int]
        L.mldg_level_info.argtypes = [vp, C.c_int, C.POINTER(C.c_int64)]
        L.mldg_last_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.mldg_apply_bytes.argtypes = [vp, C.POINTER(C.c_int64)]
        L.mldg_apply_impl_bytes.argtypes = [vp, C.POINTER(C.c_int64)]
        L.mldg_probe_set.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.mldg_probe_read.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64)]
        L.mldg_profile.argtypes = [vp, C.c_char, C.c_int, C.POINTER(_KStat),
                                   C.POINTER(C.c_int)]
        L.mldg_profile_multi.argtypes = [vp, C.c_char, C.c_int, C.c_int, C.POINTER(_KStat),
                                         C.POINTER(C.c_int)]
        L.mldg_relres_noalloc.argtypes = [vp, C.POINTER(_CSR), C.c_void_p, C.c_void_p,
                                          C.POINTER(C.c_double)]
        L.mldg_adjoint.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int]
        L.mldg_kappa_grad.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_int]
        L.mldg_last_error.argtypes = [vp]
        L.mldg_last_error.restype = C.c_char_p
        L.mldg_destroy.argtypes = [vp]
        L.mldp_create.argtypes = [C.POINTER(vp), C.c_int]
        L.mldp_init.argtypes = [vp, C.c_char_p]
        L.mldp_seti.argtypes = [vp, C.c_char_p, C.c_int, C.c_int]
        L.mldp_setr.argtypes = [vp, C.c_char_p, C.c_double, C.c_int]
        L.mldp_setc.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int]
        L.mldp_hierarchy_build.argtypes = [vp, C.c_int, ip, ip, dp]
        L.mldp_smoothers_build.argtypes = [vp]
        L.mldp_smoothers_build_host.argtypes = [vp]
        L.mldp_build.argtypes = [vp, C.c_int, ip, ip, dp]
        L.mldp_apply.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_char, C.c_int]
        L.mldp_krylov.argtypes = [vp, C.c_char_p, C.c_int, ip, ip, dp, C.c_void_p, C.c_void_p,
                                  C.c_double, C.c_int, C.POINTER(C.c_int),
                                  C.POINTER(C.c_double), C.c_int]
        L.mldp_nlev.argtypes = [vp]
        L.mldp_dump.argtypes = [vp, C.c_char_p]
        L.mldp_load_dump.argtypes = [vp, C.c_char_p, C.c_int, C.c_int, ip, ip, dp]
        L.mldp_level_info.argtypes = [vp, C.c_int, C.POINTER(C.c_int64), dp]
        L.mldp_level_csr.argtypes = [vp, C.c_int, C.c_char_p, ip, ip, dp]
        L.mldp_level_vec.argtypes = [vp, C.c_int, C.c_char_p, dp, ip]
        L.mldp_descr.argtypes = [vp, C.c_char_p, C.c_int]
        L.mldp_gpu.argtypes = [vp]
        L.mldp_gpu.restype = vp
        L.mldp_last_error.argtypes = [vp]
        L.mldp_last_error.restype = C.c_char_p
        L.mldp_destroy.argtypes = [vp]
        L.mldp_pde3d_nnz.argtypes = [C.c_int]
        L.mldp_pde3d_nnz.restype = C.c_int64
        L.mldp_gen_pde3d.argtypes = [C.c_int, C.c_int, dp, ip, ip, dp]
        L.mldp_gen_kappa3d.argtypes = [C.c_int, dp, ip, ip, dp]
        _lib = L
    return _lib


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class CSR:
    """0-based CSR triple (int32 indices, float64 values)."""

    def __init__(self, irp, ja, val, ncols=None):
        self.irp = np.ascontiguousarray(irp, dtype=np.int32)
        self.ja = np.ascontiguousarray(ja, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        self.nrows = len(self.irp) - 1
        self.ncols = self.nrows if ncols is None else int(ncols)

    @property
    def nnz(self) -> int:
        return int(self.irp[-1])

    def c(self) -> _CSR:
        return _CSR(self.nrows, self.ncols, _ip(self.irp), _ip(self.ja), _dp(self.val))

    def matvec(self, x):
        x = np.asarray(x, dtype=np.float64)
        rows = np.repeat(np.arange(self.nrows), np.diff(self.irp))
        return np.bincount(rows, weights=self.val * x[self.ja], minlength=self.nrows)


def gen_pde3d(idim: int, hden: int = 1, coef=(1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0)) -> CSR:
    """3D 7-point convection-diffusion matrix, h = 1/(idim+hden)."""
    L = lib()
    n = idim ** 3
    nnz = L.mldp_pde3d_nnz(idim)
    irp = np.zeros(n + 1, np.int32)
    ja = np.zeros(nnz, np.int32)
    val = np.zeros(nnz, np.float64)
    c = np.ascontiguousarray(coef, np.float64)
    rc = L.mldp_gen_pde3d(idim, hden, _dp(c), _ip(irp), _ip(ja), _dp(val))
    if rc:
        raise MldError(rc, "gen_pde3d")
    return CSR(irp, ja, val)


def gen_kappa3d(idim: int, kappa: np.ndarray) -> CSR:
    """-div(kappa grad u) on idim^3 unknowns, harmonic-mean faces, h=1/(idim+1)."""
    L = lib()
    n = idim ** 3
    kappa = np.ascontiguousarray(kappa, np.float64).ravel()
    assert kappa.size == n
    nnz = L.mldp_pde3d_nnz(idim)
    irp = np.zeros(n + 1, np.int32)
    ja = np.zeros(nnz, np.int32)
    val = np.zeros(nnz, np.float64)
    rc = L.mldp_gen_kappa3d(idim, _dp(kappa), _ip(irp), _ip(ja), _dp(val))
    if rc:
        raise MldError(rc, "gen_kappa3d")
    return CSR(irp, ja, val)


def grf3d(idim: int, corr_len: float = 0.1, variance: float = 1.0, seed: int = 0) -> np.ndarray:
    """Smooth Gaussian random field on the idim^3 cells of the unit cube.

    White noise filtered in Fourier space by exp(-(corr_len k)^2 / 4) (its
    square is the spectrum of the squared-exponential covariance of length
    corr_len) on a periodic grid padded by 3 correlation lengths, then
    standardised to mean 0 and the requested variance.  Returned flat in the
    generator's row order (x slowest, z fastest).
    """
    h = 1.0 / (idim + 1)
    pad = int(np.ceil(3 * corr_len / h))
    N = idim + pad
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((N, N, N))
    k = 2 * np.pi * np.fft.fftfreq(N, d=h)
    kz = 2 * np.pi * np.fft.rfftfreq(N, d=h)
    K2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    f = np.fft.irfftn(np.fft.rfftn(w) * np.exp(-(corr_len ** 2) * K2 / 4.0), s=(N, N, N))
    f = f[:idim, :idim, :idim]
    f = (f - f.mean()) / f.std() * np.sqrt(variance)
    return np.ascontiguousarray(f.reshape(-1))


def _vec_args(x, y):
    """Return (xptr, yptr, mem_kind, keepalive) for numpy or torch tensors."""
    try:
        import torch
        if isinstance(x, torch.Tensor):
            assert x.dtype == torch.float64 and y.dtype == torch.float64
            assert x.is_contiguous() and y.is_contiguous()
            mem = MEM_DEVICE if x.is_cuda else MEM_HOST
            return C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), mem
    except ImportError:
        pass
    return C.c_void_p(x.ctypes.data), C.c_void_p(y.ctypes.data), MEM_HOST


class Hierarchy(_GpuDiag):
    """The drop-in boundary: upload levels, finalize, apply on the GPU."""

    def _gpu(self):
        return self._h

    def __init__(self, device: int = 0, use_graphs: bool = True, index_base: int = 0,
                 autotune: bool = True):
        self._h = C.c_void_p()
        o = _Opts(device, index_base, 1 if use_graphs else 0, 1 if autotune else 0)
        rc = lib().mldg_create(C.byref(self._h), C.byref(o))
        if rc:
            raise MldError(rc, "mldg_create failed (no usable CUDA device?)")
        self._keep = []
        self.n = 0

    def _check(self, rc):
        if rc:
            raise MldError(rc, lib().mldg_last_error(self._h).decode())

    def upload_level(self, lev: int, A: CSR, P: CSR | None = None, R: CSR | None = None,
                     ND: CSR | None = None, L: CSR | None = None, U: CSR | None = None,
                     d=None, smoother=SMOOTHER_BJAC, sweeps_pre=1, sweeps_post=1,
                     damping=1.0):
        def cc(m):
            return m.c() if m is not None else _CSR(0, 0, None, None, None)
        dd = np.ascontiguousarray(d, np.float64) if d is not None else None
        desc = _LevelDesc(cc(A), cc(P), cc(R), cc(ND), cc(L), cc(U),
                          _dp(dd) if dd is not None else None, smoother, sweeps_pre,
                          sweeps_post, damping)
        self._keep.append((A, P, R, ND, L, U, dd))
        self._check(lib().mldg_upload_level(self._h, lev, C.byref(desc)))
        if lev == 0:
            self.n = A.nrows

    def set_cycle(self, cycle: int):
        """MLDG_CYCLE_V (0), _W (1), _K (2, inner GCR) or _KSYM (3, inner FCG)."""
        self._check(lib().mldg_set_cycle(self._h, cycle))

    def finalize(self, nlev: int, precision: int = PREC_FP64):
        self._check(lib().mldg_finalize(self._h, nlev, precision))
        self._keep = []

    def apply(self, x, y=None, trans: str = "N"):
        if y is None:
            y = np.zeros_like(x)
        xp, yp, mem = _vec_args(x, y)
        self._check(lib().mldg_apply(self._h, xp, yp, trans.encode(), 1, self.n, mem))
        return y

    def krylov(self, method: str, b, x=None, eps=1e-10, itmax=500, A: CSR | None = None):
        m = {"CG": 0, "FCG": 1}[method.upper()]
        if x is None:
            x = np.zeros_like(b)
        xp, bp, mem = _vec_args(x, b)
        it = C.c_int(0)
        err = C.c_double(0)
        Ac = A.c() if A is not None else None
        rc = lib().mldg_krylov(self._h, m, C.byref(Ac) if Ac is not None else None, bp, xp, eps,
                               itmax, C.byref(it), C.byref(err), mem)
        if rc and rc != ERR_NOT_CONVERGED:
            self._check(rc)
        return x, it.value, err.value

    def level_info(self, lev: int):
        info = (C.c_int64 * 5)()
        self._check(lib().mldg_level_info(self._h, lev, info))
        return {"n": info[0], "nnzA": info[1], "nnzP": info[2], "nnz_smoother": info[3],
                "nlev": info[4]}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().mldg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MldPrec(_GpuDiag):
    """Mirror of type(mld_dprec_type): init / set / build / apply / descr / free."""

    def _gpu(self):
        return lib().mldp_gpu(self._p)

    def __init__(self, device: int = 0):
        self._p = C.c_void_p()
        rc = lib().mldp_create(C.byref(self._p), device)
        if rc:
            raise MldError(rc, "mldp_create")
        self.n = 0

    def _check(self, rc):
        if rc:
            raise MldError(rc, lib().mldp_last_error(self._p).decode())

    def init(self, ptype: str = "ML"):
        self._check(lib().mldp_init(self._p, ptype.encode()))

    def set(self, what: str, val, ilev: int | None = None):
        il = -1 if ilev is None else ilev
        if isinstance(val, str):
            rc = lib().mldp_setc(self._p, what.encode(), val.encode(), il)
        elif isinstance(val, (int, np.integer)) and not isinstance(val, bool):
            rc = lib().mldp_seti(self._p, what.encode(), int(val), il)
        else:
            rc = lib().mldp_setr(self._p, what.encode(), float(val), il)
        self._check(rc)

    def hierarchy_build(self, a: CSR):
        self._a = a
        self.n = a.nrows
        self._check(lib().mldp_hierarchy_build(self._p, a.nrows, _ip(a.irp), _ip(a.ja), _dp(a.val)))

    def smoothers_build(self):
        self._check(lib().mldp_smoothers_build(self._p))

    def smoothers_build_host(self):
        """Smoother/solver data on the host only (no GPU upload), for checking."""
        self._check(lib().mldp_smoothers_build_host(self._p))

    def build(self, a: CSR):
        self.hierarchy_build(a)
        self.smoothers_build()

    def apply(self, x, y=None, trans: str = "N"):
        if y is None:
            y = np.zeros_like(x)
        xp, yp, mem = _vec_args(x, y)
        self._check(lib().mldp_apply(self._p, xp, yp, trans.encode(), mem))
        return y

    @property
    def nlev(self) -> int:
        return lib().mldp_nlev(self._p)

    def level_info(self, lev: int) -> dict:
        info = np.zeros(10, np.int64)
        dinfo = np.zeros(2, np.float64)
        self._check(lib().mldp_level_info(self._p, lev, info.ctypes.data_as(C.POINTER(C.c_int64)),
                                          _dp(dinfo)))
        keys = ["n", "nnzA", "nnzP", "nnzR", "nnzL", "nnzU", "nnzND", "naggr", "smoother",
                "sweeps_pre"]
        d = {k: int(v) for k, v in zip(keys, info)}
        d["omega"], d["damp"] = float(dinfo[0]), float(dinfo[1])
        return d

    def level_csr(self, lev: int, which: str) -> CSR | None:
        info = self.level_info(lev)
        nnz = info[{"A": "nnzA", "P": "nnzP", "R": "nnzR", "L": "nnzL", "U": "nnzU",
                    "ND": "nnzND"}[which]]
        if which == "P":
            if lev == 0:
                return None
            nr, nc = self.level_info(lev - 1)["n"], info["n"]
        elif which == "R":
            if lev == 0:
                return None
            nr, nc = info["n"], self.level_info(lev - 1)["n"]
        else:
            nr = nc = info["n"]
        irp = np.zeros(nr + 1, np.int32)
        ja = np.zeros(max(nnz, 1), np.int32)
        val = np.zeros(max(nnz, 1), np.float64)
        rc = lib().mldp_level_csr(self._p, lev, which.encode(), _ip(irp), _ip(ja), _dp(val))
        if rc:
            return None
        return CSR(irp, ja[:nnz], val[:nnz], ncols=nc)

    def level_vec(self, lev: int, which: str):
        if which == "ilaggr":
            n = self.level_info(lev - 1)["n"]
            iv = np.zeros(n, np.int32)
            rc = lib().mldp_level_vec(self._p, lev, b"ilaggr", None, _ip(iv))
            return None if rc else iv
        n = self.level_info(lev)["n"]
        dv = np.zeros(n, np.float64)
        rc = lib().mldp_level_vec(self._p, lev, which.encode(), _dp(dv), None)
        return None if rc else dv

    def dump(self, prefix: str):
        """Write the built hierarchy as the reference's prec%dump would (MatrixMarket)."""
        self._check(lib().mldp_dump(self._p, prefix.encode()))

    def load_dump(self, prefix: str, nlev: int, a: CSR):
        """Build from a prec%dump file set: level 1 is `a`, the rest from the files."""
        self._check(lib().mldp_load_dump(self._p, prefix.encode(), nlev, a.nrows, _ip(a.irp),
                                         _ip(a.ja), _dp(a.val)))

    def descr(self) -> str:
        buf = C.create_string_buffer(8192)
        self._check(lib().mldp_descr(self._p, buf, 8192))
        return buf.value.decode()

    def free(self):
        if getattr(self, "_p", None) and self._p.value:
            lib().mldp_destroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def krylov(method: str, a: CSR, prec: MldPrec, b, x=None, eps: float = 1e-10,
           itmax: int = 500, use_prec_matrix: bool = False):
    """psb_krylov(method, a, prec, b, x, eps, ..., istop=2) on the GPU.

    Returns (x, iters, relres).  ``use_prec_matrix`` reuses the preconditioner's
    level-0 copy of ``a`` instead of uploading ``a`` again.
    """
    if x is None:
        x = np.zeros_like(b)
    xp, bp, mem = _vec_args(x, b)
    it = C.c_int(0)
    err = C.c_double(0)
    if use_prec_matrix:
        rc = lib().mldp_krylov(prec._p, method.encode(), a.nrows, None, None, None, bp, xp, eps,
                               itmax, C.byref(it), C.byref(err), mem)
    else:
        rc = lib().mldp_krylov(prec._p, method.encode(), a.nrows, _ip(a.irp), _ip(a.ja),
                               _dp(a.val), bp, xp, eps, itmax, C.byref(it), C.byref(err), mem)
    if rc and rc != ERR_NOT_CONVERGED:
        prec._check(rc)
    return x, it.value, err.value


def krylov_batch(method: str, precs, bs, xs=None, eps: float = 1e-10, itmax: int = 500):
    """Independent systems solved together (mldg_krylov_batch): precs[i] is a built
    MldPrec or a finalized Hierarchy whose finest level is system i's matrix; bs[i]
    its right-hand side (numpy or torch, all of one kind).  Returns
    (xs, iters[nsys], relres[nsys], device ms of the whole batch)."""
    m = {"CG": 0, "FCG": 1}[method.upper()]
    nsys = len(precs)
    if len(bs) != nsys or (xs is not None and len(xs) != nsys):
        raise ValueError("krylov_batch: precs, bs and xs must have one entry per system")
    if xs is None:
        xs = [np.zeros_like(b) if isinstance(b, np.ndarray) else b.new_zeros(b.shape) for b in bs]
    hs = (C.c_void_p * max(nsys, 1))()
    bp = (C.c_void_p * max(nsys, 1))()
    xp = (C.c_void_p * max(nsys, 1))()
    mem = MEM_HOST
    for i, (p, b, x) in enumerate(zip(precs, bs, xs)):
        hs[i] = p._gpu()
        xptr, bptr, mem = _vec_args(x, b)
        xp[i], bp[i] = xptr, bptr
    it = (C.c_int * max(nsys, 1))()
    rr = (C.c_double * max(nsys, 1))()
    ms = C.c_double(0)
    rc = lib().mldg_krylov_batch(nsys, hs, m, bp, xp, eps, itmax, it, rr, mem, C.byref(ms))
    if rc and rc != ERR_NOT_CONVERGED:
        raise MldError(rc, lib().mldg_last_error(hs[0]).decode() if nsys else "krylov_batch")
    return xs, np.array(it[:nsys]), np.array(rr[:nsys]), ms.value
