"""GPU: the allocation-free relative residual (mldg_relres_noalloc).

Some callers cannot allocate device memory: applications whose own memory
pool or allocator owns every device byte, and tight host-side convergence
loops where each cudaMalloc/cudaFree would synchronise the whole device.
For them the library computes ||b - A x|| / ||b||
with its scratch in a fixed file-scope device array instead of memory it
allocates.  This test calls that entry point through the C ABI twice in a
row and checks each result against the regular path (mldg_krylov with
itmax = 0, which computes the same relative residual in scratch allocated
at mldg_finalize) to 1e-12 relative, and checks the size limit.

This file is collected last so that a stop-at-first-failure run has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _dev_csr(mld, torch, m):
    irp = torch.tensor(m.irp, dtype=torch.int32, device="cuda")
    ja = torch.tensor(m.ja, dtype=torch.int32, device="cuda")
    val = torch.tensor(m.val, dtype=torch.float64, device="cuda")
    c = mld._CSR(m.nrows, m.nrows, C.cast(C.c_void_p(irp.data_ptr()), C.POINTER(C.c_int32)),
                 C.cast(C.c_void_p(ja.data_ptr()), C.POINTER(C.c_int32)),
                 C.cast(C.c_void_p(val.data_ptr()), C.POINTER(C.c_double)))
    return c, (irp, ja, val)


def test_noalloc_relres_matches_regular_path(mld, orc):
    import torch
    a = orc.gen_pde3d(20, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=500))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    csr, keep = _dev_csr(mld, torch, a)
    rng = np.random.default_rng(11)
    b = torch.tensor(orc.spmv(a, np.ones(a.nrows)), dtype=torch.float64, device="cuda")
    for call in range(2):  # two calls in a row share (and overwrite) the scratch
        xh = rng.uniform(-1, 1, a.nrows)
        x = torch.tensor(xh, dtype=torch.float64, device="cuda")
        rr = C.c_double(-1.0)
        rc = mld.lib().mldg_relres_noalloc(h._h, C.byref(csr), C.c_void_p(x.data_ptr()),
                                           C.c_void_p(b.data_ptr()), C.byref(rr))
        assert rc == 0, mld.lib().mldg_last_error(h._h)
        # regular path: FCG with itmax = 0 returns the initial relative residual
        _, it, rr_ref = h.krylov("FCG", b, x=x.clone(), eps=0.0, itmax=0)
        assert it == 0
        assert abs(rr.value - rr_ref) <= TOL * rr_ref, (call, rr.value, rr_ref)
        bh = b.cpu().numpy()
        rr_np = np.linalg.norm(bh - a.to_scipy() @ xh) / np.linalg.norm(bh)
        assert abs(rr.value - rr_np) <= 1e-10 * rr_np


def test_noalloc_rejects_oversized_input(mld, orc):
    a = orc.gen_pde3d(6, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=50))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    big = mld.MLDG_NOALLOC_MAX_N + 1 if hasattr(mld, "MLDG_NOALLOC_MAX_N") else 524289
    dummy = (C.c_int32 * 1)()
    csr = mld._CSR(big, big, dummy, dummy, C.cast(dummy, C.POINTER(C.c_double)))
    rr = C.c_double(0.0)
    rc = mld.lib().mldg_relres_noalloc(h._h, C.byref(csr), C.c_void_p(1), C.c_void_p(1), C.byref(rr))
    assert rc == 36
    assert b"MLDG_NOALLOC_MAX_N" in mld.lib().mldg_last_error(h._h)
