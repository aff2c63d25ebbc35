"""GPU: the FP16 operator form (MLDG_PREC_FP32_H16).

Every level's A, P, R and Jacobi off-diagonal part ND is stored as FP16
values with an FP32 row scale: rs_i = max_j |a_ij| rounded to FP32,
h_ij = a_ij / rs_i rounded to FP32 and then to FP16 (nearest even), and the
kernels form rs_i * sum_j h_ij x_j.  (A point-Jacobi level of at most two
sweeps stores ND with its columns scaled by the inverse diagonal, so there
the quantized matrix is ND D.)  Two bars:

* exactness of the form: the FP16 apply equals, to FP32 accuracy, the FP64
  apply of the same hierarchy whose A, P, R and ND were quantized that way
  on the host (numpy) -- so the quantization and the kernels that read it
  are what the form says, level by level (trans 'N'; the transposed
  operators are quantized by their own rows);
* effect on the method: the apply stays within TOL_H16 of the unquantized
  FP64 oracle apply, and FP64 FCG preconditioned by it reaches 1e-10 with at
  most 2 more iterations than with the FP64 V-cycle.
"""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu

TOL_EXACT = 2e-5  # FP32 arithmetic on identical operator values
TOL_H16 = 2e-2    # FP16 operator values against the unquantized FP64 apply


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def quantize_h16(m):
    """The FP16 row-scaled values of a CSR matrix, returned as FP64 values
    rs_i * h_ij (exact in FP64: a 24-bit by 11-bit significand product)."""
    irp = np.asarray(m.irp, dtype=np.int64)
    val = np.asarray(m.val, dtype=np.float64)
    n = len(irp) - 1
    rows = np.repeat(np.arange(n), np.diff(irp))
    mx = np.zeros(n)
    np.maximum.at(mx, rows, np.abs(val))
    s32 = mx.astype(np.float32)
    s32[mx == 0] = 1.0
    h = (val / s32.astype(np.float64)[rows]).astype(np.float32).astype(np.float16)
    return s32.astype(np.float64)[rows] * h.astype(np.float64)


def _upload(mld, orc, op, quantized, precision):
    h = mld.Hierarchy(use_graphs=True, autotune=True)
    for l in range(op.nlev):
        info = op.level_info(l)
        kind = info["smoother"]
        tri = kind in (orc.BJAC, orc.FBGS)

        def conv(m, q=True):
            if m is None:
                return None
            v = quantize_h16(m) if (quantized and q) else m.val
            return mld.CSR(m.irp, m.ja, v, ncols=m.ncols)

        d = op.level_vec(l, "d") if tri else op.level_vec(l, "dinv")

        def conv_nd(m):
            # a point-Jacobi level of at most two sweeps stores ND with its
            # columns scaled by d, and the FP16 form quantizes that product
            if m is None or not quantized or tri or info["sweeps_pre"] > 2:
                return conv(m)
            dc = np.asarray(d)[np.asarray(m.ja)]

            class S:
                irp, val = m.irp, np.asarray(m.val) * dc
            return mld.CSR(m.irp, m.ja, quantize_h16(S) / dc, ncols=m.ncols)

        h.upload_level(
            l, conv(op.level_csr(l, "A")),
            P=conv(op.level_csr(l, "P")) if l else None,
            R=conv(op.level_csr(l, "R")) if l else None,
            ND=conv_nd(op.level_csr(l, "ND")) if info["nnzND"] else None,
            L=conv(op.level_csr(l, "L"), False) if tri else None,
            U=conv(op.level_csr(l, "U"), False) if tri else None,
            d=d, smoother=kind, sweeps_pre=info["sweeps_pre"], sweeps_post=info["sweeps_pre"],
            damping=info["damp"])
    h.finalize(op.nlev, precision)
    return h


def test_quantizer_matches_definition():
    class M:
        irp = np.array([0, 3, 3, 5])
        val = np.array([3.0, -1.5, 1e-9, 0.1, 0.2])
    q = quantize_h16(M)
    assert q[0] == 3.0 and q[1] == -1.5
    assert q[2] == 0.0                                   # below FP16's range relative to the row max
    assert abs(q[3] - 0.1) <= 0.2 * 2.0 ** -11 and q[4] == np.float64(np.float32(0.2))


@pytest.mark.parametrize("smoother,sweeps,damp,coef,idim", [
    ("JACOBI", 2, 0.8, ANISO, 40), ("JACOBI", 2, 0.8, ISO, 32), ("BJAC", 1, 1.0, ISO, 28),
    ("FBGS", 1, 1.0, ANISO, 24)])
def test_h16_apply_equals_fp64_apply_of_quantized_hierarchy(mld, orc, smoother, sweeps, damp, coef, idim):
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, smoother, sweeps, damp, coarse_sweeps=4, mcs=300))
    op.build(a)
    assert op.nlev >= 3
    x = np.random.default_rng(idim).uniform(-1, 1, a.nrows)
    h16 = _upload(mld, orc, op, False, mld.PREC_FP32_H16)
    q64 = _upload(mld, orc, op, True, mld.PREC_FP64)
    y16, yq = h16.apply(x), q64.apply(x)
    assert _rel(y16, yq) <= TOL_EXACT, _rel(y16, yq)
    # and it is the FP16 form, not the FP32 one: far closer to the quantized
    # hierarchy's apply than to the unquantized one
    y_ref = op.apply(x)
    assert 5 * _rel(y16, yq) <= _rel(yq, y_ref), (_rel(y16, yq), _rel(yq, y_ref))
    assert _rel(y16, y_ref) <= TOL_H16, _rel(y16, y_ref)
    if smoother != "FBGS":  # Gauss-Seidel levels have no transposed apply
        assert _rel(h16.apply(x, trans="T"), op.apply(x, "T")) <= TOL_H16
    h16.close()
    q64.close()


@pytest.mark.parametrize("coef,idim", [(ANISO, 64), (ISO, 48)])
def test_h16_fcg_iterations(mld, orc, coef, idim):
    a = orc.gen_pde3d(idim, 1, coef)
    op = orc.Prec(oracle_params(orc, "JACOBI", 2, 0.8, coarse_sweeps=4, mcs=2000))
    op.build(a)
    b = np.random.default_rng(0).uniform(-1.0, 1.0, a.nrows)
    x_ref, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    h = upload_oracle_hierarchy(mld, orc, op, precision=mld.PREC_FP32_H16)
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert rr <= 1e-10
    assert it <= it_ref + 2, (it, it_ref)
    assert _rel(x, x_ref) < 1e-8, _rel(x, x_ref)
    h.close()
