"""GPU FCG/CG against the oracle's Krylov solves (iteration counts within 1)."""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,eps", [("CG", 1e-9), ("FCG", 1e-10)])
@pytest.mark.parametrize("smoother,sweeps,damp", [("BJAC", 1, 1.0), ("JACOBI", 2, 0.8)])
def test_krylov_iterations_match(mld, orc, method, eps, smoother, sweeps, damp):
    a = orc.gen_pde3d(24, 1, ISO)
    op = orc.Prec(oracle_params(orc, smoother, sweeps, damp, mcs=400))
    op.build(a)
    b = orc.spmv(a, np.ones(a.nrows))
    x_ref, it_ref, rr_ref, _ = orc.krylov(method, a, op, b, eps=eps)
    h = upload_oracle_hierarchy(mld, orc, op)
    x, it, rr = h.krylov(method, b.copy(), eps=eps)
    assert abs(it - it_ref) <= 1, (it, it_ref)
    assert rr <= eps
    assert np.linalg.norm(x - 1) / np.sqrt(a.nrows) < 1e-6


def test_fileread_fixture_solution(mld, orc):
    """The reference's recorded fixture: solve to the recorded solution."""
    import os
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "fileread_fixture.npz"))
    a = orc.CSR(f["irp"], f["ja"], f["val"])
    op = orc.Prec(oracle_params(orc, "BJAC", coarse_sweeps=1, mcs=-1))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    x, it, rr = h.krylov("CG", f["rhs"].copy(), eps=1e-12)
    assert rr <= 1e-12
    assert np.linalg.norm(x - f["sol"]) / np.linalg.norm(f["sol"]) < 1e-9


def test_fp32_vcycle_inside_fp64_fcg(mld, orc):
    a = orc.gen_pde3d(24, 1, ANISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=400))
    op.build(a)
    rng = np.random.default_rng(0)
    b = rng.uniform(-1, 1, a.nrows)
    x_ref, it_ref, _, _ = orc.krylov("FCG", a, op, b, eps=1e-10)
    h = upload_oracle_hierarchy(mld, orc, op, precision=mld.PREC_FP32)
    x, it, rr = h.krylov("FCG", b.copy(), eps=1e-10)
    assert rr <= 1e-10
    assert it <= it_ref + 2
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-8
