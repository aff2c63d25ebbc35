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


@pytest.mark.parametrize("prec", [0, 1, 3])
@pytest.mark.parametrize("method", ["CG", "FCG"])
def test_graph_solve_equals_host_stepped_solve(mld, orc, method, prec):
    """A solve without a probe is one graph launch (device-side stopping
    test in a conditional WHILE node); with a probe set, the same kernels run
    with one host check per iteration.  Both must give the same bits -- also
    with an FP32 V-cycle (prec 1, 3), whose graph solve reads the V-cycle's
    FP32 output and writes its FP32 input inside the Krylov kernels, while
    the host-stepped solve casts at the V-cycle's ends."""
    a = orc.gen_pde3d(20, 1, ISO)
    op = orc.Prec(oracle_params(orc, "JACOBI", 2, 0.8, mcs=300))
    op.build(a)
    b = np.random.default_rng(5).uniform(-1, 1, a.nrows)
    h = upload_oracle_hierarchy(mld, orc, op, precision=prec)
    x1, it1, r1 = h.krylov(method, b.copy(), eps=1e-10)
    _, nl1 = h.last_timing()
    h.probe_set(mld.KERNEL_SPMV, 0, 0)  # forces the host-stepped loop
    x2, it2, r2 = h.krylov(method, b.copy(), eps=1e-10)
    h.probe_set(0, 0, 0)
    x3, it3, r3 = h.krylov(method, b.copy(), eps=1e-10)  # graph again
    assert it1 == it2 == it3 and r1 == r2 == r3
    assert np.array_equal(x1, x2) and np.array_equal(x1, x3)
    assert r1 <= 1e-10 and nl1 > it1


def test_itmax_and_zero_rhs(mld, orc):
    """itmax stops the device loop exactly; a zero right-hand side or an
    exact initial guess stops before the first iteration."""
    a = orc.gen_pde3d(12, 1, ISO)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=200))
    op.build(a)
    h = upload_oracle_hierarchy(mld, orc, op)
    b = orc.spmv(a, np.ones(a.nrows))
    _, it, rr = h.krylov("FCG", b.copy(), eps=1e-14, itmax=3)
    _, it_ref, rr_ref, _ = orc.krylov("FCG", a, op, b, eps=1e-14, itmax=3)
    assert it == 3 and it_ref == 3 and rr > 1e-14
    assert abs(rr - rr_ref) <= 1e-6 * rr_ref
    x, it, rr = h.krylov("FCG", np.zeros(a.nrows), eps=1e-10)
    assert it == 0 and np.all(x == 0)
    x, it, rr = h.krylov("FCG", b.copy(), x=np.ones(a.nrows), eps=1e-10)
    assert it == 0 and rr <= 1e-10
