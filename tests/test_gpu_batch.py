"""Batching of independent systems: several hierarchies solved together.

mldg_krylov_batch launches every system's whole-solve graph (initial
residual, then a device-controlled loop of V-cycle and CG/FCG iteration) on
the system's own stream, once; the systems run concurrently to their own
convergence.  Every system runs exactly the graph of its own mldg_krylov, so
iterations and solutions must be identical to solving the systems one by one.
"""
import numpy as np
import pytest

from conftest import ANISO, ISO, oracle_params, upload_oracle_hierarchy

pytestmark = pytest.mark.gpu


def _systems(mld, orc, dims, precision=0, smoother="BJAC"):
    out = []
    for k, idim in enumerate(dims):
        a = orc.gen_pde3d(idim, 1, ISO if k % 2 == 0 else ANISO)
        op = orc.Prec(oracle_params(orc, smoother, 1 if smoother == "BJAC" else 2,
                                    1.0 if smoother == "BJAC" else 0.8, mcs=200))
        op.build(a)
        h = upload_oracle_hierarchy(mld, orc, op, precision=precision)
        b = np.random.default_rng(idim).uniform(-1, 1, a.nrows)
        out.append((a, h, b))
    return out


@pytest.mark.parametrize("precision,method,smoother", [(0, "FCG", "BJAC"), (1, "FCG", "BJAC"),
                                                       (0, "CG", "BJAC"), (0, "FCG", "JACOBI")])
def test_batch_equals_one_by_one(mld, orc, precision, method, smoother):
    sy = _systems(mld, orc, [10, 14, 20, 12, 17, 8], precision, smoother)
    hs = [h for _, h, _ in sy]
    bs = [b for _, _, b in sy]
    xs, its, rel, ms = mld.krylov_batch(method, hs, bs, eps=1e-10, itmax=300)
    assert ms > 0
    for (a, h, b), x, it, r in zip(sy, xs, its, rel):
        x1, it1, r1 = h.krylov(method, b.copy(), eps=1e-10, itmax=300)
        assert it == it1 and r == r1
        assert np.array_equal(x, x1)
        assert r <= 1e-10
        assert np.linalg.norm(b - orc.spmv(a, x)) <= 2e-10 * np.linalg.norm(b)


def test_batch_device_vectors_and_initial_guess(mld, orc):
    import torch
    sy = _systems(mld, orc, [16, 9, 13])
    hs = [h for _, h, _ in sy]
    bs = [torch.tensor(b, device="cuda") for _, _, b in sy]
    x0 = [torch.full_like(b, 0.5) for b in bs]
    xs, its, rel, _ = mld.krylov_batch("FCG", hs, bs, [x.clone() for x in x0], eps=1e-9)
    for (a, h, b), x, xi, it in zip(sy, xs, x0, its):
        x1, it1, _ = h.krylov("FCG", torch.tensor(b, device="cuda"), xi.clone(), eps=1e-9)
        assert it == it1
        assert torch.equal(x, x1)


def test_batch_errors(mld, orc):
    sy = _systems(mld, orc, [8, 10])
    hs = [h for _, h, _ in sy]
    bs = [b for _, _, b in sy]
    with pytest.raises(mld.MldError) as e:
        mld.krylov_batch("FCG", [hs[0], hs[0]], [bs[0], bs[0].copy()])
    assert e.value.code == 30
    # a zero right-hand side converges at iteration 0 and leaves x at zero
    xs, its, rel, _ = mld.krylov_batch("FCG", hs, [np.zeros_like(bs[0]), bs[1]])
    assert its[0] == 0 and np.all(xs[0] == 0.0) and its[1] > 0
    # itmax reached: the iterate comes back (the C ABI reports 4030)
    xs, its, rel, _ = mld.krylov_batch("FCG", hs, bs, eps=1e-15, itmax=2)
    assert np.all(its == 2)
