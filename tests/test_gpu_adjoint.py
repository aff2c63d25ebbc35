"""GPU: the differentiation form (config 5 shapes).

-div(kappa grad u) = 1 on idim^3 cells, harmonic-mean faces, log kappa a
smooth Gaussian random field (correlation 0.1, variance 1).  Loss
L = 1/2 ||x - x_t||^2 with x_t the solution for a second field.  The
gradient is the adjoint one: A^T lambda = x - x_t solved by FCG with the
transposed V-cycle, then dL/dkappa by the scatter kernel; the forward
solution is recomputed in backward rather than stored.
"""
import numpy as np
import pytest

from conftest import oracle_params

pytestmark = pytest.mark.gpu

EPS = 1e-13  # tight solves: finite differences resolve ~1e-9 of L


def _prec(mld, a, dev_smoother="BJAC"):
    p = mld.MldPrec()
    p.init("ML")
    p.set("SMOOTHER_TYPE", dev_smoother)
    p.set("COARSE_SOLVE", "BJAC")
    p.set("COARSE_SUBSOLVE", "ILU")
    p.set("COARSE_SWEEPS", 4)
    p.set("MIN_COARSE_SIZE", 200)
    p.build(a)
    return p


def _solve(mld, idim, kappa):
    a = mld.gen_kappa3d(idim, kappa)
    p = _prec(mld, a)
    x, it, rr = mld.krylov("FCG", a, p, np.ones(a.nrows), eps=EPS, itmax=1000, use_prec_matrix=True)
    assert rr <= 10 * EPS
    return a, p, x


def _autograd_fn(mld, idim):
    import torch

    class SolveKappa(torch.autograd.Function):
        @staticmethod
        def forward(ctx, kappa):
            k = kappa.detach().cpu().numpy().astype(np.float64)
            _, _, x = _solve(mld, idim, k)
            ctx.save_for_backward(kappa)
            return torch.from_numpy(x)

        @staticmethod
        def backward(ctx, gx):
            (kappa,) = ctx.saved_tensors
            k = kappa.detach().cpu().numpy().astype(np.float64)
            a, p, x = _solve(mld, idim, k)           # forward solution recomputed
            lam, it, rr = p.adjoint(gx.detach().cpu().numpy().astype(np.float64), eps=EPS,
                                    itmax=1000)
            assert rr <= 10 * EPS
            g = p.kappa_grad(idim, k, x, lam)
            return torch.from_numpy(g)

    return SolveKappa.apply


def _loss_and_grad(mld, idim, kappa, xt):
    import torch
    kt = torch.tensor(kappa, dtype=torch.float64, requires_grad=True)
    x = _autograd_fn(mld, idim)(kt)
    loss = 0.5 * torch.sum((x - torch.from_numpy(xt)) ** 2)
    loss.backward()
    return float(loss.detach()), kt.grad.numpy()


def _loss(mld, idim, kappa, xt):
    _, _, x = _solve(mld, idim, kappa)
    return 0.5 * float(np.sum((x - xt) ** 2))


def grad_reference(idim, kappa, x, lam):
    """Independent numpy restatement of the chain rule (CPU reference gradient)."""
    h = 1.0 / (idim + 1)
    K = kappa.reshape(idim, idim, idim)
    X = x.reshape(idim, idim, idim)
    Lm = lam.reshape(idim, idim, idim)
    g = np.zeros_like(K)
    for ax in range(3):
        for sgn in (-1, 1):
            Ks = np.roll(K, -sgn, axis=ax)
            Xs = np.roll(X, -sgn, axis=ax)
            Ls = np.roll(Lm, -sgn, axis=ax)
            inside = np.ones_like(K, dtype=bool)
            idx = [slice(None)] * 3
            idx[ax] = (idim - 1) if sgn == 1 else 0
            inside[tuple(idx)] = False
            term = np.where(inside, 2 * Ks ** 2 / (K + Ks) ** 2 * (Lm - Ls) * (X - Xs), Lm * X)
            g += term
    return (-g / h ** 2).reshape(-1)


def test_adjoint_solve_transposed_vcycle(mld):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    idim = 14
    kappa = np.exp(mld.grf3d(idim, seed=2))
    a = mld.gen_kappa3d(idim, kappa)
    p = _prec(mld, a)
    g = np.random.default_rng(4).uniform(-1, 1, a.nrows)
    lam, it, rr = p.adjoint(g, eps=1e-11)
    assert rr <= 1e-11 and it > 0
    A = sp.csr_matrix((a.val, a.ja, a.irp))
    ref = spla.spsolve(A.T.tocsc(), g)
    assert np.linalg.norm(lam - ref) / np.linalg.norm(ref) < 1e-8


def test_gradient_matches_cpu_reference(mld, orc):
    """GPU adjoint gradient vs the CPU reference: oracle solves + numpy chain rule."""
    idim = 12
    kappa = np.exp(mld.grf3d(idim, seed=2))
    xt = _solve(mld, idim, np.exp(mld.grf3d(idim, seed=3)))[2]
    a = mld.gen_kappa3d(idim, kappa)
    ao = orc.CSR(a.irp, a.ja, a.val)
    op = orc.Prec(oracle_params(orc, "BJAC", mcs=200))
    op.build(ao)
    x_cpu, _, _, _ = orc.krylov("FCG", ao, op, np.ones(a.nrows), eps=EPS, itmax=1000)
    # A is symmetric, so A^T lambda = x - xt is the same system
    lam_cpu, _, _, _ = orc.krylov("FCG", ao, op, x_cpu - xt, eps=EPS, itmax=1000)
    g_cpu = grad_reference(idim, kappa, x_cpu, lam_cpu)
    _, g_gpu = _loss_and_grad(mld, idim, kappa, xt)
    assert np.linalg.norm(g_gpu - g_cpu) / np.linalg.norm(g_cpu) < 1e-9


def test_gradient_matches_finite_differences(mld):
    idim = 10
    kappa = np.exp(mld.grf3d(idim, seed=2))
    xt = _solve(mld, idim, np.exp(mld.grf3d(idim, seed=3)))[2]
    _, grad = _loss_and_grad(mld, idim, kappa, xt)
    rng = np.random.default_rng(5)
    cells = rng.choice(kappa.size, 20, replace=False)
    for c in cells:
        d = 1e-4 * kappa[c]
        kp, km = kappa.copy(), kappa.copy()
        kp[c] += d
        km[c] -= d
        fd = (_loss(mld, idim, kp, xt) - _loss(mld, idim, km, xt)) / (2 * d)
        assert abs(fd - grad[c]) <= 1e-6 * max(abs(grad[c]), 1e-3 * np.abs(grad).max()), (c, fd, grad[c])


def test_directional_derivative_full_size(mld):
    """idim=96 (884,736 cells): <grad, v> against a central difference along v."""
    idim = 96
    kappa = np.exp(mld.grf3d(idim, seed=2))
    xt = _solve(mld, idim, np.exp(mld.grf3d(idim, seed=3)))[2]
    _, grad = _loss_and_grad(mld, idim, kappa, xt)
    v = np.random.default_rng(6).uniform(-1, 1, kappa.size) * kappa
    t = 1e-5
    fd = (_loss(mld, idim, kappa + t * v, xt) - _loss(mld, idim, kappa - t * v, xt)) / (2 * t)
    assert abs(fd - grad @ v) <= 1e-6 * abs(fd)
