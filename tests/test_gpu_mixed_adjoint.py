"""GPU: mixed-precision VP solves and adjoint gradients.

The reference has neither (all FP64, no gradients), so these are pinned by
the FP64 path and by dense numpy: a VP solve with an FP32 / BF16 inner method
must reach the requested true FP64 relative residual and agree with the FP64
solution; adjoint gradients must match dense gradients and central finite
differences (h = 1e-6) to 1e-6 relative.
"""
import numpy as np
import pytest

from solver_cpp_b200.matrices import config_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("outer,inner,prec", [
    ("VPCG", "CG", "fp32"), ("VPCG", "CG", "bf16"), ("VPGMRES", "GMRES", "fp32"), ("VPGMRES", "CG", "fp32"),
    ("VPGCR", "CG", "fp32"), ("VPCG", "CG", "fp64"),
])
def test_mixed_vp_reaches_fp64_residual(ks, ctx, outer, inner, prec):
    A, b, _ = config_problem("varcoef3d", 20)
    M = ctx.matrix(A, transpose=True, fp32=True, bf16=True)
    ref = ks.solve(ctx, M, "CG", b, E=1e-12)
    r = ks.solve(ctx, M, outer, b, inner=inner, E=1e-10, l=20, e=1e-30, r=21, R=30, inner_precision=prec)
    assert r.converged, (r.status, r.loop)
    assert r.true_rel_res < 2e-10
    err = np.linalg.norm(r.x - ref.x) / np.linalg.norm(ref.x)
    assert err < 1e-6


def _dense_grad(A, b, xstar):
    D = A.to_scipy().toarray()
    x = np.linalg.solve(D, b)
    g = x - xstar
    lam = np.linalg.solve(D.T, g)
    rows = np.repeat(np.arange(A.n), np.diff(A.ptr))
    return x, lam, -lam[rows] * x[A.col]


def _loss(A, val, b, xstar):
    D = np.zeros((A.n, A.n))
    rows = np.repeat(np.arange(A.n), np.diff(A.ptr))
    D[rows, A.col] = val
    x = np.linalg.solve(D, b)
    return 0.5 * np.sum((x - xstar) ** 2)


@pytest.mark.parametrize("prob,solver", [("varcoef2d", "CG"), ("convdiff2d", "BICG"), ("convdiff2d", "GMRES")])
def test_adjoint_gradient_dense_and_fd(ks, ctx, prob, solver):
    A, b, _ = config_problem(prob, 32)
    xstar = np.random.default_rng(6).standard_normal(A.n)
    M = ctx.matrix(A, transpose=True)
    fw = ks.solve(ctx, M, solver, b, E=1e-13, R=60, L=20000)
    assert fw.converged
    X = ctx.vector(fw.x)
    G = ctx.vector(fw.x - xstar)
    GB, GV = ctx.vector(n=A.n), ctx.vector(n=A.nnz)
    st, rep = ks.adjoint_grad(ctx, M, solver, X, G, GB, GV, E=1e-13, R=60, L=20000)
    assert st == 0
    x_d, lam_d, gv_d = _dense_grad(A, b, xstar)
    gb, gv = GB.numpy(), GV.numpy()
    assert np.linalg.norm(gb - lam_d) / np.linalg.norm(lam_d) < 1e-9
    assert np.linalg.norm(gv - gv_d) / np.linalg.norm(gv_d) < 1e-9
    # central differences on 64 random CSR entries and 8 entries of b
    rng = np.random.default_rng(7)
    h = 1e-6
    for j in rng.choice(A.nnz, 64, replace=False):
        vp, vm = A.val.copy(), A.val.copy()
        step = h * max(1.0, abs(A.val[j]))
        vp[j] += step
        vm[j] -= step
        fd = (_loss(A, vp, b, xstar) - _loss(A, vm, b, xstar)) / (2 * step)
        assert abs(gv[j] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.max(np.abs(gv_d)))
    for i in rng.choice(A.n, 8, replace=False):
        bp, bm = b.copy(), b.copy()
        bp[i] += h
        bm[i] -= h
        fd = (_loss(A, A.val, bp, xstar) - _loss(A, A.val, bm, xstar)) / (2 * h)
        assert abs(gb[i] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.max(np.abs(lam_d)))


@pytest.mark.parametrize("prob,solver", [("varcoef2d", "CG"), ("convdiff2d", "BICG")])
def test_adjoint_gradient_fd_512(ks, ctx, prob, solver):
    """The 512^2 adjoint configuration: gradients with respect to 64 random
    CSR values (and 8 entries of b) against central finite differences with
    h = 1e-6 (relative to the entry), to 1e-6 relative. Each difference
    quotient is formed from the exact identity for the two perturbed
    solutions, so that it does not cancel in the loss (L ~ n/2): with
    A+- = A +- h e_i e_c^T and A- x- = b, the difference d = x+ - x- solves
    A+ d = -2 h x-_c e_i, and L(x+) - L(x-) = d^T (x- + d/2 - x*)."""
    from solver_cpp_b200.matrices import CSR

    A, b, _ = config_problem(prob, 512)
    xstar = np.random.default_rng(6).standard_normal(A.n)
    kw = dict(E=1e-14, L=40000)
    tr = solver == "BICG"
    M = ctx.matrix(A, transpose=True)
    fw = ks.solve(ctx, M, solver, b, **kw)
    assert fw.converged
    X = ctx.vector(fw.x)
    G = ctx.vector(fw.x - xstar)
    GB, GV = ctx.vector(n=A.n), ctx.vector(n=A.nnz)
    st, _ = ks.adjoint_grad(ctx, M, solver, X, G, GB, GV, **kw)
    assert st == 0
    gb, gv = GB.numpy(), GV.numpy()
    rows = np.repeat(np.arange(A.n), np.diff(A.ptr))
    rng = np.random.default_rng(7)
    worst = []
    for j in rng.choice(A.nnz, 64, replace=False):
        i, c = rows[j], A.col[j]
        step = 1e-6 * max(1.0, abs(A.val[j]))
        vm, vp = A.val.copy(), A.val.copy()
        vm[j] -= step
        vp[j] += step
        Mm = ctx.matrix(CSR(A.ptr, A.col, vm), transpose=tr)
        xm = ks.solve(ctx, Mm, solver, b, **kw)
        Mm.close()
        rhs = np.zeros(A.n)
        rhs[i] = -2.0 * step * xm.x[c]
        Mp = ctx.matrix(CSR(A.ptr, A.col, vp), transpose=tr)
        d = ks.solve(ctx, Mp, solver, rhs, **kw)
        Mp.close()
        assert xm.converged and d.converged
        fd = d.x @ (xm.x + 0.5 * d.x - xstar) / (2.0 * step)
        worst.append(abs(gv[j] - fd) / (abs(fd) + 1e-9 * np.max(np.abs(gv))))
    # b: x+ - x- = 2h A^{-1} e_i exactly, so the quotient is e_i^T A^{-T} (x - x*)
    for i in rng.choice(A.n, 8, replace=False):
        rhs = np.zeros(A.n)
        rhs[i] = 2e-6
        d = ks.solve(ctx, M, solver, rhs, **kw)
        fd = d.x @ (fw.x - xstar) / 2e-6
        worst.append(abs(gb[i] - fd) / (abs(fd) + 1e-9 * np.max(np.abs(gb))))
    assert max(worst) <= 1e-6, f"largest relative deviation {max(worst):.3e}"
