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
    # the FP64 true-residual check is on by default for FP32 / BF16 inner
    # solves; the FP64 inner solve asks for it
    r = ks.solve(ctx, M, outer, b, inner=inner, E=1e-10, l=20, e=1e-30, r=21, R=30, inner_precision=prec,
                 true_residual=1 if prec == "fp64" else 0)
    assert r.converged, (r.status, r.loop)
    assert r.true_rel_res < 1e-10
    assert r.report["true_residual_checks"] >= 1
    err = np.linalg.norm(r.x - ref.x) / np.linalg.norm(ref.x)
    assert err < 1e-6


def test_failed_true_residual_check_restarts(ks, ctx):
    """VPGMRES stops on its Givens residual, which runs ahead of b - A x: with
    the check off it can stop above the eps; with it on it carries on until
    the FP64 true residual passes, and the history continues past the first
    stop."""
    A, b, _ = config_problem("varcoef3d", 20)
    M = ctx.matrix(A, transpose=True, fp32=True, bf16=True)
    kw = dict(E=1e-10, l=20, e=1e-30, R=30, inner_precision="fp32")
    off = ks.solve(ctx, M, "VPGMRES", b, inner="CG", true_residual=2, **kw)
    on = ks.solve(ctx, M, "VPGMRES", b, inner="CG", true_residual=1, **kw)
    assert off.report["true_residual_checks"] == 0
    assert on.converged and on.true_rel_res < 1e-10
    assert on.report["true_residual_checks"] >= 1
    if off.true_rel_res >= 1e-10:  # the check had to restart
        assert on.report["true_residual_checks"] >= 2 and on.loop > off.loop
    n = min(len(off.hist_err), len(on.hist_err))
    assert np.array_equal(off.hist_err[:n], on.hist_err[:n])  # same run up to the first stop


def test_x_rel_diff_in_report(ks, ctx):
    """params.x_ref: the report carries |x - x_ref| / |x_ref| against an FP64
    solution, as every mixed-precision result should."""
    A, b, _ = config_problem("varcoef3d", 16)
    M = ctx.matrix(A, fp32=True)
    B = ctx.vector(b)
    ref = ks.solve(ctx, M, "CG", B, E=1e-12)
    xr = ctx.vector(n=A.n)
    ks.solve(ctx, M, "CG", B, x=xr, E=1e-12)
    X = ctx.vector(n=A.n)
    r = ks.solve(ctx, M, "VPCG", B, inner="CG", x=X, E=1e-10, l=20, e=1e-30, inner_precision="fp32",
                 x_ref=xr.device_ptr)
    xm, x64 = X.numpy(), xr.numpy()
    want = np.linalg.norm(xm - x64) / np.linalg.norm(x64)
    assert r.report["x_rel_diff"] == pytest.approx(want, rel=1e-6)
    assert 0 < r.report["x_rel_diff"] < 1e-6
    assert ks.solve(ctx, M, "CG", B, x=X, E=1e-10).report["x_rel_diff"] == -1.0
    del ref


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
    A+ d = -2 h x-_c e_i, and L(x+) - L(x-) = d^T (x- + d/2 - x*).
    The gradient is the library's default path (BiCG: the on-chip kernel);
    the finite-difference solves use the kernel-per-step engine
    (cluster_solve 1). BiCG on the upwind system lets its residual grow
    about 1000-fold before it converges, and from there its trajectory
    depends on the rounding of its dot sums: with the on-chip kernel's order
    one of these 64 perturbed systems (entry 46693) stalls at a residual of
    O(1) for 40,000 iterations, where the engine's order converges in 2,174."""
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
        xm = ks.solve(ctx, Mm, solver, b, cluster_solve=1, **kw)
        Mm.close()
        rhs = np.zeros(A.n)
        rhs[i] = -2.0 * step * xm.x[c]
        Mp = ctx.matrix(CSR(A.ptr, A.col, vp), transpose=tr)
        d = ks.solve(ctx, Mp, solver, rhs, cluster_solve=1, **kw)
        Mp.close()
        assert xm.converged and d.converged
        fd = d.x @ (xm.x + 0.5 * d.x - xstar) / (2.0 * step)
        worst.append(abs(gv[j] - fd) / (abs(fd) + 1e-9 * np.max(np.abs(gv))))
    # b: x+ - x- = 2h A^{-1} e_i exactly, so the quotient is e_i^T A^{-T} (x - x*)
    for i in rng.choice(A.n, 8, replace=False):
        rhs = np.zeros(A.n)
        rhs[i] = 2e-6
        d = ks.solve(ctx, M, solver, rhs, cluster_solve=1, **kw)
        fd = d.x @ (fw.x - xstar) / 2e-6
        worst.append(abs(gb[i] - fd) / (abs(fd) + 1e-9 * np.max(np.abs(gb))))
    assert max(worst) <= 1e-6, f"largest relative deviation {max(worst):.3e}"


@pytest.mark.parametrize("prob,solver", [("varcoef2d", "CG"), ("convdiff2d", "BICG")])
def test_autograd_binding_gradcheck(ks, ctx, prob, solver):
    """The torch.autograd binding (forward solve, backward adjoint solve and
    pattern gather) passes torch.autograd.gradcheck on a 32 x 32 instance:
    its gradients with respect to b and every CSR value match central
    finite differences of the solve itself."""
    import torch

    from solver_cpp_b200.autograd import sparse_solve

    A, b, _ = config_problem(prob, 32)
    vals = torch.tensor(A.val, dtype=torch.float64, requires_grad=True)
    bt = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    w = torch.tensor(np.random.default_rng(6).standard_normal(A.n))

    def f(v, rhs):  # a scalar of x keeps gradcheck to one Jacobian row
        return (sparse_solve(ctx, A, v, rhs, solver, E=1e-12, L=20000) * w).sum()

    assert torch.autograd.gradcheck(f, (vals, bt), eps=1e-6, atol=1e-5, rtol=1e-4, fast_mode=True)


def test_vpcg_direction_ring_is_bitwise(ks, ctx):
    """160^3 VPCG with the on-chip FP32 inner CG defers x += alpha p to a ring
    of directions (its outer vectors do not fit in L2); x_update 1 keeps the
    update in the x/r pass. x is the same bits either way, and so are the
    history, the iteration count and the true residual."""
    A, b, _ = config_problem("varcoef3d", 160)
    M = ctx.matrix(A, fp32=True)
    kw = dict(E=1e-10, L=20000, l=20, e=1e-30, inner_precision="fp32")
    ring = ks.solve(ctx, M, "VPCG", b, inner="CG", **kw)
    flat = ks.solve(ctx, M, "VPCG", b, inner="CG", x_update=1, **kw)
    assert ring.status == flat.status == 0 and ring.loop == flat.loop
    assert np.array_equal(ring.hist_err, flat.hist_err)
    assert np.array_equal(ring.x, flat.x)
    assert ring.true_rel_res == flat.true_rel_res < 1e-10
