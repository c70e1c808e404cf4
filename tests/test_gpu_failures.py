"""GPU: the failure statuses, each made without faulting the GPU.

* KS_BREAKDOWN: a Krylov denominator that is exactly zero. The reference
  divides regardless (cg.cpp:218 alpha = rr / (p, Ap); kskipcg.cpp:268-271;
  gmres.cpp:384-399) and iterates on inf / NaN until maxloop; the library
  stops at once. Crafted systems: a skew-symmetric A has (p, A p) = 0 for every
  p, so CG's first alpha divides by zero.
* KS_TIMEOUT: the kernels' bounded waits (the CSR SpMV's shared-memory
  staging barriers) get a limit of 1 ns (ks_ctx_set_wait_limit), so a wait
  gives up; the kernel drains its own copies in flight under the default limit
  and finishes, the call returns KS_TIMEOUT, and the context keeps working.
* KS_NAN_DETECTED: b = 0 makes the stopping test 0/0.
"""
import numpy as np
import pytest

from solver_cpp_b200.matrices import CSR, config_problem

pytestmark = pytest.mark.gpu


def _skew(n):
    """Tridiagonal skew-symmetric matrix: A[i][i+1] = 1, A[i+1][i] = -1."""
    ptr, col, val = [0], [], []
    for i in range(n):
        if i > 0:
            col.append(i - 1)
            val.append(-1.0)
        if i < n - 1:
            col.append(i + 1)
            val.append(1.0)
        ptr.append(len(col))
    return CSR(np.array(ptr, np.int32), np.array(col, np.int32), np.array(val))


@pytest.mark.parametrize("n", [2, 3, 8])
@pytest.mark.parametrize("cluster_solve", [0, 1])
def test_cg_breakdown_on_skew_symmetric_system(ks, ctx, n, cluster_solve):
    """(p, A p) sums p_i p_{i+1} - p_{i+1} p_i pairs; on a few rows every term
    is exact and the sum is 0 in any order (larger systems leave a rounding
    residue, and the method then runs on). cluster_solve 0: one cluster
    launch; 1: the kernel-per-step engine."""
    A = _skew(n)
    b = np.random.default_rng(3).standard_normal(n)
    M = ctx.matrix(A, transpose=True)
    r = ks.solve(ctx, M, "CG", b, E=1e-10, L=100, cluster_solve=cluster_solve)
    assert r.status == 3, r.status  # KS_BREAKDOWN
    assert r.loop <= 2


def test_cr_and_bicg_breakdown(ks, ctx):
    """Skew-symmetric A, r = b: BiCG's first alpha is (r, r) / (r, A r) = x / 0
    (bicg.cpp:237); CR's first rs = (r, A r) is 0, so alpha = 0 and the
    next beta = (r, A r) / rs = 0 / 0 (cr.cpp:225,253). Both stop with
    KS_BREAKDOWN at once, on the cluster-resident path and on the engine."""
    A = _skew(64)
    b = np.random.default_rng(4).standard_normal(64)
    M = ctx.matrix(A, transpose=True)
    for name in ("CR", "BICG"):
        for cs in (0, 1):
            r = ks.solve(ctx, M, name, b, E=1e-10, L=100, cluster_solve=cs)
            assert r.status == 3, (name, cs, r.status)
            assert r.loop <= 3, (name, cs, r.loop)


def test_bounded_wait_runs_out_and_context_survives(ks, ctx):
    A, _, _ = config_problem("poisson3d", 64)
    M = ctx.matrix(A, diag=False)  # CSR: the TMA-staged SpMV with mbarrier waits
    x = np.random.default_rng(5).standard_normal(A.n)
    X, Y = ctx.vector(x), ctx.vector(n=A.n)
    ks.spmv(M, X, Y)
    want = Y.numpy()
    ctx.set_wait_limit(1)
    try:
        ks.spmv(M, X, Y)  # asynchronous: the timeout shows at the next synchronisation
        with pytest.raises(ks.KrylovError) as e:
            ctx.synchronize()
        assert e.value.status == 7  # KS_TIMEOUT
    finally:
        ctx.set_wait_limit(0)
    ctx.synchronize()  # the flag was reported once and cleared
    Y.fill(0.0)
    ks.spmv(M, X, Y)
    assert np.array_equal(Y.numpy(), want)
    r = ks.solve(ctx, M, "CG", np.ones(A.n), E=1e-8)
    assert r.converged


def test_zero_rhs_is_nan_detected(ks, ctx):
    A, _, _ = config_problem("poisson2d", 16)
    M = ctx.matrix(A)
    r = ks.solve(ctx, M, "CG", np.zeros(A.n), E=1e-10, cluster_solve=1)
    assert r.status == 4


@pytest.mark.parametrize("case", ["cg", "cr", "bicg", "vpcg"])
def test_on_chip_wait_runs_out_and_context_survives(ks, ctx, case):
    """The cooperative on-chip kernels (whole CG / CR / BiCG solves, the VP
    methods' FP32 inner CG) bound every grid reduction and publication wait
    by the context's wait limit. With a limit of 1 ns the waits give up: the
    kernel sets the timeout flag, releases its TMEM columns and returns, the
    solve reports KS_TIMEOUT, and the context keeps working (the same solve
    converges once the limit is back)."""
    prob, g, method, kw = {
        "cg": ("poisson3d", 40, "CG", {}),
        "cr": ("poisson3d", 40, "CR", {}),
        "bicg": ("convdiff2d", 200, "BICG", {}),
        "vpcg": ("varcoef3d", 24, "VPCG", dict(inner="CG", l=20, e=1e-30, inner_precision="fp32")),
    }[case]
    A, b, _ = config_problem(prob, g)
    M = ctx.matrix(A, transpose=True, fp32=True)
    ctx.set_wait_limit(1)
    try:
        with pytest.raises(ks.KrylovError) as e:
            ks.solve(ctx, M, method, b, E=1e-10, L=5, **kw)
        assert e.value.status == 7  # KS_TIMEOUT
    finally:
        ctx.set_wait_limit(0)
    ctx.synchronize()
    r = ks.solve(ctx, M, method, b, E=1e-10, L=20000, **kw)
    assert r.converged and r.true_rel_res < 1e-9, (r.status, r.true_rel_res)
