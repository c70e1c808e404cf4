"""GPU: the diagonal copy of stencil matrices.

A matrix whose rows hold their columns at no more than 8 distinct offsets
from the row, in increasing column order, with the diagonals at least 3/4
full, keeps a diagonal copy that the SpMV reads instead of CSR (no column
indices). A row summed diagonal by diagonal is summed in its CSR order, so
the SpMV must equal the reference's (the oracle's) bit for bit in FP64, equal
the CSR kernel's bit for bit in FP32 and BF16, and every method must give the
same history and solution bit for bit on either layout. Matrices that do not
qualify keep CSR only and give the oracle's SpMV.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from solver_cpp_b200.matrices import CSR, config_problem

pytestmark = pytest.mark.gpu

# offsets that are multiples of 4 take the SpMV's quad path (4 rows per
# thread); 37^2 (odd n, offsets +-37) the row path
STENCILS = [("poisson2d", 40, 5), ("poisson3d", 12, 7), ("convdiff3d", 12, 7), ("varcoef3d", 12, 7),
            ("varcoef2d", 40, 5), ("convdiff2d", 40, 5), ("convdiff2d", 37, 5), ("varcoef3d", 20, 7)]


def _csr(M):
    M = sp.csr_matrix(M)
    M.sort_indices()
    return CSR(M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data.astype(np.float64))


@pytest.mark.parametrize("prob,g,nd", STENCILS)
def test_stencils_get_a_diagonal_copy(ks, ctx, prob, g, nd):
    A, _, _ = config_problem(prob, g)
    info = ctx.matrix(A, transpose=True).info()
    assert info["diagonals"] == nd and info["t_diagonals"] == nd
    assert ctx.matrix(A, transpose=True, diag=False).info()["diagonals"] == 0


@pytest.mark.parametrize("prob,g,nd", STENCILS)
def test_diagonal_spmv_is_bitwise(ks, ctx, oracle, prob, g, nd):
    A, _, _ = config_problem(prob, g)
    P = oracle.Problem(A)
    x = np.random.default_rng(11).standard_normal(A.n)
    D = ctx.matrix(A, transpose=True, fp32=True, bf16=True)
    S = ctx.matrix(A, transpose=True, fp32=True, bf16=True, diag=False)
    X, Y = ctx.vector(x), ctx.vector(n=A.n)
    for trans in (False, True):
        ks.spmv(D, X, Y, trans=trans)
        assert np.array_equal(Y.numpy(), oracle.spmv(P, x, transpose=trans))
    X32 = ctx.vector(x.astype(np.float32), dtype=ks.FP32)
    Yd, Ys = ctx.vector(n=A.n, dtype=ks.FP32), ctx.vector(n=A.n, dtype=ks.FP32)
    for vals in (ks.FP32, ks.BF16):
        ks.spmv(D, X32, Yd, values=vals)
        ks.spmv(S, X32, Ys, values=vals)
        assert np.array_equal(Yd.numpy(), Ys.numpy()), vals


def _nine_point(g):
    T = sp.diags([-1.0, 2.5, -1.0], [-1, 0, 1], shape=(g, g))
    return sp.kron(T, T) + sp.identity(g * g)  # 9 diagonals


def _unsorted(A):
    """Same matrix with the first two entries of every row of >= 2 entries swapped."""
    col, val = A.col.copy(), A.val.copy()
    for i in range(A.n):
        j = A.ptr[i]
        if A.ptr[i + 1] - j >= 2:
            col[j], col[j + 1] = col[j + 1], col[j]
            val[j], val[j + 1] = val[j + 1], val[j]
    return CSR(A.ptr.copy(), col, val)


def _sparse_far_diagonal(n):
    M = sp.lil_matrix((n, n))
    M.setdiag(4.0)
    for i in range(0, n - 700, 97):  # a few entries far off the diagonal: two diagonals, half empty
        M[i, i + 700] = -1.0
    return M.tocsr()


@pytest.mark.parametrize("case", ["nine_point", "unsorted", "random", "half_empty"])
def test_non_stencils_keep_csr(ks, ctx, oracle, case):
    if case == "nine_point":
        A = _csr(_nine_point(30))
    elif case == "unsorted":
        A = _unsorted(config_problem("poisson2d", 30)[0])
    elif case == "random":
        rng = np.random.default_rng(4)
        R = sp.random(900, 900, density=0.01, random_state=rng, format="csr") + 10 * sp.identity(900)
        A = _csr(R)
    else:
        A = _csr(_sparse_far_diagonal(2000))
    M = ctx.matrix(A)
    assert M.info()["diagonals"] == 0
    x = np.random.default_rng(5).standard_normal(A.n)
    X, Y = ctx.vector(x), ctx.vector(n=A.n)
    ks.spmv(M, X, Y)
    assert np.array_equal(Y.numpy(), oracle.spmv(oracle.Problem(A), x))


SOLVES = [
    ("poisson3d", "CG", "NONE", {"cluster_solve": 1}),
    ("poisson3d", "CR", "NONE", {}),
    ("convdiff3d", "BICG", "NONE", {}),
    ("convdiff3d", "GMRES", "NONE", {"R": 10}),
    ("convdiff3d", "GCR", "NONE", {"R": 5}),
    ("poisson3d", "KSKIPCG", "NONE", {"K": 2}),
    ("convdiff3d", "KSKIPBICG", "NONE", {"K": 2}),
    ("varcoef3d", "VPCG", "CG", {"l": 20, "e": 1e-30, "inner_precision": "fp32"}),
    ("varcoef3d", "VPCG", "CG", {"l": 20, "e": 1e-30, "inner_precision": "bf16"}),
    ("varcoef3d", "VPGMRES", "CG", {"R": 20, "l": 10, "e": 1e-30, "inner_precision": "fp32"}),
]


@pytest.mark.parametrize("prob,outer,inner,kw", SOLVES)
def test_solves_identical_on_both_layouts(ks, ctx, prob, outer, inner, kw):
    """inner_fast=1: both layouts run the inner solves kernel by kernel (the
    on-chip inner CG needs the diagonal copy; it is compared below)."""
    A, b, _ = config_problem(prob, 16)
    res = []
    for diag in (True, False):
        M = ctx.matrix(A, transpose=True, fp32=True, bf16=True, diag=diag)
        assert (M.info()["diagonals"] > 0) == diag
        res.append(ks.solve(ctx, M, outer, b, inner=inner, E=1e-10, L=3000, inner_fast=1, **kw))
    d, c = res
    assert d.status == c.status and d.loop == c.loop
    assert np.array_equal(d.hist_err, c.hist_err) and np.array_equal(d.x, c.x)


SYMMETRIC = [("poisson2d", 40, True), ("poisson3d", 12, True), ("varcoef3d", 12, True), ("varcoef2d", 40, True),
             ("convdiff3d", 12, False), ("convdiff2d", 40, False)]


@pytest.mark.parametrize("prob,g,sym", SYMMETRIC)
def test_symmetric_matrices_keep_half_the_diagonals(ks, ctx, oracle, prob, g, sym):
    """A matrix equal to its transpose bit for bit keeps only its main and
    upper diagonals; its SpMV (lower terms read from the upper mirror) is
    still the reference's bit for bit, and so is A^T's."""
    A, _, _ = config_problem(prob, g)
    M = ctx.matrix(A, transpose=True, fp32=True, bf16=True)
    assert M.info()["dia_symmetric"] == (1 if sym else 0)
    assert M.info()["t_dia_symmetric"] == (1 if sym else 0)
    P = oracle.Problem(A)
    x = np.random.default_rng(12).standard_normal(A.n)
    X, Y = ctx.vector(x), ctx.vector(n=A.n)
    for trans in (False, True):
        ks.spmv(M, X, Y, trans=trans)
        assert np.array_equal(Y.numpy(), oracle.spmv(P, x, transpose=trans))


def test_almost_symmetric_matrix_keeps_every_diagonal(ks, ctx, oracle):
    """One value off by one ulp: not symmetric, all 7 diagonals kept, SpMV exact."""
    A, _, _ = config_problem("varcoef3d", 12)
    val = A.val.copy()
    j = int(A.ptr[500])  # the first (lowest) entry of row 500
    val[j] = np.nextafter(val[j], np.inf)
    B = CSR(A.ptr, A.col, val)
    M = ctx.matrix(B, fp32=True)
    assert M.info()["diagonals"] == 7 and M.info()["dia_symmetric"] == 0
    x = np.random.default_rng(13).standard_normal(B.n)
    X, Y = ctx.vector(x), ctx.vector(n=B.n)
    ks.spmv(M, X, Y)
    assert np.array_equal(Y.numpy(), oracle.spmv(oracle.Problem(B), x))


@pytest.mark.parametrize("grid", [16, 18, 28])  # 18: offsets 18, 324 take the generic quad path
@pytest.mark.parametrize("outer,inner,prec,kw", [
    ("VPCG", "CG", "fp32", {}), ("VPCG", "CG", "bf16", {}), ("VPGMRES", "CG", "fp32", {"R": 20, "l": 10}),
    ("VPGCR", "CG", "fp32", {"R": 20, "l": 10}), ("VPCR", "CG", "fp32", {"L": 40}),
])
def test_on_chip_inner_cg_matches_kernel_per_step(ks, ctx, grid, outer, inner, prec, kw):
    """The inner CG as one cooperative kernel with its vectors on chip applies
    the kernel-per-step loop's FP32 operations to every element; its inner dot
    products add exact FP64 products of FP32 values in another order, so the
    two agree to rounding of the sums: the same verdict and iteration count
    (within 2 %), histories and solutions within 1e-6."""
    A, b, _ = config_problem("varcoef3d", grid)
    M = ctx.matrix(A, transpose=True, fp32=True, bf16=True)
    p = dict(E=1e-10, L=3000, l=20, e=1e-30, inner_precision=prec, true_residual=2)
    p.update(kw)
    chip = ks.solve(ctx, M, outer, b, inner=inner, inner_fast=0, **p)
    step = ks.solve(ctx, M, outer, b, inner=inner, inner_fast=1, **p)
    assert chip.status == step.status
    assert abs(chip.loop - step.loop) <= max(1, 0.02 * step.loop)
    m = min(len(chip.hist_err), len(step.hist_err), 30)
    assert np.allclose(chip.hist_err[:m], step.hist_err[:m], rtol=1e-6, atol=0)
    if step.status == 0:
        assert np.linalg.norm(chip.x - step.x) <= 1e-6 * np.linalg.norm(step.x)


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_on_chip_inner_cg_several_quads_per_thread(ks, ctx, prec):
    """96^3 (884,736 rows, 5,984 per CTA): every thread owns two quads of
    rows, so the on-chip kernel's passes span all 32 warps and its solution
    write-out reads rows other warps updated last. Two solves give the same
    bits, and they equal the kernel-per-step inner path's history and
    solution bit for bit (alpha and beta are rounded to FP32, which absorbs
    the different order of the FP64 dot sums)."""
    A, b, _ = config_problem("varcoef3d", 96)
    M = ctx.matrix(A, fp32=True, bf16=True)
    p = dict(E=1e-10, L=2000, l=20, e=1e-30, inner_precision=prec, true_residual=2)
    c1 = ks.solve(ctx, M, "VPCG", b, inner="CG", inner_fast=0, **p)
    c2 = ks.solve(ctx, M, "VPCG", b, inner="CG", inner_fast=0, **p)
    step = ks.solve(ctx, M, "VPCG", b, inner="CG", inner_fast=1, **p)
    assert c1.status == 0 and c1.true_rel_res <= 1e-10
    assert np.array_equal(c1.x, c2.x) and np.array_equal(c1.hist_err, c2.hist_err)
    assert c1.loop == step.loop
    assert np.array_equal(c1.hist_err, step.hist_err)
    assert np.array_equal(c1.x, step.x)


@pytest.mark.parametrize("prob,g,xu", [("convdiff3d", 120, 0), ("convdiff3d", 128, 0), ("convdiff3d", 128, 1)])
def test_bicg_pair_spmv_against_two_spmvs(ks, ctx, prob, g, xu):
    """Above 2^20 rows, with a diagonal copy larger than 60 % of L2 (120^3:
    97 MB, 128^3: 117 MB), BiCG computes q = A p and A^T p* in one pass over A's
    diagonal copy (A^T's diagonals read as A's, mirrored; q and A^T p* are
    the bits of the separate SpMVs) and updates r and r* (and x, with
    x_update 1; else x is deferred to the direction ring) in one pass, whose
    (r*, r) sum adds its terms in another order. A one-rank split solve over
    the in-process transport still runs the two separate SpMVs: the same
    verdict, iteration counts within 10 %, solutions within 1e-6 (the upwind
    residual first grows several-fold, which magnifies the last-bit
    differences of (r*, r) in the histories to ~1e-6)."""
    A, b, _ = config_problem(prob, g)
    assert A.n > 1 << 20
    M = ctx.matrix(A, transpose=True)
    assert M.info()["diagonals"] in (5, 7) and M.info()["dia_symmetric"] == 0
    pair = ks.solve(ctx, M, "BICG", b, E=1e-10, L=6000, x_update=xu)
    c = ks.Context(0)
    comm = ks.Comm.local([c])[0]
    try:
        S = ks.SplitMatrix(c, comm, A, 0, A.n, transpose=True)
        two = ks.solve(c, S, "BICG", b, E=1e-10, L=6000, x_update=xu)
        S.close()
    finally:
        comm.close()
        c.close()
    assert pair.status == two.status == 0
    # BiCG's iteration count moves with the order of the (r*, r) sums: 120^3
    # takes 517 iterations this way and 490 with the A^T SpMV's order (128^3:
    # 502 both, the reference's count)
    assert abs(pair.loop - two.loop) <= max(2, 0.10 * two.loop)
    assert np.array_equal(pair.hist_err[:2], two.hist_err[:2])  # before the first (r*, r) sum differs
    assert np.linalg.norm(pair.x - two.x) <= 1e-6 * np.linalg.norm(two.x)
    # BiCG's recurrence residual can drift from b - A x (upwind systems):
    # within ten times the two-SpMV solve's own
    assert pair.true_rel_res <= 10 * two.true_rel_res + 1e-12


def test_kskip_bicg_pair_spmv_is_bitwise(ks, ctx):
    """k-skip BiCG's inner steps take A p and r* -= a A^T p* from one pass
    over A's diagonal copy above 2^20 rows with a copy larger than 60 % of
    L2; the epilogue has no sums, so the solve equals the one-rank split
    solve (two separate SpMVs) bit for bit."""
    A, b, _ = config_problem("convdiff3d", 128)
    M = ctx.matrix(A, transpose=True)
    pair = ks.solve(ctx, M, "KSKIPBICG", b, E=1e-10, L=3000, K=2)
    c = ks.Context(0)
    comm = ks.Comm.local([c])[0]
    try:
        S = ks.SplitMatrix(c, comm, A, 0, A.n, transpose=True)
        two = ks.solve(c, S, "KSKIPBICG", b, E=1e-10, L=3000, K=2)
        S.close()
    finally:
        comm.close()
        c.close()
    assert pair.status == two.status == 0
    assert pair.loop == two.loop
    assert np.array_equal(pair.hist_err, two.hist_err) and np.array_equal(pair.x, two.x)


def test_bicg_pair_spmv_on_the_transposed_system(ks, ctx):
    """A transposed solve (A^T x = b, as the adjoint solve runs it) takes the
    pair path with the roles of the two copies swapped: it must converge to
    the same solution as the two-SpMV path (one-rank split) and reach b - A^T x
    to the tolerance, with iteration counts within 10 %."""
    A, b, _ = config_problem("convdiff3d", 128)
    M = ctx.matrix(A, transpose=True)
    kw = dict(E=1e-10, L=6000, transpose=1)
    pair = ks.solve(ctx, M, "BICG", b, **kw)
    c = ks.Context(0)
    comm = ks.Comm.local([c])[0]
    try:
        S = ks.SplitMatrix(c, comm, A, 0, A.n, transpose=True)
        two = ks.solve(c, S, "BICG", b, **kw)
        S.close()
    finally:
        comm.close()
        c.close()
    assert pair.status == two.status == 0
    assert abs(pair.loop - two.loop) <= max(2, 0.10 * two.loop)
    assert np.linalg.norm(pair.x - two.x) <= 1e-6 * np.linalg.norm(two.x)
    AT = A.to_scipy().T.tocsr()
    true = np.linalg.norm(b - AT @ pair.x) / np.linalg.norm(b)
    assert true <= 10 * two.true_rel_res + 1e-12 and true < 1e-8
