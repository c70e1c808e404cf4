"""GPU: the sm_100a primitives against the CPU oracle.

FP64 SpMV over rows of up to 16 nonzeros on average sums in the reference's
order and must match blas::MtxVec_mult bit for bit; denser rows (warp or
block per row) within 1e-13 relative. Reductions are compared with the
oracle's sequential sums to 1e-12 relative.
"""
import numpy as np
import pytest

from solver_cpp_b200.matrices import CSR, config_problem, transpose

pytestmark = pytest.mark.gpu


def ragged_matrix(n=6000, seed=0):
    """Rows of 0..2 nnz, a band of 100-400 nnz rows (warp-per-row blocks) and
    two rows of several thousand nnz (block-per-row)."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 3, n)
    lens[100:140] = rng.integers(100, 400, 40)
    lens[777] = 5000
    lens[n - 1] = 3100
    lens[5] = 0
    rows = []
    for i, L in enumerate(lens):
        c = np.sort(rng.choice(n, size=min(L, n), replace=False)) if L else np.zeros(0, dtype=np.int64)
        rows.append(c)
    ptr = np.zeros(n + 1, dtype=np.int64)
    ptr[1:] = np.cumsum([len(c) for c in rows])
    col = np.concatenate(rows).astype(np.int32)
    val = rng.standard_normal(col.shape[0])
    return CSR(ptr.astype(np.int32), col, val)


PROBLEMS = [("poisson2d", 64), ("poisson3d", 20), ("convdiff3d", 17), ("varcoef3d", 13), ("varcoef2d", 40)]


@pytest.mark.parametrize("index32", [False, True])
@pytest.mark.parametrize("prob,grid", PROBLEMS)
def test_spmv_fp64_bitwise_equals_reference_order(ks, ctx, oracle, prob, grid, index32):
    A, b, _ = config_problem(prob, grid)
    M = ctx.matrix(A, transpose=True, index32=index32)
    info = M.info()
    assert info["index_bytes"] == info["t_index_bytes"] == (4 if index32 else 2)
    x = np.random.default_rng(1).standard_normal(A.n)
    X, Y = ctx.vector(x), ctx.vector(n=A.n)
    ks.spmv(M, X, Y)
    P = oracle.Problem(A)
    assert np.array_equal(Y.numpy(), oracle.spmv(P, x))
    ks.spmv(M, X, Y, trans=True)
    assert np.array_equal(Y.numpy(), oracle.spmv(P, x, transpose=True))


def test_device_transpose_equals_csr2csc_layout(ks, ctx):
    A, _, _ = config_problem("convdiff3d", 15)
    M = ctx.matrix(A, transpose=True)
    tptr, trow, tval = M.transpose_arrays()
    T = transpose(A)
    assert np.array_equal(tptr, T.ptr) and np.array_equal(trow, T.col) and np.array_equal(tval, T.val)


def test_spmv_ragged_rows_all_bins(ks, ctx, oracle):
    A = ragged_matrix()
    M = ctx.matrix(A, transpose=True)
    info = M.info()
    assert info["row_blocks"] > 10
    x = np.random.default_rng(2).standard_normal(A.n)
    X, Y = ctx.vector(x), ctx.vector(n=A.n)
    ks.spmv(M, X, Y)
    ref = oracle.spmv(oracle.Problem(A), x)
    y = Y.numpy()
    rows_abs = np.bincount(np.repeat(np.arange(A.n), np.diff(A.ptr)), weights=np.abs(A.val * x[A.col]),
                           minlength=A.n)
    assert np.all(np.abs(y - ref) <= 1e-13 * rows_abs + 1e-300)
    # row blocks made only of short rows sum in index order (rows 200..700)
    assert np.array_equal(y[200:700], ref[200:700])
    ks.spmv(M, X, Y, trans=True)
    ref_t = oracle.spmv(oracle.Problem(A), x, transpose=True)
    T = transpose(A)
    rows_t = np.bincount(np.repeat(np.arange(A.n), np.diff(T.ptr)), weights=np.abs(T.val * x[T.col]),
                         minlength=A.n)
    assert np.all(np.abs(Y.numpy() - ref_t) <= 1e-13 * rows_t + 1e-300)


@pytest.mark.parametrize("values,tol", [("fp32", 2e-6), ("bf16", 2e-2)])
def test_spmv_low_precision_values(ks, ctx, values, tol):
    A, _, _ = config_problem("varcoef3d", 14)
    M = ctx.matrix(A, fp32=True, bf16=True)
    x = np.random.default_rng(4).standard_normal(A.n).astype(np.float32)
    X, Y = ctx.vector(x, dtype=ks.FP32), ctx.vector(n=A.n, dtype=ks.FP32)
    vt = ks.FP32 if values == "fp32" else ks.BF16
    ks.spmv(M, X, Y, values=vt)
    ref = A.to_scipy() @ x.astype(np.float64)
    absrow = abs(A.to_scipy()) @ np.abs(x.astype(np.float64))
    y = Y.numpy()
    assert np.all(np.abs(y - ref) <= tol * absrow + 1e-30)
    # the 16-bit column offsets change nothing in the sums
    M32 = ctx.matrix(A, fp32=True, bf16=True, index32=True)
    assert M.info()["index_bytes"] == 2 and M32.info()["index_bytes"] == 4
    ks.spmv(M32, X, Y, values=vt)
    assert np.array_equal(Y.numpy(), y)


def offset_matrix(n, up, down):
    """Rows i with the diagonal and columns i + up and i - down where they
    exist: A's column offsets reach +up and -down, those of A^T +down and -up."""
    rows = []
    for i in range(n):
        c = [j for j in (i - down, i, i + up) if 0 <= j < n]
        rows.append(c)
    ptr = np.zeros(n + 1, dtype=np.int32)
    ptr[1:] = np.cumsum([len(c) for c in rows])
    col = np.concatenate([np.array(c, dtype=np.int32) for c in rows])
    val = np.random.default_rng(n + up + down).standard_normal(col.shape[0])
    return CSR(ptr, col, val)


@pytest.mark.parametrize("up,down,a_bytes,t_bytes",
                         [(32767, 32767, 2, 2), (32767, 32768, 2, 4), (32768, 32767, 4, 2), (40000, 40000, 4, 4)])
def test_spmv_column_offsets_at_int16_limits(ks, ctx, oracle, up, down, a_bytes, t_bytes):
    A = offset_matrix(70000, up, down)
    M = ctx.matrix(A, transpose=True)
    info = M.info()
    assert (info["index_bytes"], info["t_index_bytes"]) == (a_bytes, t_bytes)
    x = np.random.default_rng(5).standard_normal(A.n)
    X, Y = ctx.vector(x), ctx.vector(n=A.n)
    P = oracle.Problem(A)
    ks.spmv(M, X, Y)
    assert np.array_equal(Y.numpy(), oracle.spmv(P, x))
    ks.spmv(M, X, Y, trans=True)
    assert np.array_equal(Y.numpy(), oracle.spmv(P, x, transpose=True))


def test_device_upload_checks_columns(ks, ctx):
    import ctypes as C

    import torch

    from solver_cpp_b200 import _abi

    A, _, _ = config_problem("poisson2d", 30)
    dev = torch.device("cuda", 0)
    ptr = torch.from_numpy(A.ptr.astype(np.int32)).to(dev)
    col = torch.from_numpy(A.col.astype(np.int32)).to(dev)
    val = torch.from_numpy(A.val.astype(np.float64)).to(dev)
    torch.cuda.synchronize()
    L = ks.lib()
    h = C.c_void_p()
    st = L.ks_csr_upload_device(ctx.handle, A.n, A.nnz, C.c_void_p(ptr.data_ptr()), C.c_void_p(col.data_ptr()),
                                C.c_void_p(val.data_ptr()), 0, C.byref(h))
    assert st == _abi.KS_OK
    a, t = C.c_int(), C.c_int()
    assert L.ks_mat_index_bytes(h, C.byref(a), C.byref(t)) == _abi.KS_OK and (a.value, t.value) == (2, 0)
    assert L.ks_mat_destroy(h) == _abi.KS_OK
    col[17] = A.n  # one column out of range
    torch.cuda.synchronize()
    h = C.c_void_p()
    st = L.ks_csr_upload_device(ctx.handle, A.n, A.nnz, C.c_void_p(ptr.data_ptr()), C.c_void_p(col.data_ptr()),
                                C.c_void_p(val.data_ptr()), 0, C.byref(h))
    assert st == _abi.KS_BAD_INPUT and not h.value
    assert b"out of range" in L.ks_last_error(ctx.handle)


def test_dot_nrm2_axpy(ks, ctx, oracle):
    n = 1_000_003
    rng = np.random.default_rng(5)
    x, y, w = rng.standard_normal(n), rng.standard_normal(n), rng.standard_normal(n)
    X, Y, W = ctx.vector(x), ctx.vector(y), ctx.vector(w)
    d = ks.dot(X, Y)
    assert d == pytest.approx(oracle.dot(x, y), rel=1e-12)
    assert ks.dot(X, Y) == d  # deterministic
    assert ks.nrm2(X) == pytest.approx(np.sqrt(oracle.dot(x, x)), rel=1e-13)
    ks.axpy(0.375, X, Y)
    yy = (0.375 * x) + y
    assert np.array_equal(Y.numpy(), yy)
    r = ks.axpy_dot(-1.25, W, Y, X)
    yy = (-1.25 * w) + yy
    assert np.array_equal(Y.numpy(), yy)
    assert r == pytest.approx(oracle.dot(yy, x), rel=1e-12)


def test_block_dot_and_axpy_match_gmres_sp(ks, ctx):
    n, k = 200_001, 13
    rng = np.random.default_rng(6)
    V = rng.standard_normal((k, n))
    w = rng.standard_normal(n)
    VV, WW = ctx.vector(V.ravel()), ctx.vector(w)
    h = ks.block_dot(VV, n, k, WW)
    np.testing.assert_allclose(h, V @ w, rtol=1e-12)
    ks.block_axpy(VV, n, k, h, WW)
    ref = w.copy()
    for i in range(k):  # blas::Gmres_sp_1 order
        ref = ref - h[i] * V[i]
    assert np.array_equal(WW.numpy(), ref)


def test_block_dot_and_axpy_with_device_coefficients(ks, ctx):
    """h in device memory: the block dot writes its k results there and the
    block AXPY reads them there, in stream order; the bits equal the
    host-array calls'."""
    n, k = 300_007, 21
    rng = np.random.default_rng(8)
    V = rng.standard_normal((k, n))
    w = rng.standard_normal(n)
    VV, W1, W2 = ctx.vector(V.ravel()), ctx.vector(w), ctx.vector(w)
    H = ctx.vector(n=k)
    h = ks.block_dot(VV, n, k, W1)
    assert ks.block_dot(VV, n, k, W2, out_device_ptr=H.device_ptr) is None
    assert np.array_equal(H.numpy(), h)
    ks.block_axpy(VV, n, k, h, W1)
    ks.block_axpy(VV, n, k, H.device_ptr, W2)
    assert np.array_equal(W1.numpy(), W2.numpy())


@pytest.mark.parametrize("k", [0, 1, 2, 4])
def test_matpow_and_gram(ks, ctx, oracle, k):
    A, _, _ = config_problem("convdiff3d", 12)
    P = oracle.Problem(A)
    M = ctx.matrix(A)
    rng = np.random.default_rng(7)
    r, p, rs, ps = (rng.standard_normal(A.n) for _ in range(4))
    Ar_o, Ap_o = oracle.matpow(P, r, p, k)
    R, Pv = ctx.vector(r), ctx.vector(p)
    Ar, Ap = ctx.vector(n=(2 * k + 1) * A.n), ctx.vector(n=(2 * k + 2) * A.n)
    ks.matpow(M, R, Pv, k, Ar, Ap)
    assert np.array_equal(Ar.numpy().reshape(2 * k + 1, A.n), Ar_o)
    assert np.array_equal(Ap.numpy().reshape(2 * k + 2, A.n), Ap_o)
    d, e, z = ks.gram_cg(Ar, Ap, R, Pv, k)
    d_o, e_o, z_o = oracle.gram_cg(r, p, Ar_o, Ap_o, k)
    np.testing.assert_allclose(d, d_o, rtol=1e-11)
    np.testing.assert_allclose(e, e_o, rtol=1e-11)
    np.testing.assert_allclose(z, z_o, rtol=1e-11)
    RS, PS = ctx.vector(rs), ctx.vector(ps)
    t, e2, rho, phi = ks.gram_bicg(Ar, Ap, RS, PS, k)
    t_o, e2_o, rho_o, phi_o = oracle.gram_bicg(rs, ps, Ar_o, Ap_o, k)
    for a, b_ in ((t, t_o), (e2, e2_o), (rho, rho_o), (phi, phi_o)):
        np.testing.assert_allclose(a, b_, rtol=1e-10, atol=1e-12 * np.max(np.abs(b_)) if b_.size else 0)


def test_pattern_grad_bitwise(ks, ctx, oracle):
    A, _, _ = config_problem("varcoef2d", 30)
    M = ctx.matrix(A)
    rng = np.random.default_rng(8)
    lam, x = rng.standard_normal(A.n), rng.standard_normal(A.n)
    L, X, G = ctx.vector(lam), ctx.vector(x), ctx.vector(n=A.nnz)
    ks.pattern_grad(M, L, X, G)
    assert np.array_equal(G.numpy(), oracle.pattern_grad(oracle.Problem(A), lam, x))


def test_check_error_matches_reference(ks, ctx, oracle):
    A, b, _ = config_problem("poisson3d", 10)
    M = ctx.matrix(A)
    x = np.random.default_rng(9).standard_normal(A.n) * 0.01
    lg, rel = ks.check_error(M, ctx.vector(b), ctx.vector(x))
    P = oracle.Problem(A)
    import ctypes as C

    x0 = np.zeros(A.n)
    ref = oracle.lib().oracle_check_error(C.byref(P.mat), b.ctypes.data, x.ctypes.data, x0.ctypes.data)
    assert lg == pytest.approx(ref, rel=1e-13)
