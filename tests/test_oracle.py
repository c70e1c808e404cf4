"""CPU: the oracle (C restatement) is pinned against the reference's own runs.

The golden fixtures hold what the reference printed (13 significant digits)
for 29 runs covering every method and every inner solver; the oracle must
reproduce each history entry, the iteration count, the verdict, the printed
true residual and the solution to that precision.
"""
import hashlib

import numpy as np
import pytest

from golden_cases import index, load, rel_close
from solver_cpp_b200.matrices import config_problem, transpose

PRINT_RTOL = 6e-13  # %.12E -> 13 significant digits


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


CASES = sorted(index().keys())


@pytest.mark.parametrize("cid", CASES)
def test_oracle_matches_reference_golden(oracle, cid):
    meta, g = load(cid)
    A, b, _ = config_problem(meta["problem"], meta["grid"])
    assert _digest(A.val) == meta["sha_val"], "matrix generator changed"
    assert _digest(b) == meta["sha_b"], "right-hand side generator changed"
    r = oracle.solve(A, b, meta["outer"], meta["inner"], **meta["params"])
    assert r["loop"] == meta["loop"]
    assert (r["status"] == 0) == meta["converged"]
    assert np.array_equal(r["hist_iter"], g["hist_iter"])
    assert np.all(rel_close(r["hist_err"], g["hist_err"], PRINT_RTOL))
    assert round(r["true_res_log10"], 1) == pytest.approx(meta["true_res_log10"], abs=0.051)
    if g["x"].size:
        assert np.all(np.abs(r["x"] - g["x"]) <= PRINT_RTOL * np.abs(g["x"]) + 1e-300)


@pytest.mark.parametrize("cid", ["cd2_bicg", "cd2_gmres", "vc3_cg", "vc3_vpcg_cg", "cd3_kskipbicg"])
def test_parity_criterion_accepts_a_reordered_sum(oracle, cid):
    """The history criterion used for the GPU accepts the oracle run with its
    dot products summed in 3 or 5 parts (another legitimate summation order)."""
    from golden_cases import check_history

    meta, g = load(cid)
    A, b, _ = config_problem(meta["problem"], meta["grid"])
    for chunks in (3, 5):
        r = oracle.solve(A, b, meta["outer"], meta["inner"], sum_chunks=chunks, **meta["params"])
        check_history(r["hist_iter"], r["hist_err"], g["hist_iter"], g["hist_err"], g["envelope"], r["loop"],
                      meta["loop"], meta["loop_range"])


def test_c1_configuration(oracle):
    """CG on the 64x64 Poisson problem, tol 1e-10, 202 iterations."""
    meta, g = load("c1_cg")
    assert meta["n"] == 4096 and meta["nnz"] == 20224
    assert meta["loop"] == 202 and meta["converged"]


def test_transpose_matches_numpy(oracle):
    A, _, _ = config_problem("convdiff2d", 16)
    T = transpose(A)
    tptr = np.zeros(A.n + 1, dtype=np.int32)
    trow = np.zeros(A.nnz, dtype=np.int32)
    tval = np.zeros(A.nnz)
    import ctypes as C

    oracle.lib().oracle_csr_transpose.argtypes = [C.c_long, C.c_long] + [C.c_void_p] * 6
    oracle.lib().oracle_csr_transpose(A.n, A.nnz, A.ptr.ctypes.data, A.col.ctypes.data, A.val.ctypes.data,
                                      tptr.ctypes.data, trow.ctypes.data, tval.ctypes.data)
    assert np.array_equal(tptr, T.ptr) and np.array_equal(trow, T.col) and np.array_equal(tval, T.val)
    dense = A.to_scipy().toarray()
    assert np.array_equal(T.to_scipy().toarray(), dense.T)


def test_matpow_and_gram_match_numpy(oracle):
    A, b, _ = config_problem("convdiff2d", 12)
    P = oracle.Problem(A)
    rng = np.random.default_rng(11)
    r, p, rs, ps = (rng.standard_normal(A.n) for _ in range(4))
    k = 2
    Ar, Ap = oracle.matpow(P, r, p, k)
    M = A.to_scipy()
    v, w = r.copy(), p.copy()
    for i in range(2 * k + 2):
        w = M @ w
        np.testing.assert_allclose(Ap[i], w, rtol=1e-12, atol=1e-12)
        if i < 2 * k + 1:
            v = M @ v
            np.testing.assert_allclose(Ar[i], v, rtol=1e-12, atol=1e-12)
    d, e, z = oracle.gram_cg(r, p, Ar, Ap, k)
    np.testing.assert_allclose(d, Ar[:2 * k] @ r, rtol=1e-12)
    np.testing.assert_allclose(e, Ap[:2 * k + 1] @ r, rtol=1e-12)
    np.testing.assert_allclose(z, Ap @ p, rtol=1e-12)
    t, e2, rho, phi = oracle.gram_bicg(rs, ps, Ar, Ap, k)
    np.testing.assert_allclose(t, Ar[:2 * k] @ rs, rtol=1e-12)
    np.testing.assert_allclose(e2, Ap[:2 * k + 1] @ rs, rtol=1e-12)
    np.testing.assert_allclose(rho, Ar @ ps, rtol=1e-12)
    np.testing.assert_allclose(phi, Ap @ ps, rtol=1e-12)


@pytest.mark.parametrize("k", [1, 2, 4])
def test_corrected_kskipcg_tracks_cg(oracle, k):
    """The reference's k-skip CG recurrences never converge (kskipcg.cpp:284-287);
    the corrected ones reproduce plain CG."""
    A, b, _ = config_problem("poisson2d", 32)
    cg = oracle.solve(A, b, "CG", E=1e-10)
    ks = oracle.solve(A, b, "KSKIPCG", E=1e-10, K=k, fix_kskipcg=1)
    bad = oracle.solve(A, b, "KSKIPCG", E=1e-10, K=k, L=300)
    assert ks["status"] == 0 and cg["status"] == 0
    assert ks["true_res_log10"] < -9.5
    assert abs(ks["loop"] - cg["loop"]) <= 2 * (k + 1)
    assert bad["status"] == 2
    # the k-skip history samples CG's every k+1 iterations
    blocks = ks["hist_iter"]
    np.testing.assert_allclose(ks["hist_err"][:5], cg["hist_err"][blocks[:5] - 1], rtol=1e-6)


def test_corrected_gmres_assembly(oracle):
    """On convergence inside a restart cycle the reference keeps only the last
    basis term (gmres.cpp:290-297); the corrected assembly reaches the residual
    its history reports."""
    A, b, _ = config_problem("convdiff2d", 32)
    ref = oracle.solve(A, b, "GMRES", E=1e-10, R=30)
    fixd = oracle.solve(A, b, "GMRES", E=1e-10, R=30, fix_gmres_assembly=1)
    assert np.array_equal(ref["hist_err"], fixd["hist_err"])
    assert ref["true_res_log10"] > -9.5
    assert fixd["true_res_log10"] < -9.9


def test_pattern_grad_matches_dense(oracle):
    A, _, _ = config_problem("varcoef2d", 8)
    P = oracle.Problem(A)
    rng = np.random.default_rng(3)
    lam, x = rng.standard_normal(A.n), rng.standard_normal(A.n)
    g = oracle.pattern_grad(P, lam, x)
    dense = -np.outer(lam, x)
    rows = np.repeat(np.arange(A.n), np.diff(A.ptr))
    np.testing.assert_array_equal(g, dense[rows, A.col])
