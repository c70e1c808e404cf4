"""GPU: every Krylov method reproduces the reference's own run.

Against the golden fixtures (the reference's CPU path, -t 1): the residual
history to 1e-8 relative per entry up to the point where the reference
departs from itself under a change of OpenMP thread count, within 10x that
self-departure afterwards, the iteration count within the reference's own
spread +-1 %, the same verdict and the same printed true residual
(golden_cases.check_history). SpMV and every element-wise update match the
reference bit for bit; only the order of the terms of each dot product
differs. Methods with reference defects run with reference_defects=1 here;
the corrected forms are checked against the corrected oracle below.
"""
import numpy as np
import pytest

from golden_cases import check_history, index, load, oracle_envelope
from solver_cpp_b200.matrices import config_problem

pytestmark = pytest.mark.gpu


def _mat(ctx, A):
    return ctx.matrix(A, transpose=True, fp32=True, bf16=True)


@pytest.mark.parametrize("cid", sorted(index().keys()))
def test_history_matches_reference(ks, ctx, cid):
    meta, g = load(cid)
    A, b, _ = config_problem(meta["problem"], meta["grid"])
    M = _mat(ctx, A)
    r = ks.solve(ctx, M, meta["outer"], b, inner=meta["inner"], reference_defects=1, **meta["params"])
    assert r.converged == meta["converged"]
    check_history(r.hist_iter, r.hist_err, g["hist_iter"], g["hist_err"], g["envelope"], r.loop, meta["loop"],
                  meta["loop_range"])
    if meta["converged"] or meta["true_res_log10"] < 0:
        assert round(r.true_res_log10, 1) == pytest.approx(meta["true_res_log10"], abs=0.21)


@pytest.mark.parametrize("k", [1, 2, 4])
def test_corrected_kskipcg_matches_corrected_oracle(ks, ctx, oracle, k):
    A, b, _ = config_problem("poisson3d", 16)
    M = _mat(ctx, A)
    r = ks.solve(ctx, M, "KSKIPCG", b, E=1e-10, K=k)
    o, env, lr = oracle_envelope(oracle, A, b, "KSKIPCG", E=1e-10, K=k, fix_kskipcg=1)
    assert r.converged and o["status"] == 0
    check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)
    assert r.true_res_log10 < -9.5


@pytest.mark.parametrize("outer,inner", [("GMRES", "NONE"), ("VPGMRES", "CG")])
def test_corrected_gmres_assembly(ks, ctx, oracle, outer, inner):
    A, b, _ = config_problem("convdiff2d", 32)
    M = _mat(ctx, A)
    kw = dict(E=1e-10, R=30, l=10, e=0.1)
    r = ks.solve(ctx, M, outer, b, inner=inner, **kw)
    o, env, lr = oracle_envelope(oracle, A, b, outer, inner, fix_gmres_assembly=1, **kw)
    assert r.converged == (o["status"] == 0)
    check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)
    if r.converged:
        assert r.true_res_log10 < -9.5


def test_not_implemented_methods(ks, ctx):
    A, b, _ = config_problem("poisson2d", 8)
    M = _mat(ctx, A)
    for name in ("KSKIPCR", "VPBICG"):
        with pytest.raises(ks.KrylovError) as e:
            ks.solve(ctx, M, name, b, inner="CG")
        assert e.value.status == 99


def test_maxloop_and_loop_reporting(ks, ctx, oracle):
    A, b, _ = config_problem("poisson2d", 32)
    M = _mat(ctx, A)
    for name, kw in (("CG", {}), ("CR", {}), ("BICG", {}), ("GCR", {"R": 5}), ("GMRES", {"R": 5}),
                     ("KSKIPBICG", {"K": 2})):
        r = ks.solve(ctx, M, name, b, L=7, E=1e-14, **kw)
        o = oracle.solve(A, b, name, L=7, E=1e-14, **kw)
        assert r.status == 2 and o["status"] == 2
        assert r.loop == o["loop"], name
        assert np.array_equal(r.hist_iter, o["hist_iter"]), name


def test_breakdown_and_nan_paths(ks, ctx):
    """b = 0: |b| = 0 gives a NaN residual ratio; the reference loops to maxloop
    on NaNs, the library stops at once with KS_NAN_DETECTED."""
    A, _, _ = config_problem("poisson2d", 8)
    M = _mat(ctx, A)
    r = ks.solve(ctx, M, "CG", np.zeros(A.n), L=50)
    assert r.status == 4
    assert r.loop <= 2


def test_repeat_solves_are_deterministic(ks, ctx):
    A, b, _ = config_problem("convdiff3d", 14)
    M = _mat(ctx, A)
    r1 = ks.solve(ctx, M, "BICG", b, E=1e-10)
    r2 = ks.solve(ctx, M, "BICG", b, E=1e-10)
    assert np.array_equal(r1.hist_err, r2.hist_err) and np.array_equal(r1.x, r2.x)


def test_device_vectors_path(ks, ctx):
    A, b, _ = config_problem("poisson3d", 12)
    M = _mat(ctx, A)
    B = ctx.vector(b)
    X = ctx.vector(n=A.n)
    r = ks.solve(ctx, M, "CG", B, x=X, E=1e-10)
    h = ks.solve(ctx, M, "CG", b, E=1e-10)
    assert r.converged and np.array_equal(X.numpy(), h.x)


@pytest.mark.parametrize("diag", [True, False])
@pytest.mark.parametrize("name", ["CG", "CR", "BICG"])
def test_deferred_solution_update_at_ring_boundaries(ks, ctx, oracle, name, diag):
    """CG, CR and BiCG apply x += alpha p either every iteration or through a
    ring of 32 directions (x_update 1 / 2; 0 picks by L2 fit). Stopping
    before, at and after a full ring (and at maxloop = the ring size) must
    leave the same x bit for bit, and the x of the per-iteration update. On
    the diagonal copy (this size) CG and BiCG form the direction inside the
    SpMV, on CSR they run a separate direction update. CG runs the
    kernel-per-step engine here (cluster_solve 1)."""
    A, b, _ = config_problem("convdiff3d" if name == "BICG" else "poisson3d", 24)
    M = ctx.matrix(A, transpose=True, diag=diag)
    kw = {"cluster_solve": 1} if name == "CG" else {}
    for L in (1, 5, 31, 32, 33, 64, 65, 90):
        r1 = ks.solve(ctx, M, name, b, L=L, E=1e-30, x_update=1, **kw)
        r2 = ks.solve(ctx, M, name, b, L=L, E=1e-30, x_update=2, **kw)
        assert np.array_equal(r1.x, r2.x) and np.array_equal(r1.hist_err, r2.hist_err), (name, L)
        o = oracle.solve(A, b, name, L=L, E=1e-30)
        assert r2.loop == o["loop"] and r2.status == o["status"] == 2, (name, L)
        scale = np.linalg.norm(o["x"])
        assert np.linalg.norm(r2.x - o["x"]) <= 1e-10 * scale, (name, L)
