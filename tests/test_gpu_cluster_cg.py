"""GPU: CG, CR and BiCG on small systems as one thread-block-cluster launch.

Up to 32768 rows (one GPU, FP64) CG, CR and BiCG run as a single launch of one
cluster of up to 16 CTAs (ks_params.cluster_solve 0, the default); cluster_solve 1
selects the kernel-per-step engine used for larger systems. Both paths do the
same element-wise arithmetic and differ only in the order in which the dot
products add their terms, so each must reproduce the reference's golden
histories under the same criterion (golden_cases.check_history), agree with
the other to rounding, and report the same iteration counts, verdicts and
maxloop behaviour as the oracle.
"""
import numpy as np
import pytest

from golden_cases import check_history, index, load, oracle_envelope
from solver_cpp_b200.matrices import config_problem

pytestmark = pytest.mark.gpu

CG_CASES = sorted(c for c, m in index().items() if m["outer"] == "CG")


@pytest.mark.parametrize("cluster_solve", [0, 1])
@pytest.mark.parametrize("cid", CG_CASES)
def test_cg_golden_history_on_both_paths(ks, ctx, cid, cluster_solve):
    meta, g = load(cid)
    A, b, _ = config_problem(meta["problem"], meta["grid"])
    M = ctx.matrix(A)
    r = ks.solve(ctx, M, "CG", b, cluster_solve=cluster_solve, **meta["params"])
    assert r.converged == meta["converged"]
    check_history(r.hist_iter, r.hist_err, g["hist_iter"], g["hist_err"], g["envelope"], r.loop, meta["loop"],
                  meta["loop_range"])
    assert round(r.true_res_log10, 1) == pytest.approx(meta["true_res_log10"], abs=0.21)


# grid edges giving n = 1, 25, 961 (not a multiple of 32), 2025, 16384, 32761
# and 32768 (the largest single-cluster system: 16 CTAs of 2048 rows), and
# 33124 (above the limit: cluster_solve 0 runs it as one on-chip kernel of one
# CTA per SM, 1 as one kernel per step)
SHAPES = [("poisson2d", 1), ("poisson2d", 5), ("poisson2d", 31), ("poisson2d", 45), ("poisson2d", 128),
          ("poisson2d", 181), ("poisson3d", 32), ("poisson2d", 182)]


@pytest.mark.parametrize("prob,g", SHAPES)
def test_cluster_and_engine_agree(ks, ctx, prob, g):
    A, b, _ = config_problem(prob, g)
    M = ctx.matrix(A)
    r0 = ks.solve(ctx, M, "CG", b, E=1e-12, L=5000, cluster_solve=0)
    r1 = ks.solve(ctx, M, "CG", b, E=1e-12, L=5000, cluster_solve=1)
    assert r0.status == r1.status == 0
    assert abs(r0.loop - r1.loop) <= max(1, r1.loop // 100)
    assert np.linalg.norm(r0.x - r1.x) <= 1e-10 * np.linalg.norm(r1.x)
    m = min(len(r0.hist_err), len(r1.hist_err)) // 2  # the first half agrees closely
    assert np.allclose(r0.hist_err[:m], r1.hist_err[:m], rtol=1e-8, atol=0)
    assert r0.true_rel_res < 2e-12


def test_cluster_int32_columns_and_device_vectors(ks, ctx):
    """Columns kept as int32 (KS_MAT_INDEX32) and as 16-bit offsets give the
    same solve bit for bit; device vectors give the host path's x."""
    A, b, _ = config_problem("varcoef3d", 16)
    r16 = ks.solve(ctx, ctx.matrix(A), "CG", b, E=1e-10)
    M32 = ctx.matrix(A, index32=True)
    assert M32.info()["index_bytes"] == 4
    r32 = ks.solve(ctx, M32, "CG", b, E=1e-10)
    assert np.array_equal(r16.x, r32.x) and np.array_equal(r16.hist_err, r32.hist_err)
    B, X = ctx.vector(b), ctx.vector(n=A.n)
    rd = ks.solve(ctx, M32, "CG", B, x=X, E=1e-10)
    assert rd.converged and np.array_equal(X.numpy(), r32.x)
    r2 = ks.solve(ctx, M32, "CG", b, E=1e-10)  # repeat: deterministic
    assert np.array_equal(r2.x, r32.x) and np.array_equal(r2.hist_err, r32.hist_err)


@pytest.mark.parametrize("L", [0, 1, 7, 255, 256, 257, 300])
def test_cluster_maxloop_and_history_flushes(ks, ctx, oracle, L):
    """The history is kept in shared memory and written out every 256 entries
    and at the end: maxloop values around that boundary must give the
    oracle's loop count, labels and verdict, and a history within the
    reference-envelope criterion."""
    A, b, _ = config_problem("varcoef2d", 40)
    M = ctx.matrix(A)
    r = ks.solve(ctx, M, "CG", b, L=L, E=1e-30)
    o, env, lr = oracle_envelope(oracle, A, b, "CG", L=L, E=1e-30)
    assert r.status == o["status"] == 2
    assert r.loop == o["loop"]
    assert np.array_equal(r.hist_iter, o["hist_iter"])
    if L > 0:  # L = 0 stops before the first entry
        check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)
    e = ks.solve(ctx, M, "CG", b, L=L, E=1e-30, cluster_solve=1)
    assert np.array_equal(e.hist_iter, r.hist_iter)
    assert np.linalg.norm(e.x - r.x) <= 1e-9 * max(np.linalg.norm(e.x), 1e-300)


def test_cluster_solve_rejects_bad_value(ks, ctx):
    A, b, _ = config_problem("poisson2d", 8)
    with pytest.raises(ks.KrylovError) as e:
        ks.solve(ctx, ctx.matrix(A), "CG", b, cluster_solve=2)
    assert e.value.status == 5


# ------------------------------------------------------------------ BiCG
BICG_CASES = sorted(c for c, m in index().items() if m["outer"] == "BICG")


@pytest.mark.parametrize("cluster_solve", [0, 1])
@pytest.mark.parametrize("cid", BICG_CASES)
def test_bicg_golden_history_on_both_paths(ks, ctx, cid, cluster_solve):
    meta, g = load(cid)
    A, b, _ = config_problem(meta["problem"], meta["grid"])
    M = ctx.matrix(A, transpose=True)
    r = ks.solve(ctx, M, "BICG", b, cluster_solve=cluster_solve, **meta["params"])
    assert r.converged == meta["converged"]
    check_history(r.hist_iter, r.hist_err, g["hist_iter"], g["hist_err"], g["envelope"], r.loop, meta["loop"],
                  meta["loop_range"])
    assert round(r.true_res_log10, 1) == pytest.approx(meta["true_res_log10"], abs=0.21)


# BiCG departs from itself under a change of summation order much sooner than
# CG. On the small systems both paths are held to the oracle's envelope; on
# the larger ones (the oracle's own chunked sums differ by 1e-4 within the
# first half of the 128^2 history and its iteration counts spread over
# 428-463; at 182^2 the engine converged in 608 iterations, the oracle in 693)
# to convergence with a true residual near the oracle's (BiCG stops on its
# recurrence residual, and the true one lies above it by as much in the
# oracle: 1.2e-11 at 128^2).
BICG_SHAPES = [("convdiff2d", 1, True), ("convdiff2d", 5, True), ("convdiff2d", 31, True),
               ("convdiff2d", 45, True), ("convdiff2d", 128, False), ("convdiff2d", 181, False),
               ("convdiff3d", 32, False), ("convdiff2d", 182, False)]


@pytest.mark.parametrize("prob,g,strict", BICG_SHAPES)
def test_bicg_cluster_and_engine_against_oracle(ks, ctx, oracle, prob, g, strict):
    A, b, _ = config_problem(prob, g)
    M = ctx.matrix(A, transpose=True)
    o, env, lr = oracle_envelope(oracle, A, b, "BICG", E=1e-12, L=5000)
    o_true = np.linalg.norm(b - A.to_scipy() @ o["x"]) / np.linalg.norm(b)
    for cs in (0, 1):
        r = ks.solve(ctx, M, "BICG", b, E=1e-12, L=5000, cluster_solve=cs)
        assert r.status == o["status"] == 0, (cs, r.status)
        if strict:
            check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)
        assert r.true_rel_res < 3 * max(o_true, 1e-12), (cs, r.true_rel_res, o_true)


@pytest.mark.parametrize("L", [0, 1, 7, 255, 256, 257])
def test_bicg_cluster_maxloop_and_history_flushes(ks, ctx, oracle, L):
    A, b, _ = config_problem("convdiff2d", 40)
    M = ctx.matrix(A, transpose=True)
    r = ks.solve(ctx, M, "BICG", b, L=L, E=1e-30)
    o, env, lr = oracle_envelope(oracle, A, b, "BICG", L=L, E=1e-30)
    assert r.status == o["status"] == 2
    assert r.loop == o["loop"]
    assert np.array_equal(r.hist_iter, o["hist_iter"])
    if L > 0:
        check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)


# ------------------------------------------------------------------ CR
CR_CASES = sorted(c for c, m in index().items() if m["outer"] == "CR")


@pytest.mark.parametrize("cluster_solve", [0, 1])
@pytest.mark.parametrize("cid", CR_CASES)
def test_cr_golden_history_on_both_paths(ks, ctx, cid, cluster_solve):
    meta, g = load(cid)
    A, b, _ = config_problem(meta["problem"], meta["grid"])
    M = ctx.matrix(A)
    r = ks.solve(ctx, M, "CR", b, cluster_solve=cluster_solve, **meta["params"])
    assert r.converged == meta["converged"]
    check_history(r.hist_iter, r.hist_err, g["hist_iter"], g["hist_err"], g["envelope"], r.loop, meta["loop"],
                  meta["loop_range"])
    assert round(r.true_res_log10, 1) == pytest.approx(meta["true_res_log10"], abs=0.21)


@pytest.mark.parametrize("prob,g", SHAPES)
def test_cr_cluster_and_engine_within_envelope(ks, ctx, oracle, prob, g):
    A, b, _ = config_problem(prob, g)
    M = ctx.matrix(A)
    o, env, lr = oracle_envelope(oracle, A, b, "CR", E=1e-12, L=5000)
    for cs in (0, 1):
        r = ks.solve(ctx, M, "CR", b, E=1e-12, L=5000, cluster_solve=cs)
        assert r.status == o["status"] == 0, (cs, r.status)
        check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)
        assert r.true_rel_res < 2e-12, (cs, r.true_rel_res)


@pytest.mark.parametrize("L", [0, 1, 7, 255, 256, 257])
def test_cr_cluster_maxloop_and_history_flushes(ks, ctx, oracle, L):
    A, b, _ = config_problem("varcoef2d", 40)
    M = ctx.matrix(A)
    r = ks.solve(ctx, M, "CR", b, L=L, E=1e-30)
    o, env, lr = oracle_envelope(oracle, A, b, "CR", L=L, E=1e-30)
    assert r.status == o["status"] == 2
    assert r.loop == o["loop"]
    assert np.array_equal(r.hist_iter, o["hist_iter"])
    if L > 0:
        check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)


@pytest.mark.parametrize("prob,g", [("varcoef3d", 40), ("poisson3d", 64), ("varcoef2d", 256)])
def test_onchip_cg_within_reference_envelope(ks, ctx, oracle, prob, g):
    """CG on systems above one cluster's reach but with vectors that fit on chip
    across the GPU runs as one cooperative kernel (cluster_solve 0); it must
    meet the reference's parity criterion against the oracle (envelope of
    the oracle's chunked-sum runs), as the kernel-per-step engine
    (cluster_solve 1) does, with the same verdict and solution."""
    A, b, _ = config_problem(prob, g)
    M = ctx.matrix(A)
    chip = ks.solve(ctx, M, "CG", b, E=1e-10, L=20000, cluster_solve=0)
    step = ks.solve(ctx, M, "CG", b, E=1e-10, L=20000, cluster_solve=1)
    o, env, lr = oracle_envelope(oracle, A, b, "CG", E=1e-10, L=20000)
    for r in (chip, step):
        assert r.converged and o["status"] == 0
        check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)
        assert r.true_res_log10 < -9.5
    assert np.linalg.norm(chip.x - step.x) <= 1e-8 * np.linalg.norm(step.x)


@pytest.mark.parametrize("prob,g", [("convdiff2d", 200), ("convdiff3d", 40), ("convdiff2d", 256), ("varcoef2d", 256),
                                    ("convdiff2d", 182), ("convdiff3d", 37)])
def test_onchip_bicg_against_oracle_and_engine(ks, ctx, oracle, prob, g):
    """BiCG above one cluster's reach, its six vectors in shared memory across
    the GPU: one cooperative launch (cluster_solve 0; the profile counts the
    whole solve as one SpMV-class launch and no dot kernels). It applies the
    engine's element operations and adds the dot products in another order.
    BiCG's iteration count on the upwind systems moves with that order alone
    (convdiff2d 200^2: the oracle takes 791 iterations with sequential sums,
    749 / 704 / 663 with 16 / 256 / 4096 partial sums, 654 pairwise), so the
    count of either GPU path must lie in the range of the oracle's orders
    (+-2 %). Then the oracle's verdict, a true residual within 3x the
    oracle's, the engine's solution to 1e-7 and the first history entries to
    1e-9. varcoef2d is symmetric (symmetric diagonal storage for A and its
    transpose); 182^2 and 37^3 have offsets that are not multiples of 4 (the
    generic quad path)."""
    A, b, _ = config_problem(prob, g)
    M = ctx.matrix(A, transpose=True)
    chip = ks.solve(ctx, M, "BICG", b, E=1e-12, L=20000, cluster_solve=0, profile=1)
    step = ks.solve(ctx, M, "BICG", b, E=1e-12, L=20000, cluster_solve=1)
    assert chip.report["n_mv"] == 1 and chip.report["n_dot"] == 0, chip.report
    o, _, _ = oracle_envelope(oracle, A, b, "BICG", E=1e-12, L=20000)
    o_true = np.linalg.norm(b - A.to_scipy() @ o["x"]) / np.linalg.norm(b)
    P = oracle.Problem(A)
    loops = [oracle.solve(P, b, "BICG", E=1e-12, L=20000, sum_chunks=c)["loop"] for c in (0, 16, 256, 4096, -1)]
    lo, hi = min(loops) * 0.98 - 1, max(loops) * 1.02 + 1
    assert chip.status == step.status == o["status"] == 0
    assert lo <= chip.loop <= hi, (chip.loop, loops)
    assert lo <= step.loop <= hi, (step.loop, loops)
    assert chip.true_rel_res < 3 * max(o_true, 1e-12)
    assert np.linalg.norm(chip.x - step.x) <= 1e-7 * np.linalg.norm(step.x)
    m = min(len(chip.hist_err), len(step.hist_err), 10)
    assert np.allclose(chip.hist_err[:m], step.hist_err[:m], rtol=1e-9, atol=0)


def test_onchip_bicg_maxloop_and_zero_rhs(ks, ctx):
    """The on-chip BiCG stops at maxloop with the engine's loop count and
    history labels, and a zero right-hand side stops at once (NaN test of
    0/0), as the engine does."""
    A, b, _ = config_problem("convdiff2d", 200)
    M = ctx.matrix(A, transpose=True)
    for L in (1, 7, 300):
        chip = ks.solve(ctx, M, "BICG", b, E=1e-30, L=L, cluster_solve=0)
        step = ks.solve(ctx, M, "BICG", b, E=1e-30, L=L, cluster_solve=1)
        assert chip.status == step.status == 2
        assert chip.loop == step.loop
        assert np.array_equal(chip.hist_iter, step.hist_iter)
    z = np.zeros(A.n)
    chip = ks.solve(ctx, M, "BICG", z, E=1e-10, L=100, cluster_solve=0)
    step = ks.solve(ctx, M, "BICG", z, E=1e-10, L=100, cluster_solve=1)
    assert chip.status == step.status
    assert chip.loop == step.loop


@pytest.mark.parametrize("prob,g", [("varcoef3d", 40), ("poisson3d", 64), ("varcoef2d", 256), ("poisson2d", 300)])
def test_onchip_cr_within_reference_envelope(ks, ctx, oracle, prob, g):
    """CR above one cluster's reach, r and p in shared memory, q and s in TMEM
    and x in global memory: one cooperative launch (cluster_solve 0; the
    profile counts the whole solve as one SpMV-class launch). It must meet the
    reference's parity criterion against the oracle (envelope of the
    oracle's chunked-sum runs) as the engine (cluster_solve 1) does, with the
    same verdict and solution. poisson2d 300^2 has offsets +-300, multiples
    of 4; 64^3 has 4 quads of rows per thread."""
    A, b, _ = config_problem(prob, g)
    M = ctx.matrix(A)
    chip = ks.solve(ctx, M, "CR", b, E=1e-10, L=20000, cluster_solve=0, profile=1)
    step = ks.solve(ctx, M, "CR", b, E=1e-10, L=20000, cluster_solve=1)
    assert chip.report["n_mv"] == 1 and chip.report["n_dot"] == 0, chip.report
    o, env, lr = oracle_envelope(oracle, A, b, "CR", E=1e-10, L=20000)
    for r in (chip, step):
        assert r.converged and o["status"] == 0
        check_history(r.hist_iter, r.hist_err, o["hist_iter"], o["hist_err"], env, r.loop, o["loop"], lr)
        assert r.true_res_log10 < -9.5
    assert np.linalg.norm(chip.x - step.x) <= 1e-8 * np.linalg.norm(step.x)


def test_onchip_cr_maxloop_and_generic_offsets(ks, ctx):
    """The on-chip CR stops at maxloop with the engine's loop count and
    history labels; varcoef3d 37^3 has offsets 37 and 1369 (not multiples of
    4: the generic quad path) and agrees with the engine to rounding."""
    A, b, _ = config_problem("varcoef3d", 37)
    M = ctx.matrix(A)
    for L in (1, 7, 300):
        chip = ks.solve(ctx, M, "CR", b, E=1e-30, L=L, cluster_solve=0)
        step = ks.solve(ctx, M, "CR", b, E=1e-30, L=L, cluster_solve=1)
        assert chip.status == step.status == 2
        assert chip.loop == step.loop
        assert np.array_equal(chip.hist_iter, step.hist_iter)
        m = min(len(chip.hist_err), 20)
        assert np.allclose(chip.hist_err[:m], step.hist_err[:m], rtol=1e-9, atol=0)
