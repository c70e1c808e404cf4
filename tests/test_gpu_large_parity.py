"""GPU: the benchmark configurations at full size against the reference's own runs.

The fixtures (tests/golden/make_golden.py --large) hold the reference's CPU
path run on the 128^3 Poisson and convection-diffusion systems and the 160^3
log-normal system, at -t 1 (the history) and -t 2/3/4/8 (its self-departure
envelope and loop counts). The GPU solve of the same seeded system must give
the history within golden_cases.check_history's criterion, the same verdict
and the same printed true residual.

Iteration counts. SpMVs and vector updates match the reference bit for bit;
only the order in which a dot product adds its terms differs, and on the
ill-conditioned systems that order alone moves the count: the reference
itself takes 5158 to 5209 CG iterations on the 160^3 system depending on its
thread count. The loop-count range is therefore the reference's own counts
over its thread counts together with the counts of the oracle (the C
restatement, which reproduces the reference's -t 1 history bit for bit) with
its dot products summed in further orders, up to pairwise summation, the
accuracy class of the GPU's tree reductions (make_golden.py --orders), +-1 %.
"""
import hashlib

import numpy as np
import pytest

from golden_cases import check_history, index_large, load_large
from solver_cpp_b200.matrices import config_problem

pytestmark = pytest.mark.gpu

_PROBLEMS = {}


def _problem(name, grid):
    key = (name, grid)
    if key not in _PROBLEMS:
        _PROBLEMS.clear()  # one full-size system in host memory at a time
        _PROBLEMS[key] = config_problem(name, grid)
    return _PROBLEMS[key]


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def loop_range(meta):
    """Reference counts over its thread counts, plus the oracle's under the
    other summation orders."""
    loops = list(meta["loops_by_threads"].values()) + list(meta.get("oracle_loops_by_order", {}).values())
    return min(loops), max(loops)


@pytest.mark.parametrize("cid", sorted(index_large().keys()))
def test_full_size_history_matches_reference(ks, ctx, cid):
    meta, g = load_large(cid)
    A, b, _ = _problem(meta["problem"], meta["grid"])
    assert _digest(A.val) == meta["sha_val"] and _digest(b) == meta["sha_b"], "generator changed"
    M = ctx.matrix(A, transpose=meta["outer"] in ("BICG", "KSKIPBICG"))
    try:
        r = ks.solve(ctx, M, meta["outer"], b, inner=meta["inner"], reference_defects=1, **meta["params"])
    finally:
        M.close()
    assert r.converged == meta["converged"]
    strict, worst = check_history(r.hist_iter, r.hist_err, g["hist_iter"], g["hist_err"], g["envelope"], r.loop,
                                  meta["loop"], loop_range(meta))
    assert round(r.true_res_log10, 1) == pytest.approx(meta["true_res_log10"], abs=0.21)
