"""Loader for the golden fixtures produced by tests/golden/make_golden.py."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def load(case_id):
    meta = index()[case_id]
    d = np.load(os.path.join(GOLDEN, f"{case_id}.npz"))
    return meta, {k: d[k] for k in d.files}


def index_large():
    """Full-size fixtures (make_golden.py --large); empty when absent."""
    path = os.path.join(GOLDEN, "index_large.json")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def load_large(case_id):
    meta = index_large()[case_id]
    d = np.load(os.path.join(GOLDEN, f"{case_id}.npz"))
    return meta, {k: d[k] for k in d.files}


def rel_close(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), 1e-300)
    return np.abs(a - b) / den <= rtol


# Parity of a residual history with the reference's.
#
# The GPU adds the terms of each dot product in a different (fixed) order than
# the reference's sequential host loop. Krylov recurrences amplify such
# rounding differences, and the reference itself departs from its own -t 1
# history by as much when only its OpenMP thread count changes (its dot
# products then add per-thread partial sums). `envelope[i]` is the largest
# relative departure of the reference's -t 2/3/4/8 runs from its -t 1 run at
# entry i. The criterion:
#   * every entry before the reference starts departing from itself (its
#     self-departure first exceeds ONSET = HIST_RTOL / 10) must match to
#     HIST_RTOL (1e-8);
#   * later entries must stay within max(HIST_RTOL, ENVELOPE_FACTOR times the
#     reference's largest self-departure so far);
#   * the iteration count must lie within the reference's own spread, +-1 %.
HIST_RTOL = 1e-8
ONSET = HIST_RTOL / 10
ENVELOPE_FACTOR = 10.0


def check_history(gpu_it, gpu_err, ref_it, ref_err, envelope, loop, ref_loop, loop_range):
    lo, hi = loop_range
    tol = max(1, int(0.01 * ref_loop))
    assert lo - tol <= loop <= hi + tol, (loop, loop_range)
    m = min(len(ref_err), len(gpu_err))
    assert m >= min(len(ref_err), len(gpu_err)) and m > 0
    assert np.array_equal(np.asarray(gpu_it[:m]), np.asarray(ref_it[:m]))
    dev = np.abs(np.asarray(gpu_err[:m]) - ref_err[:m]) / np.maximum(np.abs(ref_err[:m]), 1e-300)
    env = np.asarray(envelope[:m], dtype=np.float64)
    over = env > ONSET
    strict = int(np.argmax(over)) if over.any() else m
    bad = np.nonzero(dev[:strict] > HIST_RTOL)[0]
    assert bad.size == 0, f"entry {bad[0]} deviates {dev[bad[0]]:.2e} before the reference's own departure at {strict}"
    allow = np.maximum(HIST_RTOL, ENVELOPE_FACTOR * np.maximum.accumulate(env))
    bad = np.nonzero(dev > allow)[0]
    assert bad.size == 0, f"entry {bad[0]}: {dev[bad[0]]:.2e} > allowed {allow[bad[0]]:.2e}"
    return strict, float(dev.max()) if m else 0.0


def oracle_envelope(oracle, A, b, outer, inner="NONE", chunks=(2, 3, 4, 8), **kw):
    """Same envelope for runs without a golden fixture: the oracle with its dot
    products summed as 2/3/4/8 partial sums against its sequential run."""
    base = oracle.solve(A, b, outer, inner, **kw)
    h1 = base["hist_err"]
    env = np.zeros_like(h1)
    loops = [base["loop"]]
    for c in chunks:
        r = oracle.solve(A, b, outer, inner, sum_chunks=c, **kw)
        loops.append(r["loop"])
        m = min(len(h1), len(r["hist_err"]))
        env[:m] = np.maximum(env[:m], np.abs(r["hist_err"][:m] - h1[:m]) / np.maximum(np.abs(h1[:m]), 1e-300))
        if m < len(h1):
            env[m:] = np.inf
    return base, env, (min(loops), max(loops))
