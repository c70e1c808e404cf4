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


def rel_close(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), 1e-300)
    return np.abs(a - b) / den <= rtol
