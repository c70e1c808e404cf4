"""ctypes binding of the CPU oracle and a runner for the reference binary.

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by the product package.

* :func:`solve` runs the C restatement (``liboracle.so``, built by
  ``make -C oracle oracle``).
* :func:`run_reference` runs the reference's own CPU path (``_ref/Solver``,
  built by ``make -C oracle ref`` from the reference sources) on a CSR problem
  by writing it in the reference's CRS text format and parsing
  ``./output/<NAME>_his.txt``, ``<NAME>_xvec.txt`` and the printed summary.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "Solver")

SOLVERS = {
    "NONE": 0, "CG": 1, "BICG": 2, "CR": 3, "GCR": 4, "GMRES": 5,
    "KSKIPCG": 6, "KSKIPCR": 7, "KSKIPBICG": 8, "VPCG": 9, "VPBICG": 10,
    "VPCR": 11, "VPGCR": 12, "VPGMRES": 13,
}


class _Mat(C.Structure):
    _fields_ = [
        ("n", C.c_long),
        ("ptr", C.POINTER(C.c_int)), ("col", C.POINTER(C.c_int)), ("val", C.POINTER(C.c_double)),
        ("tptr", C.POINTER(C.c_int)), ("tcol", C.POINTER(C.c_int)), ("tval", C.POINTER(C.c_double)),
    ]


class _Params(C.Structure):
    _fields_ = [
        ("outer", C.c_int), ("inner", C.c_int),
        ("outer_maxloop", C.c_long), ("outer_eps", C.c_double), ("outer_restart", C.c_long),
        ("outer_kskip", C.c_int), ("outer_fix", C.c_int),
        ("inner_maxloop", C.c_long), ("inner_eps", C.c_double), ("inner_restart", C.c_long),
        ("inner_kskip", C.c_int), ("inner_fix", C.c_int),
        ("fix_kskipcg", C.c_int), ("fix_gmres_assembly", C.c_int), ("sum_chunks", C.c_int),
    ]


class _Report(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("loop", C.c_long), ("hist_len", C.c_long),
        ("true_res_log10", C.c_double), ("spmv", C.c_long),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = C.CDLL(LIB_PATH)
        L.oracle_solve.argtypes = [C.POINTER(_Mat), C.POINTER(_Params), C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_long, C.POINTER(_Report)]
        L.oracle_solve.restype = C.c_int
        L.oracle_default_params.argtypes = [C.POINTER(_Params)]
        for nm in ("oracle_spmv", "oracle_spmv_t"):
            getattr(L, nm).argtypes = [C.POINTER(_Mat), C.c_void_p, C.c_void_p]
        L.oracle_dot.argtypes = [C.c_long, C.c_void_p, C.c_void_p]
        L.oracle_dot.restype = C.c_double
        L.oracle_norm2.argtypes = [C.c_long, C.c_void_p]
        L.oracle_norm2.restype = C.c_double
        L.oracle_matpow.argtypes = [C.POINTER(_Mat), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.oracle_gram_cg.argtypes = [C.c_long, C.c_int] + [C.c_void_p] * 7
        L.oracle_gram_bicg.argtypes = [C.c_long, C.c_int] + [C.c_void_p] * 8
        L.oracle_check_error.argtypes = [C.POINTER(_Mat), C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_check_error.restype = C.c_double
        L.oracle_pattern_grad.argtypes = [C.POINTER(_Mat), C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Problem:
    """Keeps the CSR arrays (and the transpose) alive for the C structs."""

    def __init__(self, A, with_transpose=True):
        from solver_cpp_b200.matrices import transpose

        self.A = A
        self.ptr = np.ascontiguousarray(A.ptr, dtype=np.int32)
        self.col = np.ascontiguousarray(A.col, dtype=np.int32)
        self.val = np.ascontiguousarray(A.val, dtype=np.float64)
        m = _Mat()
        m.n = A.n
        m.ptr = self.ptr.ctypes.data_as(C.POINTER(C.c_int))
        m.col = self.col.ctypes.data_as(C.POINTER(C.c_int))
        m.val = self.val.ctypes.data_as(C.POINTER(C.c_double))
        if with_transpose:
            T = transpose(A)
            self.T = T
            self.tptr, self.tcol, self.tval = T.ptr, T.col, T.val
            m.tptr = self.tptr.ctypes.data_as(C.POINTER(C.c_int))
            m.tcol = self.tcol.ctypes.data_as(C.POINTER(C.c_int))
            m.tval = self.tval.ctypes.data_as(C.POINTER(C.c_double))
        self.mat = m


def default_params():
    p = _Params()
    lib().oracle_default_params(C.byref(p))
    return p


def make_params(outer, inner="NONE", **kw):
    """Parameters named after the reference's flags: L E R K F (outer) and
    l e r k f (inner), plus fix_kskipcg / fix_gmres_assembly."""
    p = default_params()
    p.outer = SOLVERS[outer.upper()]
    p.inner = SOLVERS[inner.upper()]
    names = {"L": "outer_maxloop", "E": "outer_eps", "R": "outer_restart", "K": "outer_kskip",
             "F": "outer_fix", "l": "inner_maxloop", "e": "inner_eps", "r": "inner_restart",
             "k": "inner_kskip", "f": "inner_fix"}
    for k, v in kw.items():
        setattr(p, names.get(k, k), v)
    return p


def solve(problem, b, outer, inner="NONE", hist_cap=200000, **kw):
    """Run the oracle. Returns dict(status, loop, hist_iter, hist_err, x,
    true_res_log10, spmv)."""
    if not isinstance(problem, Problem):
        problem = Problem(problem)
    p = make_params(outer, inner, **kw)
    n = problem.A.n
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n)
    hi = np.zeros(hist_cap, dtype=np.int64)
    he = np.zeros(hist_cap)
    rep = _Report()
    lib().oracle_solve(C.byref(problem.mat), C.byref(p), _p(b), _p(x), _p(hi), _p(he), hist_cap, C.byref(rep))
    m = min(rep.hist_len, hist_cap)
    return {"status": rep.status, "loop": rep.loop, "hist_iter": hi[:m].copy(), "hist_err": he[:m].copy(),
            "x": x, "true_res_log10": rep.true_res_log10, "spmv": rep.spmv}


def spmv(problem, x, transpose=False):
    if not isinstance(problem, Problem):
        problem = Problem(problem)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(problem.A.n)
    fn = lib().oracle_spmv_t if transpose else lib().oracle_spmv
    fn(C.byref(problem.mat), _p(x), _p(y))
    return y


def dot(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib().oracle_dot(x.shape[0], _p(x), _p(y))


def matpow(problem, r, p, k):
    n = problem.A.n
    Ar = np.zeros((2 * k + 1, n))
    Ap = np.zeros((2 * k + 2, n))
    lib().oracle_matpow(C.byref(problem.mat), _p(np.ascontiguousarray(r)), _p(np.ascontiguousarray(p)), k,
                        _p(Ar), _p(Ap))
    return Ar, Ap


def gram_cg(r, p, Ar, Ap, k):
    n = r.shape[0]
    d, e, z = np.zeros(2 * k), np.zeros(2 * k + 1), np.zeros(2 * k + 2)
    lib().oracle_gram_cg(n, k, _p(Ar), _p(Ap), _p(r), _p(p), _p(d), _p(e), _p(z))
    return d, e, z


def gram_bicg(rs, ps, Ar, Ap, k):
    n = rs.shape[0]
    t, e, r_, f = np.zeros(2 * k), np.zeros(2 * k + 1), np.zeros(2 * k + 1), np.zeros(2 * k + 2)
    lib().oracle_gram_bicg(n, k, _p(Ar), _p(Ap), _p(rs), _p(ps), _p(t), _p(e), _p(r_), _p(f))
    return t, e, r_, f


def pattern_grad(problem, lam, x):
    g = np.zeros(problem.A.nnz)
    lib().oracle_pattern_grad(C.byref(problem.mat), _p(np.ascontiguousarray(lam)), _p(np.ascontiguousarray(x)), _p(g))
    return g


# --------------------------------------------------------------------------
# The reference binary
# --------------------------------------------------------------------------

_OUTNAME = {"CG": "CG", "CR": "CR", "BICG": "BICG", "GCR": "GCR", "GMRES": "GMRES",
            "KSKIPCG": "KSKIPCG", "KSKIPBICG": "KSKIPBICG", "VPCG": "VPCG", "VPCR": "VPCR",
            "VPGCR": "VPGCR", "VPGMRES": "VPGMRES"}


def reference_available():
    return os.path.exists(REF_BIN)


def run_reference(A, b, args, threads=1, workdir=None, name="prob", timeout=3600, keep_x=True,
                  run_dir=None):
    """Run the reference CPU binary on (A, b) with extra CLI ``args`` (a list,
    e.g. ``["-S", "cg", "-E", "1e-10"]``). Returns a dict with the history,
    x, the printed loop/time/true residual and the verdict.

    ``A`` may be None when ``workdir`` already holds the CRS files of
    ``name``. ``run_dir`` (default ``<workdir>/run``) receives ``./output``;
    give concurrent runs of one matrix their own."""
    from solver_cpp_b200.matrices import write_crs

    own = workdir is None
    wd = tempfile.mkdtemp(prefix="ref_") if own else workdir
    mdir = os.path.join(wd, "Matrix", "CRS", name)
    if not os.path.exists(os.path.join(mdir, "ColVal.txt")):
        write_crs(mdir, A, b)
    run_dir = run_dir or os.path.join(wd, "run")
    os.makedirs(os.path.join(run_dir, "output"), exist_ok=True)
    cmd = [REF_BIN, "-p", wd, "-m", name, "-t", str(threads)] + list(args)
    proc = subprocess.run(cmd, cwd=run_dir, capture_output=True, text=True, timeout=timeout)
    out = proc.stdout
    solver = args[args.index("-S") + 1].upper()
    res = {"stdout": out, "stderr": proc.stderr, "returncode": proc.returncode}
    m = re.search(r"\|b-ax\|2/\|b\|2 = (\S+)", out)
    res["true_res_log10"] = float(m.group(1)) if m else None
    m = re.search(r"^loop = (-?\d+)", out, re.M)
    res["loop"] = int(m.group(1)) if m else None
    m = re.search(r"^time = (\S+)", out, re.M)
    res["time"] = float(m.group(1)) if m else None
    res["converged"] = "not converge" not in out and "converge" in out
    his = os.path.join(run_dir, "output", f"{_OUTNAME.get(solver, solver)}_his.txt")
    if os.path.exists(his) and os.path.getsize(his) > 0:
        h = np.loadtxt(his, ndmin=2)
        res["hist_iter"] = h[:, 0].astype(np.int64)
        res["hist_err"] = h[:, 1]
    else:
        res["hist_iter"] = np.zeros(0, dtype=np.int64)
        res["hist_err"] = np.zeros(0)
    xf = os.path.join(run_dir, "output", f"{_OUTNAME.get(solver, solver)}_xvec.txt")
    if keep_x and os.path.exists(xf) and os.path.getsize(xf) > 0:
        res["x"] = np.loadtxt(xf, ndmin=2)[:, 1]
    if own:
        import shutil

        shutil.rmtree(wd, ignore_errors=True)
    return res
