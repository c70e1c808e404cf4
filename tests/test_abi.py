"""CPU: the C-ABI library loads and exports every entry point the header
declares; host-only entry points (defaults, status strings, CRS text I/O)
work without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "krylov_sm100.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ks_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(ks):
    lib = ks.lib()
    syms = declared_symbols()
    assert len(syms) >= 40
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    from solver_cpp_b200 import _abi

    bound = {name for name, _, _ in _abi.SIGNATURES}
    assert set(syms) == bound, set(syms) ^ bound


def test_abi_version_and_status_strings(ks):
    from solver_cpp_b200 import _abi

    lib = ks.lib()
    # 2: ks_params.x_update; 3: cluster_solve; 4: inner_fast, true_residual, profile, x_ref
    assert lib.ks_abi_version() == _abi.ABI_VERSION == 4
    assert b"not converged" in lib.ks_status_string(2)
    assert b"not implemented" in lib.ks_status_string(99)


def test_params_default_match_reference(ks):
    """solver_collection.cpp:26-49 defaults."""
    p = ks.make_params()
    assert (p.outer_maxloop, p.outer_eps, p.outer_restart, p.outer_kskip, p.outer_fix) == (10000, 1e-8, 1000, 2, 2)
    assert (p.inner_maxloop, p.inner_eps, p.inner_restart, p.inner_kskip, p.inner_fix) == (50, 1e-1, 1000, 2, 2)
    assert p.inner_precision == 0 and p.reference_defects == 0
    q = ks.make_params(L=5, E=1e-3, R=7, K=3, F=1, l=9, e=0.5, r=4, k=1, f=0, inner_precision="bf16")
    assert (q.outer_maxloop, q.outer_restart, q.inner_restart, q.inner_precision) == (5, 7, 4, 2)


def test_solver_codes_match_reference_enum(ks):
    # solver_collection.hpp:7-24
    names = ["NONE", "CG", "BICG", "CR", "GCR", "GMRES", "KSKIPCG", "KSKIPCR", "KSKIPBICG", "VPCG", "VPBICG",
             "VPCR", "VPGCR", "VPGMRES"]
    assert [ks.SOLVERS[n] for n in names] == list(range(14))


def test_crs_roundtrip_through_library_and_reference_format(ks, tmp_path):
    from solver_cpp_b200.matrices import config_problem, read_crs

    A, b, _ = config_problem("varcoef2d", 9)
    x = np.random.default_rng(0).standard_normal(A.n)
    d = str(tmp_path / "m")
    ks.crs_write(d, A, b, x)
    A2, b2, x2 = ks.crs_read(d)
    assert np.array_equal(A2.ptr, A.ptr) and np.array_equal(A2.col, A.col)
    assert np.array_equal(A2.val, A.val) and np.array_equal(b2, b) and np.array_equal(x2, x)
    A3, b3, x3 = read_crs(d)  # numpy reader agrees
    assert np.array_equal(A3.val, A.val) and np.array_equal(b3, b)
    head = open(os.path.join(d, "Ptr.txt")).readline().split()
    assert head == [str(A.n), str(A.n), str(A.nnz)]


@pytest.mark.parametrize("threads", ["1", "3", "7", "64"])
def test_crs_parallel_parse_any_whitespace(ks, tmp_path, monkeypatch, threads):
    """The reader parses chunks of the text in parallel (KS_IO_THREADS forces
    the chunk count on a small file). Records may be separated by any
    whitespace, as fscanf reads them: several records on one line, blank
    lines, tabs, CRLF. Every chunk count gives the written values bit for
    bit; a file one record short, or with a token that does not parse, is an
    I/O error."""
    from solver_cpp_b200.matrices import config_problem

    monkeypatch.setenv("KS_IO_THREADS", threads)
    A, b, _ = config_problem("varcoef3d", 7)
    x = np.random.default_rng(1).standard_normal(A.n)
    d = str(tmp_path / "m")
    ks.crs_write(d, A, b, x)
    seps = [" ", "\n", "\t", "\r\n", "\n\n", "  \t "]
    rng = np.random.default_rng(2)

    def rewrite(name):
        path = os.path.join(d, name)
        lines = open(path).read().split("\n")
        toks = " ".join(lines[1:]).split()
        out = [lines[0]]
        body = "".join(t + seps[rng.integers(len(seps))] for t in toks)
        open(path, "w").write(out[0] + "\n" + body)

    for name in ("ColVal.txt", "Ptr.txt", "bx.txt"):
        rewrite(name)
    A2, b2, x2 = ks.crs_read(d)
    assert np.array_equal(A2.ptr, A.ptr) and np.array_equal(A2.col, A.col)
    assert np.array_equal(A2.val, A.val) and np.array_equal(b2, b) and np.array_equal(x2, x)
    # one record short / a token that does not parse
    path = os.path.join(d, "ColVal.txt")
    txt = open(path).read()
    open(path, "w").write(txt.rsplit(None, 2)[0])
    with pytest.raises(Exception):
        ks.crs_read(d)
    open(path, "w").write(txt.replace(txt.split()[10], "x1", 1))
    with pytest.raises(Exception):
        ks.crs_read(d)


def test_crs_header_mismatch_is_io_error(ks, tmp_path):
    from solver_cpp_b200.matrices import poisson2d

    A = poisson2d(4)
    d = str(tmp_path / "bad")
    ks.crs_write(d, A, np.ones(A.n))
    with open(os.path.join(d, "bx.txt"), "r+") as f:
        f.write("99")
    n, nnz = C.c_int64(), C.c_int64()
    st = ks.lib().ks_crs_read_header(d.encode(), C.byref(n), C.byref(nnz))
    assert st == 10  # KS_IO_ERROR ("Three N in files is not same")


def test_ctx_without_device_reports_no_device(ks):
    lib = ks.lib()
    if lib.ks_device_count() > 0:
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert lib.ks_ctx_create(0, C.byref(h)) == 9  # KS_NO_DEVICE
    with pytest.raises(ks.KrylovError):
        ks.Context(0)


def test_bench_reference_arm_json(ks, tmp_path):
    """bench.py --impl reference on the 64^2 CG case: the reference's own CPU
    binary (built from its sources when the package was built) runs a bounded
    sample and the line carries the contract's keys."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--workload", "c1_cg",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference"
    if "unavailable" in d:
        pytest.skip(d["unavailable"])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "cpu_baseline", "e2e",
              "config"):
        assert k in d, k
    # the value is one complete solve of the workload: the reference's 202
    # CG iterations on the 64^2 system, its printed time
    assert d["result"]["loop"] == 202 and d["result"]["converged"]
    assert d["value"] == d["cpu_baseline"]["value"] > 0
    # the reference arm maps no shared object of the product library
    assert not [p for p in d["repo_objects_loaded"] if "libkrylov" in p], d["repo_objects_loaded"]
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference" and d["config"]["workload"] == "c1_cg"
