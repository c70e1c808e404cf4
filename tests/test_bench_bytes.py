"""CPU: the algorithmic byte counts bench.py divides by for its roofline
(SpMV bytes per launch on the diagonal copy and on CSR), against the figures
the kernel summaries quote, and the layout names it keys DRAM traffic by."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_spmv_bytes():
    b = _bench()
    n4, nnz4 = 160 ** 3, 28_518_400  # C4
    n2, nnz2 = 128 ** 3, 14_581_760  # C2
    # diagonal copy: nd n s_val + n mask bytes + x read + y written
    assert b.spmv_bytes(n4, nnz4, "fp32", 2, 7) == 151_552_000
    assert b.spmv_bytes(n4, nnz4, "fp64", 2, 7) == 299_008_000
    assert b.spmv_bytes(n4, nnz4, "bf16", 2, 7) == 94_208_000
    assert b.spmv_bytes(n2, nnz2, "fp64", 2, 7) == 153_092_096
    # CSR: values + column indices + row offsets + x + y
    assert b.spmv_bytes(n4, nnz4, "fp32", 2) == 220_262_404
    assert b.spmv_bytes(n4, nnz4, "fp64", 2) == 367_104_004
    assert b.spmv_bytes(n4, nnz4, "fp64", 4) == 424_140_804
    assert b.spmv_bytes(n2, nnz2, "fp64", 4) == 216_924_164


def test_layout_key():
    b = _bench()
    assert b.layout_key({"diagonals": 7, "index_bytes": 2}) == "d7"
    assert b.layout_key({"diagonals": 0, "index_bytes": 2}) == "i2"
    assert b.layout_key({"diagonals": 0, "index_bytes": 4}) == "i4"
