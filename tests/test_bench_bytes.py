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
    # diagonal copy: nd n s_val (+ n mask bytes in FP64) + x read + y written
    assert b.spmv_bytes(n4, nnz4, "fp32", 2, 7) == 147_456_000
    assert b.spmv_bytes(n4, nnz4, "fp64", 2, 7) == 299_008_000
    assert b.spmv_bytes(n4, nnz4, "bf16", 2, 7) == 90_112_000
    assert b.spmv_bytes(n2, nnz2, "fp64", 2, 7) == 153_092_096
    # symmetric half: the main and 3 upper diagonals stored
    assert b.spmv_bytes(n4, nnz4, "fp32", 2, 7, 1) == 98_304_000
    assert b.spmv_bytes(n4, nnz4, "bf16", 2, 7, 1) == 65_536_000
    assert b.spmv_bytes(n4, nnz4, "fp64", 2, 7, 1) == 200_704_000
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


def test_onchip_inner_bytes():
    """One launch of the on-chip inner CG at 160^3: per iteration the 4 stored
    FP32 diagonals (16 n), p published (4 n) and the halo of the +-1, +-160,
    +-25600 offsets over 148 CTAs; once 8 n."""
    b = _bench()
    n = 160 ** 3
    info = {"offsets": [-25600, -160, -1, 0, 1, 160, 25600]}
    halo = 2 * (25600 + 160 + 1) * 148
    assert b.onchip_inner_bytes(n, "fp32", 7, 1, info, 20) == 20 * (16 * n + 4 * n + 4 * halo) + 8 * n
    assert b.onchip_inner_bytes(n, "bf16", 7, 1, info, 20) == 20 * (8 * n + 4 * n + 4 * halo) + 8 * n
    # the whole FP64 solve: FP64 values, one mask byte per row, FP64 vectors
    assert b.onchip_inner_bytes(n, "fp64", 7, 1, info, 20) == 20 * (32 * n + n + 8 * n + 8 * halo) + 16 * n
    one = b.onchip_inner_bytes(n, "fp64", 7, 1, info, 20)
    assert b.onchip_whole_bytes("CG", n, 7, 1, info, 20) == one
    assert b.onchip_whole_bytes("CR", n, 7, 1, info, 20) == one + 20 * 16 * n  # x read and written in place
    assert b.onchip_whole_bytes("BICG", n, 7, 1, info, 20) == 2 * one - 16 * n  # A and A^T, b and x once
