"""GPU: the allocation-free block dot, ks_block_dot_noalloc.

Callers that cannot allocate device memory at the point of use -- code inside
a CUDA stream capture, applications whose device memory belongs to their own
pool allocator, loops that must stay off the driver allocator -- use this
entry point instead of ks_block_dot. It keeps its reduction scratch in a fixed
device array inside the library, so it must give the same results as the
allocating entry point, call after call, even though every call reuses (and
overwrites) that array. This file is collected last so a failure here leaves
every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the tolerance the other reduction tests use


def _sync():
    import torch

    torch.cuda.synchronize()


def test_noalloc_block_dot_matches_block_dot_twice(ks, ctx):
    lib = ks.lib()
    rng = np.random.default_rng(21)
    n, k = 300_007, 37
    V = rng.standard_normal((k, n))
    w = rng.standard_normal(n)
    VV, WW = ctx.vector(V.ravel()), ctx.vector(w)
    H = ctx.vector(n=64)
    ref = ks.block_dot(VV, n, k, WW)  # the allocating entry point
    np.testing.assert_allclose(ref, V @ w, rtol=RTOL)
    for _ in range(2):  # the second call runs on the scratch the first one left
        H.fill(0.0)
        ctx.synchronize()
        st = lib.ks_block_dot_noalloc(C.c_void_p(VV.device_ptr), n, k, C.c_void_p(WW.device_ptr), n,
                                      C.c_void_p(H.device_ptr), None)
        assert st == 0
        _sync()
        np.testing.assert_allclose(H.numpy()[:k], ref, rtol=RTOL)


def test_noalloc_block_dot_limit(ks, ctx):
    lib = ks.lib()
    n = 1000
    V = ctx.vector(np.ones(65 * n))
    w = ctx.vector(np.ones(n))
    H = ctx.vector(n=65)
    st = lib.ks_block_dot_noalloc(C.c_void_p(V.device_ptr), n, 65, C.c_void_p(w.device_ptr), n,
                                  C.c_void_p(H.device_ptr), None)
    assert st == 5  # KS_BAD_INPUT: above the 64-vector scratch limit
    st = lib.ks_block_dot_noalloc(C.c_void_p(V.device_ptr), n, 64, C.c_void_p(w.device_ptr), n,
                                  C.c_void_p(H.device_ptr), None)
    assert st == 0
    _sync()
    np.testing.assert_allclose(H.numpy()[:64], np.full(64, float(n)), rtol=RTOL)
