"""Row-split plan for solves over several GPUs (CPU only): the partition, the
column windows and the halo exchange, checked by running the split SpMV on
the CPU, in one process and as two gloo ranks exchanging their halos."""
import os
import socket

import numpy as np
import pytest

from solver_cpp_b200.matrices import config_problem


def _local_rows(A, r0, r1, lo, hi):
    """Rows r0..r1-1 with columns shifted into the window [lo, hi), as scipy CSR."""
    import scipy.sparse as sp

    j0, j1 = A.ptr[r0], A.ptr[r1]
    return sp.csr_matrix((A.val[j0:j1], A.col[j0:j1] - lo, A.ptr[r0:r1 + 1] - j0), shape=(r1 - r0, hi - lo))


def test_partition_rows(ks):
    assert list(ks.partition_rows(11, 2)) == [0, 6, 11]  # ceil(n/2), the reference's two-GPU split
    rs = ks.partition_rows(160 ** 3, 8, 160 ** 2)
    assert rs[0] == 0 and rs[-1] == 160 ** 3 and np.all(np.diff(rs) == 20 * 160 ** 2)
    rs = ks.partition_rows(1000, 7, 64)
    assert np.all(np.diff(rs) >= 0) and np.all(rs[1:-1] % 64 == 0)
    rs = ks.partition_rows(5, 8)  # more ranks than rows: some blocks are empty
    assert rs[0] == 0 and rs[-1] == 5 and np.all(np.diff(rs) >= 0)
    with pytest.raises(ks.KrylovError):
        ks.partition_rows(0, 2)


def test_window_is_one_plane_each_side(ks):
    g = 12
    A, _, _ = config_problem("poisson3d", g)
    rs = ks.partition_rows(A.n, 3, g * g)
    for p in range(3):
        lo, hi = ks.halo_window(A, rs[p], rs[p + 1])
        assert lo == max(0, rs[p] - g * g) and hi == min(A.n, rs[p + 1] + g * g)


@pytest.mark.parametrize("prob,nranks,align", [("poisson3d", 3, 144), ("convdiff3d", 4, 1), ("varcoef2d", 2, 1),
                                               ("poisson2d", 5, 7)])
def test_split_spmv_with_plan_equals_global(ks, prob, nranks, align):
    A, _, _ = config_problem(prob, 12 if "3d" in prob else 40)
    x = np.random.default_rng(3).standard_normal(A.n)
    rs = ks.partition_rows(A.n, nranks, align)
    win = [ks.halo_window(A, rs[p], rs[p + 1]) for p in range(nranks)]
    lo = [w[0] for w in win]
    hi = [w[1] for w in win]
    plans = [ks.halo_plan(rs, lo, hi, p) for p in range(nranks)]
    for p in range(nranks):
        for q in range(nranks):
            assert tuple(plans[p]["send"][q]) == tuple(plans[q]["recv"][p])
    y = np.zeros(A.n)
    for p in range(nranks):
        xe = np.full(hi[p] - lo[p], np.nan)
        xe[rs[p] - lo[p]:rs[p + 1] - lo[p]] = x[rs[p]:rs[p + 1]]
        for q in range(nranks):  # what q sends to p, from q's own rows
            a, b = plans[p]["recv"][q]
            sa, sb = plans[q]["send"][p]
            assert (a, b) == (sa, sb)
            xe[a - lo[p]:b - lo[p]] = x[sa:sb]
        y[rs[p]:rs[p + 1]] = _local_rows(A, rs[p], rs[p + 1], lo[p], hi[p]) @ xe
    assert np.array_equal(y, A.to_scipy() @ x)


def _gloo_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist

    import solver_cpp_b200 as ks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A, _, _ = config_problem("poisson3d", 10)
        x = np.random.default_rng(9).standard_normal(A.n)
        rs = ks.partition_rows(A.n, world, 100)
        r0, r1 = int(rs[rank]), int(rs[rank + 1])
        lo, hi = ks.halo_window(A, r0, r1)
        wins = [None] * world
        dist.all_gather_object(wins, (lo, hi))
        plan = ks.halo_plan(rs, [w[0] for w in wins], [w[1] for w in wins], rank)
        xe = torch.full((hi - lo,), float("nan"), dtype=torch.float64)
        xe[r0 - lo:r1 - lo] = torch.from_numpy(x[r0:r1])
        reqs = []
        for peer in range(world):
            if peer == rank:
                continue
            a, b = plan["send"][peer]
            if b > a:
                reqs.append(dist.isend(torch.from_numpy(x[a:b].copy()), peer))
            a, b = plan["recv"][peer]
            if b > a:
                buf = torch.empty(b - a, dtype=torch.float64)
                dist.recv(buf, peer)
                xe[a - lo:b - lo] = buf
        for r in reqs:
            r.wait()
        y = _local_rows(A, r0, r1, lo, hi) @ xe.numpy()
        ys = [None] * world
        dist.all_gather_object(ys, y)
        if rank == 0:
            q.put(bool(np.array_equal(np.concatenate(ys), A.to_scipy() @ x)))
    finally:
        dist.destroy_process_group()


def test_split_spmv_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=10) is True
