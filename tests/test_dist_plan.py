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


def _halo_exchange(dist, torch, plan, rank, world, v, xe, lo):
    """The engine's exchange before an SpMV (Env::halo): each peer's planned
    range of its own rows lands in this rank's window."""
    reqs = []
    for peer in range(world):
        if peer == rank:
            continue
        a, b = plan["send"][peer]
        if b > a:
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(v[a:b])), peer))
    for peer in range(world):
        if peer == rank:
            continue
        a, b = plan["recv"][peer]
        if b > a:
            buf = torch.empty(b - a, dtype=torch.float64)
            dist.recv(buf, peer)
            xe[a - lo:b - lo] = buf.numpy()
    for r in reqs:
        r.wait()


def _gloo_cg_rank(rank, world, port, q):
    """CG (cg.cpp:148-240) split by rows the way the library splits it: the
    library's plan, a halo exchange before every SpMV, every reduction summed
    over the ranks before its scalar step (with_rank_sums), the stopping test
    on the summed value, so every rank takes the same decisions and the same
    number of collectives."""
    import torch
    import torch.distributed as dist

    import solver_cpp_b200 as ks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = 12
        A, b, _ = config_problem("varcoef3d", g)
        rs = ks.partition_rows(A.n, world, g * g)
        r0, r1 = int(rs[rank]), int(rs[rank + 1])
        lo, hi = ks.halo_window(A, r0, r1)
        wins = [None] * world
        dist.all_gather_object(wins, (lo, hi))
        plan = ks.halo_plan(rs, [w[0] for w in wins], [w[1] for w in wins], rank)
        Aloc = _local_rows(A, r0, r1, lo, hi)

        def allsum(v):
            t = torch.tensor([v], dtype=torch.float64)
            dist.all_reduce(t)
            return float(t.item())

        full_p = np.zeros(A.n)  # only [r0, r1) and the received halo are ever read
        bl = b[r0:r1]
        x = np.zeros(r1 - r0)
        r = bl.copy()
        p = r.copy()
        bnorm = np.sqrt(allsum(float(bl @ bl)))
        rr = allsum(float(r @ r))
        hist, status = [], 2
        for L in range(1, 2001):
            err = np.sqrt(rr) / bnorm
            hist.append(err)
            if err <= 1e-10:
                status = 0
                break
            full_p[r0:r1] = p
            xe = np.full(hi - lo, np.nan)
            xe[r0 - lo:r1 - lo] = p
            _halo_exchange(dist, torch, plan, rank, world, full_p, xe, lo)
            qv = Aloc @ xe
            alpha = rr / allsum(float(p @ qv))
            x += alpha * p
            r -= alpha * qv
            rr2 = allsum(float(r @ r))
            beta, rr = rr2 / rr, rr2
            p = beta * p + r
        xs = [None] * world
        dist.all_gather_object(xs, (status, len(hist), hist, x))
        if rank == 0:
            q.put(xs)
    finally:
        dist.destroy_process_group()


def test_split_cg_over_two_gloo_ranks(oracle):
    """Two CPU ranks run the split CG with the library's plan, exchanges and
    rank-summed reductions: identical histories and verdicts on both ranks,
    the same iteration count as one rank (+-1 %), the same solution."""
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_cg_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    (s0, n0, h0, x0), (s1, n1, h1, x1) = res
    assert s0 == s1 == 0 and n0 == n1 and h0 == h1  # the same decisions, bit for bit
    A, b, _ = config_problem("varcoef3d", 12)
    o = oracle.solve(A, b, "CG", E=1e-10)
    assert o["status"] == 0 and abs(n0 - o["loop"]) <= max(1, 0.01 * o["loop"])
    x = np.concatenate([x0, x1])
    assert np.linalg.norm(x - o["x"]) <= 1e-8 * np.linalg.norm(o["x"])
