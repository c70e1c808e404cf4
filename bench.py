"""Benchmark: time-to-solution of the Krylov hot path on B200.

One step = one complete solve, from b resident in HBM to x resident in HBM, to
a relative residual of 1e-10 (the reference's stopping test on the recurrence
residual; the true FP64 residual is checked and reported).

Workloads (the default is the one the headline metric is quoted on):
  c4_mixed  3D variable-coefficient diffusion 160^3 (n = 4,096,000, nnz =
            28,518,400, ln kappa ~ N(0, 1.5^2) per cell, harmonic-mean faces),
            b ~ N(0,1): VPCG with an FP64 outer loop and an FP32 inner CG of
            exactly 20 iterations, to rel-res 1e-10. The plain FP64 CG on the
            same system is timed beside it.
  c2_cg     3D 7-point Poisson 128^3 (n = 2,097,152), b ~ U(0,1): CG FP64.
  The other entries of WORKLOADS time the remaining methods of the
  configurations (CR and k-skip CG on the Poisson system; BiCG, k-skip BiCG,
  GCR(30) and GMRES(30) on the 128^3 upwind convection-diffusion system;
  VPGMRES and the BF16-valued VPCG on the 160^3 system), one JSON line each.
Inputs are seeded synthetic data with the configurations' shapes; the matrix
(>= 175 MB) is larger than the 126 MB L2, so no L2 flush is needed between
steps.

`--impl reference` times the reference's own CPU path (oracle/_ref/Solver,
built from the reference sources) on the host cores for the same workload.

Multi-GPU (torchrun, N > 1): the rows of the one system are split over the
ranks (contiguous blocks on grid planes; before every SpMV each rank receives
its halo from its neighbours and every reduction is summed over the ranks,
over NCCL): strong scaling, the step time the max over ranks. `--replicas`
instead solves one independent replica per rank (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

def _w(problem, grid, outer, params, inner="NONE", plain=None, ref_args=(), spmv_values="fp64", transpose=False,
       adjoint=False):
    return dict(problem=problem, grid=grid, outer=outer, inner=inner, params=params, plain=plain,
                ref_args=list(ref_args), spmv_values=spmv_values, transpose=transpose, adjoint=adjoint)


_VP20 = dict(E=1e-10, L=10000, l=20, e=1e-30)
WORKLOADS = {
    # headline: VPCG (FP64 outer, FP32 inner CG of 20 iterations) against plain FP64 CG
    "c4_mixed": _w("varcoef3d", 160, "VPCG", dict(_VP20, inner_precision="fp32"), inner="CG",
                   plain=dict(outer="CG", params=dict(E=1e-10, L=20000)),
                   ref_args=["-S", "vpcg", "-s", "cg", "-l", "20", "-e", "1e-30", "-E", "1e-10"],
                   spmv_values="fp32"),
    "c4_mixed_bf16": _w("varcoef3d", 160, "VPCG", dict(_VP20, inner_precision="bf16"), inner="CG",
                        plain=dict(outer="CG", params=dict(E=1e-10, L=20000)), spmv_values="bf16"),
    # VPGMRES (FP64 outer, reference default restart 1000) with the FP32 inner CG,
    # against plain FP64 GMRES with the same restart
    "c4_vpgmres": _w("varcoef3d", 160, "VPGMRES", dict(_VP20, inner_precision="fp32"), inner="CG",
                     plain=dict(outer="GMRES", params=dict(E=1e-10, L=20000)), spmv_values="fp32"),
    # the reference's own CPU-runnable case: 2D Poisson 64^2, b = A*1 + noise
    "c1_cg": _w("poisson2d", 64, "CG", dict(E=1e-10, L=10000), ref_args=["-S", "cg", "-E", "1e-10"]),
    "c2_cg": _w("poisson3d", 128, "CG", dict(E=1e-10, L=10000), ref_args=["-S", "cg", "-E", "1e-10"]),
    "c2_cr": _w("poisson3d", 128, "CR", dict(E=1e-10, L=10000), ref_args=["-S", "cr", "-E", "1e-10"]),
    "c2_kskipcg2": _w("poisson3d", 128, "KSKIPCG", dict(E=1e-10, L=10000, K=2)),
    "c2_kskipcg4": _w("poisson3d", 128, "KSKIPCG", dict(E=1e-10, L=10000, K=4)),
    "c3_bicg": _w("convdiff3d", 128, "BICG", dict(E=1e-10, L=10000), transpose=True,
                  ref_args=["-S", "bicg", "-E", "1e-10"]),
    "c3_kskipbicg2": _w("convdiff3d", 128, "KSKIPBICG", dict(E=1e-10, L=10000, K=2), transpose=True,
                        ref_args=["-S", "kskipbicg", "-K", "2", "-E", "1e-10"]),
    "c3_gcr30": _w("convdiff3d", 128, "GCR", dict(E=1e-10, L=10000, R=30),
                   ref_args=["-S", "gcr", "-R", "30", "-E", "1e-10"]),
    # adjoint gradients of L = 1/2 |x - x*|^2 on the 512^2 systems: one step is
    # the forward solve, the adjoint solve on A^T and the pattern gather
    "c5_adjoint_cg": _w("varcoef2d", 512, "CG", dict(E=1e-12, L=40000), transpose=True, adjoint=True),
    "c5_adjoint_bicg": _w("convdiff2d", 512, "BICG", dict(E=1e-12, L=40000), transpose=True, adjoint=True),
    "c3_gmres30": _w("convdiff3d", 128, "GMRES", dict(E=1e-10, L=10000, R=30),
                     ref_args=["-S", "gmres", "-R", "30", "-E", "1e-10"]),
}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def spmv_bytes(n, nnz, values, index_bytes=4, diagonals=0, symmetric=0):
    """Algorithmic bytes of one SpMV. CSR: values + column indices (int32, or
    the int16 row offsets the library stores when they fit) + int32 row
    offsets + x read once + y written once. Diagonal copy (`diagonals` > 0):
    the stored diagonals' values (zeros where a row has no entry; a symmetric
    matrix stores its main and upper diagonals only) + one mask byte per row
    for FP64 + x read once + y written once."""
    vb = {"fp64": 8, "fp32": 4, "bf16": 2}[values]
    xb = 8 if values == "fp64" else 4
    if diagonals:
        stored = diagonals // 2 + 1 if symmetric else diagonals
        return stored * n * vb + (n if values == "fp64" else 0) + xb * n + xb * n
    return nnz * (vb + index_bytes) + 4 * (n + 1) + xb * n + xb * n


def onchip_inner_bytes(n, values, diagonals, symmetric, info, iters, sms=148):
    """Algorithmic bytes of one launch of the on-chip CG kernel (vectors on
    chip, the matrix read every iteration): per iteration the stored
    diagonals' values (and one mask byte per row with FP64 values), p
    published (one vector) and the neighbouring CTAs' p read (each CTA owns
    ceil(n / sms) rows, and reads the rows an offset reaches beyond its own,
    at each end); once: the right-hand side read and x written. Vectors are
    FP32 for the inner solve of a VP method (fp32 / bf16 values) and FP64 for
    a whole FP64 solve (fp64 values)."""
    vb = {"fp64": 8, "fp32": 4, "bf16": 2}[values]
    xb = 8 if values == "fp64" else 4
    stored = diagonals // 2 + 1 if symmetric else diagonals
    rpc = -(-n // sms)
    offs = info.get("offsets") or []
    halo = sum(min(abs(int(o)), rpc) for o in offs if o) * sms
    mask = n if values == "fp64" else 0
    return iters * (stored * n * vb + mask + xb * n + xb * halo) + 2 * xb * n


def onchip_whole_bytes(method, n, diagonals, symmetric, info, iters, sms=148):
    """Algorithmic bytes of a whole FP64 solve as one on-chip launch: CG as
    onchip_inner_bytes; CR also updates x in place in global memory (read and
    written every iteration, 16 n); BiCG runs two SpMVs per iteration (A and
    A^T: both diagonal copies, masks, published vectors and halos)."""
    one = onchip_inner_bytes(n, "fp64", diagonals, symmetric, info, iters, sms)
    if method == "CR":
        return one + iters * 16 * n
    if method == "BICG":
        return 2 * one - 16 * n
    return one


def layout_key(info):
    """Short name of the layout the SpMV reads: d<diagonals> or i<index bytes>."""
    return f"d{info['diagonals']}" if info.get("diagonals") else f"i{info['index_bytes']}"


def run_ours(args, world, rank, local):
    import torch

    import solver_cpp_b200 as ks
    from solver_cpp_b200.matrices import config_problem

    W = WORKLOADS[args.workload]
    A, b, _ = config_problem(W["problem"], W["grid"])
    n, nnz = A.n, A.nnz
    ctx = ks.Context(local)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    split = world > 1 and not args.replicas
    comm = None
    if split:  # row-split solve of the one system over the ranks (strong scaling), NCCL transport
        import torch.distributed as dist

        if W.get("adjoint"):
            raise SystemExit("the row split does not cover the adjoint workloads (use --replicas)")
        uid = [ks.Comm.unique_id() if rank == 0 else None]
        dist.broadcast_object_list(uid, src=0)
        comm = ks.Comm.nccl(ctx, world, rank, uid[0])
        plane = W["grid"] ** 2 if "3d" in W["problem"] else W["grid"]
        rs = ks.partition_rows(n, world, plane)
        r0, r1 = int(rs[rank]), int(rs[rank + 1])
        M = ks.SplitMatrix(ctx, comm, A, r0, r1, transpose=W["transpose"], fp32=True, bf16=True)
    else:
        r0, r1 = 0, n
        M = ctx.matrix(A, transpose=W["transpose"], fp32=True, bf16=True)
    nl, nnzl = r1 - r0, M.nnz  # this rank's rows and nonzeros
    b_loc = np.ascontiguousarray(b[r0:r1])
    B = ctx.vector(b_loc)
    X = ctx.vector(n=nl)
    launches0 = ks.lib().ks_ctx_launches(ctx.handle)

    adj = None
    if W.get("adjoint"):  # loss 1/2 |x - x*|^2 with x* ~ N(0,1) (seed 6)
        XS = ctx.vector(np.random.default_rng(6).standard_normal(n))
        adj = dict(G=ctx.vector(n=n), GB=ctx.vector(n=n), GV=ctx.vector(n=nnz))

    def one(outer, inner, params):
        r = ks.solve(ctx, M, outer, B, inner=inner, x=X, **params)
        if adj is not None and params is W["params"]:
            # g = x - x*, then the adjoint solve on A^T and the pattern gather
            adj["G"].fill(0.0)
            ks.axpy(1.0, X, adj["G"])
            ks.axpy(-1.0, XS, adj["G"])
            st, _ = ks.adjoint_grad(ctx, M, outer, X, adj["G"], adj["GB"], adj["GV"], **params)
            if st != 0:
                raise RuntimeError(f"adjoint solve status {st}")
        return r

    for _ in range(args.warmup):
        r = one(W["outer"], W["inner"], W["params"])
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    launches_a = ks.lib().ks_ctx_launches(ctx.handle)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        results = []
        for _ in range(args.steps):
            results.append(one(W["outer"], W["inner"], W["params"]))
        ev1.record(stream)
    torch.cuda.synchronize()
    launches_b = ks.lib().ks_ctx_launches(ctx.handle)
    clocks = sampler.stop()
    total_ms = ev0.elapsed_time(ev1)
    total_ms = max_over_ranks(total_ms, world)
    barrier(world)
    res = results[-1]
    ms_per_step = total_ms / args.steps
    value = ms_per_step / 1e3

    # plain FP64 method on the same system (the comparison the metric names)
    plain = None
    if W.get("plain"):
        P = W["plain"]
        one(P["outer"], "NONE", P["params"])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            pr = None
            for _ in range(max(1, args.steps // 2)):
                pr = one(P["outer"], "NONE", P["params"])
            e1.record(stream)
        torch.cuda.synchronize()
        pms = e0.elapsed_time(e1) / max(1, args.steps // 2)
        xp = X.numpy()
        plain = {"method": P["outer"], "seconds": pms / 1e3, "loop": pr.loop, "true_rel_res": pr.true_rel_res,
                 "speedup_mixed_vs_plain": (pms / 1e3) / value}
        # agreement of the mixed solution with the FP64 one
        one(W["outer"], W["inner"], W["params"])
        xm = X.numpy()
        plain["x_rel_diff_vs_fp64"] = float(np.linalg.norm(xm - xp) / np.linalg.norm(xp))

    peak, peak_kind = load_peaks()
    minfo = M.info()
    ib, nd, sym = minfo["index_bytes"], minfo["diagonals"], minfo.get("dia_symmetric", 0)
    if nd:  # the diagonals' offsets col - row, from the host matrix
        rows = np.repeat(np.arange(A.n, dtype=np.int64), np.diff(A.ptr))
        minfo["offsets"] = [int(o) for o in np.unique(A.col.astype(np.int64) - rows)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")  # larger than the 126 MB L2

    def time_launches(fn, reps=50, cold=False, clean=True):
        """CUDA-event time of one launch on the solve's stream: back to back, or
        each launch after an L2 flush (cold; `l2_flush`)."""
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if not cold:
            with torch.cuda.stream(stream):
                e0.record(stream)
                for _ in range(reps):
                    fn()
                e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps
        tot = 0.0
        for _ in range(reps):
            with torch.cuda.stream(stream):
                l2_flush(flush, clean)
                e0.record(stream)
                fn()
                e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / reps

    # The SpMV alone with the workload's value precision (and the FP64 one of
    # an outer loop): back to back, and cold
    spmv = {}
    for vals in [W["spmv_values"]] + (["fp64"] if W["spmv_values"] != "fp64" else []):
        dt = ks.FP64 if vals == "fp64" else ks.FP32
        xs = ctx.vector(np.random.default_rng(0).standard_normal(nl), dtype=dt)
        ys = ctx.vector(n=nl, dtype=dt)
        vcode = {"fp64": ks.FP64, "fp32": ks.FP32, "bf16": ks.BF16}[vals]
        fn = lambda: ks.spmv(M, xs, ys, values=vcode)  # noqa: E731
        warm, cold = time_launches(fn), time_launches(fn, reps=20, cold=True)
        dirty = time_launches(fn, reps=20, cold=True, clean=False)
        alg = spmv_bytes(nl, nnzl, vals, ib, nd, sym)
        spmv[vals] = {"alg_bytes": alg, "launch_ms": round(warm, 5), "launch_ms_cold": round(cold, 5),
                      "gbs": round(alg / (warm / 1e3) / 1e9, 1), "frac": round(alg / (warm / 1e3) / 1e9 / peak, 4),
                      "frac_cold": round(alg / (cold / 1e3) / 1e9 / peak, 4),
                      "launch_ms_cold_dirty": round(dirty, 5),
                      "frac_cold_dirty": round(alg / (dirty / 1e3) / 1e9 / peak, 4)}
        xs.close()
        ys.close()

    # In the solve: one solve with per-class device times
    prof = ks.solve(ctx, M, W["outer"], B, inner=W["inner"], x=X, profile=1, **W["params"]).report
    vals = W["spmv_values"]
    inner_calls = res.inner_calls
    onchip_inner = W["inner"] != "NONE" and prof["n_mv_low"] > 0 and prof["n_mv_low"] <= inner_calls + 1
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if onchip_inner:
        # the dominant kernel: one inner solve of `l` CG iterations on chip
        iters = int(W["params"]["l"])
        per_launch_ms = prof["t_mv_low"] / max(1, prof["n_mv_low"]) * 1e3
        alg = onchip_inner_bytes(nl, vals, nd, sym, minfo, iters)
        if os.path.exists(tf):
            traffic = json.load(open(tf)).get(f"{args.workload}:onchip_inner:{vals}")
        roofline = {"bound": "hbm", "achieved": round(alg / (per_launch_ms / 1e3) / 1e9, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(alg / (per_launch_ms / 1e3) / 1e9 / peak, 4), "traffic": traffic,
                    "kernel": f"k_cg_onchip (one inner CG solve of {iters} iterations, vectors on chip, "
                              f"{vals} values)",
                    "alg_bytes_per_launch": alg, "launch_ms": round(per_launch_ms, 5),
                    "us_per_inner_iteration": round(per_launch_ms * 1e3 / iters, 3),
                    "timed": "in the solve (CUDA events around each launch, profile=1); each launch follows "
                             "the outer iteration's kernels, which stream ~600 MB through L2, so this is "
                             "also the cold figure (frac_cold)", "peak_kind": peak_kind}
        roofline["frac_cold"] = roofline["frac"]
    elif (W["inner"] == "NONE" and W["outer"] in ("CG", "CR", "BICG") and prof["n_mv"] == 1
          and prof["n_dot"] == 0):
        # the whole FP64 solve as one on-chip launch (profiled as one SpMV-class launch)
        iters = max(1, int(res.loop) - 1)  # the stopping test at the top of iteration `loop`
        launch_ms = prof["t_mv"] * 1e3
        alg = onchip_whole_bytes(W["outer"], nl, nd, sym, minfo, iters)
        kname = {"CG": "k_cg_onchip", "CR": "k_cr_onchip", "BICG": "k_bicg_onchip"}[W["outer"]]
        if os.path.exists(tf):
            traffic = json.load(open(tf)).get(f"{args.workload}:onchip_whole:fp64")
        roofline = {"bound": "hbm", "achieved": round(alg / (launch_ms / 1e3) / 1e9, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(alg / (launch_ms / 1e3) / 1e9 / peak, 4), "traffic": traffic,
                    "kernel": f"{kname} (the whole {W['outer']} solve, {iters} iterations, vectors on chip, fp64)",
                    "alg_bytes_per_launch": alg, "launch_ms": round(launch_ms, 5),
                    "us_per_iteration": round(launch_ms * 1e3 / max(1, iters), 3),
                    "timed": "in the solve (CUDA events around the launch, profile=1)", "peak_kind": peak_kind}
    else:
        w = spmv[vals]
        if os.path.exists(tf):
            traffic = json.load(open(tf)).get(f"{args.workload}:spmv:{vals}")
        roofline = {"bound": "hbm", "achieved": w["gbs"], "peak": peak, "unit": "GB/s", "frac": w["frac"],
                    "frac_cold": w["frac_cold"], "traffic": traffic, "kernel": f"spmv_{vals}",
                    "alg_bytes_per_launch": w["alg_bytes"], "launch_ms": w["launch_ms"],
                    "timed": "alone, back to back (frac) and after an L2 flush that leaves only clean lines "
                             "(frac_cold; frac_cold_dirty in spmv: after a write-only flush, whose dirty lines "
                             "the launch writes back)", "peak_kind": peak_kind}
    roofline["layout"] = layout_key(minfo) + ("s" if sym else "")
    roofline["spmv"] = spmv
    roofline["in_solve_seconds"] = {k: round(prof[k], 6) for k in ("t_mv", "t_dot", "t_other", "t_memset",
                                                                     "t_mv_low")}
    roofline["in_solve_launches"] = {k: int(prof[k]) for k in ("n_mv", "n_dot", "n_other", "n_memset",
                                                                "n_mv_low")}
    flush = None

    # end to end through the public host API: pinned b -> device -> x -> host
    e2e = None
    if not args.no_e2e and adj is None:
        bh = torch.from_numpy(b_loc).pin_memory().numpy()
        xh = torch.empty(nl, dtype=torch.float64).pin_memory().numpy()
        import ctypes as C

        p = ks.make_params(**W["params"])
        rep = ks._abi.Report()
        hi = np.zeros(W["params"]["L"] + 2, dtype=np.int64)
        he = np.zeros(W["params"]["L"] + 2)
        L = ks.lib()
        oc, ic = ks.SOLVERS[W["outer"]], ks.SOLVERS[W["inner"]]
        for _ in range(1):
            L.ks_solve_host(ctx.handle, M.handle, oc, ic, C.byref(p), bh.ctypes.data, xh.ctypes.data,
                            hi.ctypes.data, he.ctypes.data, hi.shape[0], C.byref(rep))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                L.ks_solve_host(ctx.handle, M.handle, oc, ic, C.byref(p), bh.ctypes.data, xh.ctypes.data,
                                hi.ctypes.data, he.ctypes.data, hi.shape[0], C.byref(rep))
            e1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
        e2e = {"value": ems / 1e3, "unit": "s", "h2d_bytes_per_step": 8 * nl,
               "d2h_bytes_per_step": 8 * nl + 16 * int(rep.hist_len) + 64}

    # CG on up to 32768 rows runs as one thread-block-cluster launch: its time
    # per iteration (device events around the solve, from the report)
    if W["outer"] == "CG" and not split and nl <= 32768 and adj is None and res.loop > 1:
        roofline["solve_kernel"] = {
            "kernel": "k_cg_resident (whole solve, one thread-block cluster)",
            "solve_ms": round(res.solve_seconds * 1e3, 4),
            "us_per_iteration": round(res.solve_seconds * 1e6 / (res.loop - 1), 3),
            "bound": "latency of the two cross-SM reductions per iteration (inputs in L1 / shared memory)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and adj is None:
        cpu = cpu_baseline_reference(A, b, W, res)

    out = {
        "metric": "time-to-solution at FP64 rel-res 1e-10 (mixed vs plain FP64 GPU); SpMV HBM GB/s",
        "value": round(value, 6), "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4), "higher_is_better": False,
        "scaling": "strong" if split else "weak",
        "vs_baseline": None, "dtype": ("f64 outer / " + {"fp32": "f32", "bf16": "f32 with bf16 values"}[
            W["params"]["inner_precision"]] + " inner") if "inner_precision" in W["params"] else "f64",
        "data": "synthetic (seeded generator of the configuration; no dataset)",
        "config": {"workload": args.workload, "problem": W["problem"], "grid": W["grid"], "n": n, "nnz": nnz,
                   "method": W["outer"] + ("/" + W["inner"] if W["inner"] != "NONE" else ""),
                   "params": W["params"],
                   "parallelism": f"row split x{world} (NCCL halo + all-reduce)" if split else f"replicas x{world}",
                   "l2": "inputs larger than L2 (matrix >= 175 MB)" if nnz * 12 > 126e6 else
                         "working set fits in the 126 MB L2 (no flush between steps)"},
        "result": {"status": res.status, "loop": res.loop, "true_rel_res": res.true_rel_res,
                   "inner_calls": res.inner_calls},
        "plain_fp64": plain,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        "gpu_launches": int(launches_b - launches_a),
    }
    if rank == 0:
        print(json.dumps(out))
    M.close()
    if comm is not None:
        comm.close()
    ctx.close()
    del launches0


def _ref_workdir(A, b, threads):
    """The workload's matrix in the reference's CRS text format, written by
    the pure-Python writer (no part of the product library is loaded)."""
    from solver_cpp_b200.matrices import write_crs

    wd = tempfile.mkdtemp(prefix="refbench_")
    write_crs(os.path.join(wd, "Matrix", "CRS", "bench"), A, b, workers=max(1, threads))
    return wd


def _repo_objects_loaded():
    """Shared objects of this repository mapped into this process."""
    try:
        with open("/proc/self/maps") as f:
            paths = {ln.split()[-1] for ln in f if ln.rstrip().endswith(".so") or ".so." in ln}
    except OSError:
        return []
    return sorted(p for p in paths if p.startswith(ROOT))


def cpu_baseline_reference(A, b, W, res):
    """The reference's own CPU path (oracle/_ref/Solver) on every host thread,
    on a bounded sample of the workload: `cap` iterations of the same method
    (-L cap), scaled to the GPU run's iteration count. The complete solve is
    the reference arm's measurement (`--impl reference`)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    if not pyoracle.reference_available() or not W["ref_args"]:
        return None
    threads = os.cpu_count() or 1
    wd = _ref_workdir(A, b, threads)
    vp = W["inner"] != "NONE"
    cap = 40 if vp else 400
    try:
        r = pyoracle.run_reference(None, None, W["ref_args"] + ["-L", str(cap)], threads=threads, workdir=wd,
                                   name="bench", keep_x=False)
    finally:
        import shutil

        shutil.rmtree(wd, ignore_errors=True)
    if r["time"] is None:
        return None
    # a VP run of L iterations does L + 1 inner solves (vpcg.cpp:685,743)
    units = (cap + 1) if vp else cap
    full = (res.loop + 1) if vp else res.loop
    est = r["time"] / units * max(1, full)
    return {"value": round(est, 3), "unit": "s", "cores": threads, "kind": "reference",
            "sample": f"{cap} iterations of the reference binary ({' '.join(W['ref_args'])} -L {cap} -t {threads}): "
                      f"{r['time']:.3f} s, scaled to the GPU run's {res.loop} iterations"}


def run_reference(args, world, rank):
    """The reference's own CPU path (oracle/_ref/Solver, built unmodified from
    its sources, every host thread) on the same workload. `value` is the
    printed `time =` (its solve() span, cg.cpp:150,241) of ONE complete solve
    to the workload's stopping test. The --warmup/--steps runs are bounded
    samples (`cap` iterations each, -L cap) that fill ms_per_step. Nothing of
    the product library is loaded in this process."""
    if world > 1 and rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    W = WORKLOADS[args.workload]
    if not pyoracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/Solver was not built (reference "
                          "sources absent when the package was built)"}))
        return
    if not W["ref_args"]:
        print(json.dumps({"impl": "reference", "unavailable": f"the reference has no run of {args.workload} "
                          "(its k-skip CG recurrence does not converge)"}))
        return
    from solver_cpp_b200.matrices import config_problem

    A, b, _ = config_problem(W["problem"], W["grid"])
    threads = os.cpu_count() or 1
    wd = _ref_workdir(A, b, threads)
    try:
        full = pyoracle.run_reference(None, None, W["ref_args"], threads=threads, workdir=wd, name="bench",
                                      keep_x=False, timeout=3000)
        if full["time"] is None:
            print(json.dumps({"impl": "reference", "unavailable": "the reference binary did not report a time: "
                              + (full["stderr"] or "")[-200:].replace("\n", " ")}))
            return
        vp = W["inner"] != "NONE"
        cap = 3 if vp else 40
        times = []
        for i in range(args.warmup + args.steps):
            r = pyoracle.run_reference(None, None, W["ref_args"] + ["-L", str(cap)], threads=threads, workdir=wd,
                                       name="bench", keep_x=False)
            if i >= args.warmup and r["time"] is not None:
                times.append(r["time"])
    finally:
        import shutil

        shutil.rmtree(wd, ignore_errors=True)
    value = full["time"]
    sample = (f"one complete solve ({' '.join(W['ref_args'])} -t {threads}): {full['loop']} iterations, "
              f"printed time = {value:.3f} s; each of the {args.steps} steps: {cap} iterations (-L {cap})")
    out = {"impl": "reference", "metric": "time-to-solution at FP64 rel-res 1e-10 (mixed vs plain FP64 GPU); "
           "SpMV HBM GB/s", "value": round(value, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(statistics.median(times) * 1e3, 2) if times else None,
           "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded generator of the configuration; no dataset)",
           "config": {"workload": args.workload, "problem": W["problem"], "grid": W["grid"], "n": A.n,
                      "nnz": A.nnz, "reference_flags": W["ref_args"]},
           "result": {"loop": full["loop"], "converged": full["converged"],
                      "true_res_log10": full["true_res_log10"]},
           "cpu_baseline": {"value": round(value, 4), "unit": "s", "cores": threads, "kind": "reference",
                            "sample": sample},
           "e2e": {"value": round(value, 4), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "repo_objects_loaded": _repo_objects_loaded()}
    print(json.dumps(out))


def l2_flush(buf, clean=True):
    """Evicts the L2: writes `buf` (larger than the 126 MB L2) and, with
    `clean`, reads it back, so that the L2 then holds clean lines of `buf`
    only. Without the read ~126 MB of dirty lines stay behind, and the next
    kernel pays for writing them back to DRAM (about 19 us at HBM speed)."""
    import torch

    buf.fill_(1)
    if clean:
        torch.sum(buf.view(torch.int64))


def spmv_only(args):
    """The dominant kernel alone: y = A x with the chosen value precision on
    the workload's matrix, timed with CUDA events over `steps` launches back
    to back and over `steps` launches each after an L2 flush (`l2_flush`,
    with and without the clean-up read)."""
    import torch

    import solver_cpp_b200 as ks
    from solver_cpp_b200.matrices import config_problem

    W = WORKLOADS[args.workload]
    A, _, _ = config_problem(W["problem"], W["grid"])
    ctx = ks.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    M = ctx.matrix(A, fp32=args.spmv_only == "fp32", bf16=args.spmv_only == "bf16", index32=args.index32,
                   diag=not args.csr)
    info = M.info()
    ib, nd, sym = info["index_bytes"], info["diagonals"], info.get("dia_symmetric", 0)
    dt = ks.FP64 if args.spmv_only == "fp64" else ks.FP32
    vcode = {"fp64": ks.FP64, "fp32": ks.FP32, "bf16": ks.BF16}[args.spmv_only]
    X = ctx.vector(np.random.default_rng(0).standard_normal(A.n), dtype=dt)
    Y = ctx.vector(n=A.n, dtype=dt)
    for _ in range(args.warmup):
        ks.spmv(M, X, Y, values=vcode)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            ks.spmv(M, X, Y, values=vcode)
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    # cold: each launch after a write of a buffer larger than the 126 MB L2
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda:0")

    def cold_ms(clean):
        tot = 0.0
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                l2_flush(flush, clean)
                e0.record(stream)
                ks.spmv(M, X, Y, values=vcode)
                e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / args.steps

    ms_cold, ms_dirty = cold_ms(True), cold_ms(False)
    alg = spmv_bytes(A.n, A.nnz, args.spmv_only, ib, nd, sym)
    peak, kind = load_peaks()
    gbs = alg / (ms / 1e3) / 1e9
    gbs_cold = alg / (ms_cold / 1e3) / 1e9
    print(json.dumps({"kernel": f"spmv_{args.spmv_only}", "workload": args.workload, "n": A.n, "nnz": A.nnz,
                      "layout": layout_key(info), "index_bytes": ib, "diagonals": nd, "alg_bytes": alg,
                      "ms": round(ms, 5), "gbs": round(gbs, 1), "peak": peak,
                      "frac": round(gbs / peak, 4), "ms_cold": round(ms_cold, 5), "gbs_cold": round(gbs_cold, 1),
                      "frac_cold": round(gbs_cold / peak, 4), "ms_cold_dirty": round(ms_dirty, 5),
                      "frac_cold_dirty": round(alg / (ms_dirty / 1e3) / 1e9 / peak, 4), "peak_kind": kind,
                      "timed": "back to back (ms, frac; the matrix stays partly in L2), each launch after "
                               "an L2 flush that leaves clean lines (ms_cold, frac_cold) and after a "
                               "write-only flush whose dirty lines the launch writes back (ms_cold_dirty)"}))
    M.close()
    ctx.close()


# A few iterations of every method on the 128^3 systems: one launch of each
# hot kernel class for a profiler to capture by name (ncu -k regex:...).
# (workload, method, inner, params)
KERNEL_TOUR = [
    ("c2_cg", "CG", "NONE", dict(E=1e-10, L=4)),                      # k_cg_onchip FP64 (the whole solve)
    ("c2_cg", "CG", "NONE", dict(E=1e-10, L=4, cluster_solve=1)),     # the engine: spmv_dia FP64, RUpdOp, XpbyToOp
    ("c2_cr", "CR", "NONE", dict(E=1e-10, L=4)),
    ("c3_bicg", "BICG", "NONE", dict(E=1e-10, L=4)),                  # A p and A^T p* in one pass
    ("c3_gmres30", "GMRES", "NONE", dict(E=1e-10, L=30, R=30)),       # block dot, basis kernel, Givens
    ("c3_gcr30", "GCR", "NONE", dict(E=1e-10, L=30, R=30)),           # block dot, GcrPQOp
    ("c3_kskipbicg2", "KSKIPBICG", "NONE", dict(E=1e-10, L=6, K=2)),  # two-vector matrix powers, Gram
]


def kernel_tour(args):
    """Runs KERNEL_TOUR once (no timing; a profiler's workload)."""
    import solver_cpp_b200 as ks
    from solver_cpp_b200.matrices import config_problem

    ctx = ks.Context(0)
    cache = {}
    for wl, outer, inner, params in KERNEL_TOUR:
        W = WORKLOADS[wl]
        key = (W["problem"], W["grid"])
        if key not in cache:
            for m in cache.values():
                m[0].close()
            cache.clear()
            A, b, _ = config_problem(*key)
            cache[key] = (ctx.matrix(A, transpose=True), b)
        M, b = cache[key]
        r = ks.solve(ctx, M, outer, b, inner=inner, **params)
        print(json.dumps({"tour": wl, "method": outer, "loop": r.loop, "status": r.status}), flush=True)
    for m in cache.values():
        m[0].close()
    ctx.close()


def profile_solve(args):
    """One solve of a workload's method (or, with --profile-plain, of its plain
    FP64 counterpart) stopped after --profile-loops outer iterations; no
    timing: the workload of the ncu launch lists and kernel captures whose
    summaries are kept under profiles/."""
    import solver_cpp_b200 as ks
    from solver_cpp_b200.matrices import config_problem

    W = WORKLOADS[args.profile_solve]
    A, b, _ = config_problem(W["problem"], W["grid"])
    ctx = ks.Context(0)
    vals = W["spmv_values"]
    M = ctx.matrix(A, transpose=W["transpose"], fp32=vals == "fp32", bf16=vals == "bf16")
    if args.profile_plain and W["plain"]:
        outer, inner, params = W["plain"]["outer"], "NONE", dict(W["plain"]["params"])
    else:
        outer, inner, params = W["outer"], W["inner"], dict(W["params"])
    params["L"] = args.profile_loops
    r = ks.solve(ctx, M, outer, b, inner=inner, **params)
    print(json.dumps({"profile_solve": args.profile_solve, "method": outer, "inner": inner, "loop": r.loop,
                      "status": r.status, "inner_calls": r.inner_calls}), flush=True)
    M.close()
    ctx.close()


def ortho_only(args):
    """The GMRES orthogonalisation kernels alone on vectors of the workload's
    length: h = V^T w over k basis vectors (block dot) and w -= V h (block
    AXPY), through ks_block_dot / ks_block_axpy, timed with CUDA events.
    Bytes: the block dot reads k + 1 vectors, the block AXPY reads k + 1 and
    writes 1. Timed twice: with h in device memory (the kernels back to
    back, as the solvers run them: `block_dot`, `block_axpy`) and with h a
    host array (each call also moves the k coefficients between host and
    device and waits for them: `*_host_h`)."""
    import torch

    import solver_cpp_b200 as ks
    from solver_cpp_b200.matrices import config_problem

    W = WORKLOADS[args.workload]
    A, _, _ = config_problem(W["problem"], W["grid"])
    n = A.n
    ctx = ks.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    peak, kind = load_peaks()
    kmax = max(args.ortho_only)
    V = ctx.vector(n=n * kmax)
    V.fill(1.0 / math.sqrt(n))
    w = ctx.vector(np.random.default_rng(0).standard_normal(n))
    for k in args.ortho_only:
        h = ks.block_dot(V, n, k, w)
        for _ in range(args.warmup):
            ks.block_dot(V, n, k, w)
            ks.block_axpy(V, n, k, h * 0.0, w)
        torch.cuda.synchronize()
        out = {"kernel": "gmres_orthogonalisation", "workload": args.workload, "n": n, "k": k, "peak": peak,
               "peak_kind": kind}
        hz = h * 0.0
        hd = torch.zeros(k, dtype=torch.float64, device="cuda:0")
        hp = hd.data_ptr()
        torch.cuda.synchronize()
        for name, fn, nbytes in (("block_dot", lambda: ks.block_dot(V, n, k, w, out_device_ptr=hp), (k + 1) * 8 * n),
                                 ("block_axpy", lambda: ks.block_axpy(V, n, k, hp, w), (k + 2) * 8 * n),
                                 ("block_dot_host_h", lambda: ks.block_dot(V, n, k, w), (k + 1) * 8 * n),
                                 ("block_axpy_host_h", lambda: ks.block_axpy(V, n, k, hz, w), (k + 2) * 8 * n)):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            gbs = nbytes / (ms / 1e3) / 1e9
            out[name] = {"ms": round(ms, 4), "bytes": nbytes, "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
        print(json.dumps(out), flush=True)
    V.close()
    w.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c4_mixed")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--spmv-only", choices=["fp64", "fp32", "bf16"], default=None,
                    help="time only the SpMV kernel on the workload's matrix (profiling)")
    ap.add_argument("--index32", action="store_true", help="with --spmv-only: int32 column indices")
    ap.add_argument("--csr", action="store_true", help="with --spmv-only: CSR only (no diagonal copy)")
    ap.add_argument("--replicas", action="store_true",
                    help="with --gpus N > 1: one independent replica per rank (weak scaling) instead of the "
                         "default row split of the one system over the ranks (strong scaling)")
    ap.add_argument("--ortho-only", type=int, nargs="+", default=None, metavar="K",
                    help="time only the GMRES block dot / block AXPY over K basis vectors (profiling)")
    ap.add_argument("--profile-solve", choices=sorted(WORKLOADS), default=None,
                    help="one untimed solve of the workload (a profiler's workload)")
    ap.add_argument("--profile-loops", type=int, default=3, help="with --profile-solve: outer iterations")
    ap.add_argument("--profile-plain", action="store_true", help="with --profile-solve: the plain FP64 method")
    ap.add_argument("--kernel-tour", action="store_true",
                    help="run a few iterations of every method on the 128^3 systems (profiler workload)")
    args = ap.parse_args()
    if args.kernel_tour:
        kernel_tour(args)
        return
    if args.profile_solve:
        profile_solve(args)
        return
    if args.spmv_only:
        spmv_only(args)
        return
    if args.ortho_only:
        ortho_only(args)
        return
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup()
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
