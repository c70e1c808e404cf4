"""Generate the golden fixtures from the reference's own CPU path.

Runs ``oracle/_ref/Solver`` (the reference sources compiled unmodified with a
host-only stand-in for its device class; see oracle/Makefile) with one OpenMP
thread on small instances of the benchmark problems, and stores for every run
the residual history exactly as the reference printed it
(``./output/<NAME>_his.txt``), the printed ``loop =`` and
``|b-ax|2/|b|2 =`` lines, the verdict, and the solution vector
(``./output/<NAME>_xvec.txt``, 13 significant digits).

The inputs are regenerated by solver_cpp_b200.matrices.config_problem; a
SHA-256 of the matrix values and of b is stored so the tests can detect a
generator change.

Usage: python tests/golden/make_golden.py           (needs `make -C oracle ref`)
       python tests/golden/make_golden.py --large   the full-size configurations

``--large`` runs the benchmark configurations at their full sizes (128^3
Poisson and convection-diffusion, the 160^3 log-normal system). Their
fixtures keep the history, its envelope, the loop counts of every thread
count, the verdict and the printed true residual, but no solution vector and
no matrix (the seeded generators rebuild it; the SHA-256 digests pin it).
The runs take tens of minutes of host time; they are scheduled over the host
cores, each run holding as many cores as it has OpenMP threads.

``--orders`` (after ``--large``) runs the oracle, the C restatement pinned
bit for bit to the reference, on the full-size cases whose reference loop
counts differ between thread counts, with its dot products summed in
further orders (ORDER_CHUNKS), and records the loop counts.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from solver_cpp_b200.matrices import config_problem  # noqa: E402

# (case id, problem, grid, reference flags)
CASES = [
    ("c1_cg", "poisson2d", 64, ["-S", "cg", "-E", "1e-10", "-L", "10000"]),
    ("p2_cr", "poisson2d", 64, ["-S", "cr", "-E", "1e-10"]),
    ("p3_cg", "poisson3d", 16, ["-S", "cg", "-E", "1e-10"]),
    ("p3_cr", "poisson3d", 16, ["-S", "cr", "-E", "1e-10"]),
    ("p2_kskipcg", "poisson2d", 32, ["-S", "kskipcg", "-K", "2", "-L", "60"]),
    ("cd2_bicg", "convdiff2d", 32, ["-S", "bicg", "-E", "1e-10"]),
    ("cd2_gcr", "convdiff2d", 32, ["-S", "gcr", "-R", "30", "-E", "1e-10"]),
    ("cd2_gmres", "convdiff2d", 32, ["-S", "gmres", "-R", "30", "-E", "1e-10"]),
    ("cd2_kskipbicg", "convdiff2d", 32, ["-S", "kskipbicg", "-K", "2", "-E", "1e-10"]),
    ("cd3_bicg", "convdiff3d", 12, ["-S", "bicg", "-E", "1e-10"]),
    ("cd3_kskipbicg", "convdiff3d", 12, ["-S", "kskipbicg", "-K", "2", "-E", "1e-10"]),
    ("cd3_gcr", "convdiff3d", 12, ["-S", "gcr", "-R", "30", "-E", "1e-10"]),
    ("cd3_gmres", "convdiff3d", 12, ["-S", "gmres", "-R", "30", "-E", "1e-10"]),
    ("vc3_cg", "varcoef3d", 12, ["-S", "cg", "-E", "1e-10"]),
    ("vc3_vpcg_cg", "varcoef3d", 12, ["-S", "vpcg", "-s", "cg", "-l", "20", "-e", "1e-30", "-E", "1e-10"]),
    ("vc3_gmres", "varcoef3d", 12, ["-S", "gmres", "-R", "30", "-E", "1e-10"]),
    ("p3_vpcg_cg", "poisson3d", 16, ["-S", "vpcg", "-s", "cg", "-l", "20", "-e", "1e-1", "-E", "1e-10"]),
    ("p2_vpcg_cr", "poisson2d", 32, ["-S", "vpcg", "-s", "cr", "-l", "20", "-e", "1e-1", "-E", "1e-10"]),
    ("p2_vpcg_bicg", "poisson2d", 32, ["-S", "vpcg", "-s", "bicg", "-l", "20", "-e", "1e-1", "-E", "1e-10"]),
    ("p2_vpcg_gcr", "poisson2d", 32, ["-S", "vpcg", "-s", "gcr", "-l", "20", "-e", "1e-1", "-r", "10",
                                      "-E", "1e-10"]),
    ("p2_vpcg_gmres", "poisson2d", 32, ["-S", "vpcg", "-s", "gmres", "-l", "20", "-e", "1e-1", "-r", "10",
                                        "-E", "1e-10", "-L", "60"]),
    ("p2_vpcg_kskipbicg", "poisson2d", 32, ["-S", "vpcg", "-s", "kskipbicg", "-l", "20", "-e", "1e-1",
                                            "-E", "1e-10"]),
    ("p2_vpcg_kskipcg", "poisson2d", 32, ["-S", "vpcg", "-s", "kskipcg", "-l", "20", "-e", "1e-1",
                                          "-E", "1e-10", "-L", "40"]),
    ("p2_vpcr_cg", "poisson2d", 32, ["-S", "vpcr", "-s", "cg", "-l", "20", "-e", "1e-1", "-E", "1e-10",
                                     "-L", "50"]),
    ("cd2_vpgcr_gcr", "convdiff2d", 32, ["-S", "vpgcr", "-s", "gcr", "-R", "30", "-l", "10", "-e", "1e-1",
                                         "-r", "30", "-E", "1e-10"]),
    ("cd2_vpgmres_cg", "convdiff2d", 32, ["-S", "vpgmres", "-s", "cg", "-R", "30", "-l", "10", "-e", "1e-1",
                                          "-E", "1e-10", "-L", "100"]),
    ("cd2_vpgmres_gmres", "convdiff2d", 32, ["-S", "vpgmres", "-s", "gmres", "-R", "30", "-l", "10",
                                             "-e", "1e-1", "-r", "11", "-E", "1e-10", "-L", "100"]),
    ("p2_gcr_short", "poisson2d", 16, ["-S", "gcr", "-R", "4", "-L", "9", "-E", "1e-12"]),
    ("p2_gmres_short", "poisson2d", 16, ["-S", "gmres", "-R", "4", "-L", "9", "-E", "1e-12"]),
]


# Full-size configurations: (case id, problem, grid, reference flags).
LARGE_CASES = [
    ("L_c2_cg", "poisson3d", 128, ["-S", "cg", "-E", "1e-10"]),
    ("L_c2_cr", "poisson3d", 128, ["-S", "cr", "-E", "1e-10"]),
    ("L_c3_bicg", "convdiff3d", 128, ["-S", "bicg", "-E", "1e-10"]),
    ("L_c3_kskipbicg", "convdiff3d", 128, ["-S", "kskipbicg", "-K", "2", "-E", "1e-10"]),
    ("L_c3_gcr", "convdiff3d", 128, ["-S", "gcr", "-R", "30", "-E", "1e-10"]),
    ("L_c3_gmres", "convdiff3d", 128, ["-S", "gmres", "-R", "30", "-E", "1e-10"]),
    ("L_c4_cg", "varcoef3d", 160, ["-S", "cg", "-E", "1e-10"]),
]

THREADS = (2, 3, 4, 8)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def flags_to_params(args):
    """Reference flags -> (outer, inner, params dict of flag letters)."""
    outer, inner, kw = None, "NONE", {}
    it = iter(range(len(args)))
    i = 0
    while i < len(args):
        f, v = args[i], args[i + 1]
        i += 2
        if f == "-S":
            outer = v.upper()
        elif f == "-s":
            inner = v.upper()
        else:
            letter = f[1:]
            kw[letter] = float(v) if letter in ("E", "e") else int(v)
    del it
    return outer, inner, kw


def main():
    if not pyoracle.reference_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    index = {}
    for cid, prob, grid, args in CASES:
        A, b, _ = config_problem(prob, grid)
        res = pyoracle.run_reference(A, b, args, threads=1)
        if res["returncode"] != 0:
            raise SystemExit(f"{cid}: reference failed\n{res['stderr']}")
        outer, inner, kw = flags_to_params(args)
        # The reference's own sensitivity to summation order: rerun it with
        # more OpenMP threads (its dot products and norms then add partial
        # sums) and record, per history entry, the largest relative departure
        # from the -t 1 run, plus the spread of iteration counts.
        h1 = res["hist_err"]
        env = np.zeros_like(h1)
        loops = [res["loop"]]
        verdicts = [bool(res["converged"])]
        for t in THREADS:
            rt = pyoracle.run_reference(A, b, args, threads=t, keep_x=False)
            loops.append(rt["loop"])
            verdicts.append(bool(rt["converged"]))
            m = min(len(h1), len(rt["hist_err"]))
            dev = np.abs(rt["hist_err"][:m] - h1[:m]) / np.maximum(np.abs(h1[:m]), 1e-300)
            env[:m] = np.maximum(env[:m], dev)
            if m < len(h1):  # a shorter run departs completely beyond its end
                env[m:] = np.inf
        np.savez_compressed(
            os.path.join(HERE, f"{cid}.npz"),
            hist_iter=res["hist_iter"], hist_err=h1, x=res.get("x", np.zeros(0)), envelope=env,
        )
        index[cid] = {
            "problem": prob, "grid": grid, "args": args, "outer": outer, "inner": inner, "params": kw,
            "loop": res["loop"], "converged": bool(res["converged"]),
            "true_res_log10": res["true_res_log10"], "n": A.n, "nnz": A.nnz,
            "sha_val": digest(A.val), "sha_b": digest(b),
            "threads_checked": [1] + list(THREADS), "loop_range": [min(loops), max(loops)],
            "verdicts_agree": len(set(verdicts)) == 1,
        }
        print(f"{cid:22s} loop={res['loop']:6d} conv={res['converged']!s:5s} "
              f"true={res['true_res_log10']} hist={len(res['hist_err'])}")
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


def main_large(workroot, cores, only=None):
    """Full-size goldens; see the module docstring."""
    import threading
    from concurrent.futures import ThreadPoolExecutor

    if not pyoracle.reference_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    cases = [c for c in LARGE_CASES if not only or c[0] in only]
    problems = {}
    for cid, prob, grid, args in cases:
        key = f"{prob}_{grid}"
        if key not in problems:
            A, b, _ = config_problem(prob, grid)
            wd = os.path.join(workroot, key)
            mdir = os.path.join(wd, "Matrix", "CRS", key)
            if not os.path.exists(os.path.join(mdir, "bx.txt")):
                from solver_cpp_b200.matrices import write_crs
                write_crs(mdir, A, b)
            problems[key] = {"wd": wd, "n": A.n, "nnz": A.nnz, "sha_val": digest(A.val), "sha_b": digest(b)}
            del A, b
            print(f"wrote {key}", flush=True)

    # Core tokens: a run with t OpenMP threads holds t of them.
    cond = threading.Condition()
    free = [cores]

    def run(cid, key, args, t):
        need = min(t, cores)
        with cond:
            cond.wait_for(lambda: free[0] >= need)
            free[0] -= need
        try:
            rd = os.path.join(problems[key]["wd"], f"run_{cid}_t{t}")
            os.makedirs(os.path.join(rd, "output"), exist_ok=True)
            r = pyoracle.run_reference(None, None, args, threads=t, workdir=problems[key]["wd"], name=key,
                                       timeout=6 * 3600, keep_x=False, run_dir=rd)
        finally:
            with cond:
                free[0] += need
                cond.notify_all()
        print(f"{cid} -t {t}: loop={r['loop']} conv={r['converged']} true={r['true_res_log10']} "
              f"time={r['time']}", flush=True)
        return r

    jobs = {}
    with ThreadPoolExecutor(max_workers=len(cases) * (1 + len(THREADS))) as ex:
        for cid, prob, grid, args in cases:
            key = f"{prob}_{grid}"
            for t in (1,) + THREADS:
                jobs[(cid, t)] = ex.submit(run, cid, key, args, t)
        results = {k: f.result() for k, f in jobs.items()}

    ipath = os.path.join(HERE, "index_large.json")
    index = json.load(open(ipath)) if os.path.exists(ipath) else {}
    for cid, prob, grid, args in cases:
        key = f"{prob}_{grid}"
        res = results[(cid, 1)]
        if res["returncode"] != 0:
            raise SystemExit(f"{cid}: reference failed\n{res['stderr']}")
        h1 = res["hist_err"]
        env = np.zeros_like(h1)
        loops = {1: res["loop"]}
        verdicts = [bool(res["converged"])]
        for t in THREADS:
            rt = results[(cid, t)]
            loops[t] = rt["loop"]
            verdicts.append(bool(rt["converged"]))
            m = min(len(h1), len(rt["hist_err"]))
            dev = np.abs(rt["hist_err"][:m] - h1[:m]) / np.maximum(np.abs(h1[:m]), 1e-300)
            env[:m] = np.maximum(env[:m], dev)
            if m < len(h1):
                env[m:] = np.inf
        np.savez_compressed(os.path.join(HERE, f"{cid}.npz"), hist_iter=res["hist_iter"], hist_err=h1,
                            envelope=env)
        outer, inner, kw = flags_to_params(args)
        p = problems[key]
        index[cid] = {
            "problem": prob, "grid": grid, "args": args, "outer": outer, "inner": inner, "params": kw,
            "loop": res["loop"], "converged": bool(res["converged"]),
            "true_res_log10": res["true_res_log10"], "n": p["n"], "nnz": p["nnz"],
            "sha_val": p["sha_val"], "sha_b": p["sha_b"],
            "threads_checked": [1] + list(THREADS), "loops_by_threads": {str(k): v for k, v in loops.items()},
            "loop_range": [min(loops.values()), max(loops.values())],
            "verdicts_agree": len(set(verdicts)) == 1,
        }
        with open(ipath, "w") as f:
            json.dump(index, f, indent=1, sort_keys=True)


# Summation orders of the oracle study (--orders): the reference's sequential
# order (1: pins the oracle at full size against the -t 1 golden), contiguous
# partial sums as OpenMP would add them with more threads than the host has,
# pairwise summation (-1), the accuracy class of a parallel tree, and
# pairwise summation of every dot (-2), also of those the reference always
# adds sequentially whatever its thread count (the k-skip Gram values,
# blas.cpp:401-475), as the GPU's tree reductions do.
ORDER_CHUNKS = (1, 16, 256, 4096, -1, -2)


def _oracle_order_run(args):
    cid, prob, grid, flags, chunks = args
    from solver_cpp_b200.matrices import config_problem as cp

    A, b, _ = cp(prob, grid)
    outer, inner, kw = flags_to_params(flags)
    r = pyoracle.solve(A, b, outer, inner, sum_chunks=chunks, hist_cap=100000, **kw)
    return cid, chunks, int(r["loop"]), int(r["status"]), r["hist_err"]


def main_orders(cores, only=None, chunks=ORDER_CHUNKS):
    """Oracle loop counts under ORDER_CHUNKS for the full-size cases whose
    reference runs differ between thread counts; adds them to
    index_large.json as ``oracle_loops_by_order`` (and, for chunks = 1,
    whether the oracle reproduces the -t 1 history bit for bit)."""
    import multiprocessing as mp

    ipath = os.path.join(HERE, "index_large.json")
    index = json.load(open(ipath))
    jobs = []
    for cid, prob, grid, args in LARGE_CASES:
        if (only and cid not in only) or cid not in index:
            continue
        if len(set(index[cid]["loops_by_threads"].values())) == 1:
            continue
        jobs += [(cid, prob, grid, args, c) for c in chunks]
    with mp.get_context("spawn").Pool(max(1, min(cores, len(jobs)))) as pool:
        for cid, chunks, loop, status, hist in pool.imap_unordered(_oracle_order_run, jobs):
            e = index[cid].setdefault("oracle_loops_by_order", {})
            e[str(chunks)] = loop
            if chunks == 1:
                g = np.load(os.path.join(HERE, f"{cid}.npz"))
                h1 = g["hist_err"]
                m = min(len(h1), len(hist))
                # the reference prints 13 significant digits
                ok = len(h1) == len(hist) and bool(np.all(np.abs(hist[:m] - h1[:m]) <= 1e-12 * np.abs(h1[:m])))
                index[cid]["oracle_reproduces_t1"] = ok
            print(f"{cid} chunks={chunks}: loop={loop} status={status}", flush=True)
            with open(ipath, "w") as f:
                json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if "--orders" in sys.argv:
        import argparse

        ap = argparse.ArgumentParser()
        ap.add_argument("--orders", action="store_true")
        ap.add_argument("--cores", type=int, default=max(1, (os.cpu_count() or 2) - 1))
        ap.add_argument("--only", nargs="*")
        ap.add_argument("--chunks", type=int, nargs="*", default=list(ORDER_CHUNKS))
        a = ap.parse_args()
        main_orders(a.cores, a.only, tuple(a.chunks))
    elif "--large" in sys.argv:
        import argparse

        ap = argparse.ArgumentParser()
        ap.add_argument("--large", action="store_true")
        ap.add_argument("--workdir", default=os.path.join(tempfile.gettempdir(), "solver_golden_large"))
        ap.add_argument("--cores", type=int, default=max(1, (os.cpu_count() or 2) - 1))
        ap.add_argument("--only", nargs="*")
        a = ap.parse_args()
        main_large(a.workdir, a.cores, a.only)
    else:
        main()
