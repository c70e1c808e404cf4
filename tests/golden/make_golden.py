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

Usage: python tests/golden/make_golden.py   (needs `make -C oracle ref`)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

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


if __name__ == "__main__":
    main()
