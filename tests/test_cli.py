"""The `Solver` command-line drop-in (solver_cpp_b200/bin/Solver).

CPU: option handling and the reference's input checks (collection::readCMD /
checkCRSMatrix). GPU: the reference's own command lines produce the same
./output/<NAME>_his.txt as the reference's run (within the parity envelope,
golden_cases.check_history), the same "loop =" line and verdict.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from golden_cases import check_history, load
from solver_cpp_b200.matrices import config_problem, write_crs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "solver_cpp_b200", "bin", "Solver")


def run(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=600)


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "solver_cpp_b200", "csrc")], check=True)
    return CLI


def _problem_dir(tmp_path, name, prob, grid):
    A, b, _ = config_problem(prob, grid)
    write_crs(str(tmp_path / "Matrix" / "CRS" / name), A, b)
    run_dir = tmp_path / "run"
    run_dir.mkdir(exist_ok=True)
    return A, b, str(run_dir)


def test_cli_usage_and_option_errors(cli, tmp_path):
    r = run(["--help"], str(tmp_path))
    assert r.returncode == 0 and "usage: Solver" in r.stdout
    r = run(["-m", "x"], str(tmp_path))
    assert r.returncode != 0 and "OuterSolver" in r.stderr
    r = run(["-S", "cg"], str(tmp_path))
    assert r.returncode != 0 and "Must set one input source" in r.stderr
    r = run(["-S", "nosuch", "-m", "x"], str(tmp_path))
    assert r.returncode != 0 and "can not found" in r.stderr
    r = run(["-S", "cg", "-m", "x", "-M", "y"], str(tmp_path))
    assert r.returncode != 0 and "Only can set one input source" in r.stderr
    r = run(["-S", "cg", "-m", "x", "--bogus"], str(tmp_path))
    assert r.returncode != 0 and "unknown option" in r.stderr


def test_cli_checks_crs_headers(cli, tmp_path):
    A, b, rd = _problem_dir(tmp_path, "m", "poisson2d", 8)
    bx = tmp_path / "Matrix" / "CRS" / "m" / "bx.txt"
    lines = bx.read_text().splitlines()
    lines[0] = f"{A.n + 1} {A.n + 1} {A.nnz}"
    bx.write_text("\n".join(lines) + "\n")
    r = run(["-S", "cg", "-m", "m", "-p", str(tmp_path)], rd)
    assert r.returncode != 0 and "Error in CRS files" in r.stderr


def test_cli_without_gpu_fails_cleanly(cli, tmp_path, ks):
    if ks.lib().ks_device_count() > 0:
        pytest.skip("a GPU is present")
    _, _, rd = _problem_dir(tmp_path, "m", "poisson2d", 8)
    r = run(["-S", "cg", "-m", "m", "-p", str(tmp_path)], rd)
    assert r.returncode == 1 and "no CUDA device" in r.stderr


def test_cli_not_implemented_methods(cli, tmp_path):
    _, _, rd = _problem_dir(tmp_path, "m", "poisson2d", 8)
    for m in ("kskipcr", "vpbicg"):
        r = run(["-S", m, "-s", "cg", "-m", "m", "-p", str(tmp_path)], rd)
        assert r.returncode == 0 and "Not implemented" in r.stdout


CLI_CASES = ["c1_cg", "p2_cr", "cd2_bicg", "cd2_gcr", "cd2_gmres", "cd2_kskipbicg", "p3_vpcg_cg", "cd2_vpgcr_gcr",
             "p2_kskipcg"]


@pytest.mark.gpu
@pytest.mark.parametrize("cid", CLI_CASES)
def test_cli_reproduces_reference_run(cli, tmp_path, cid):
    meta, g = load(cid)
    _, _, rd = _problem_dir(tmp_path, "prob", meta["problem"], meta["grid"])
    args = list(meta["args"]) + ["-m", "prob", "-p", str(tmp_path), "--reference-defects"]
    r = run(args, rd)
    assert r.returncode == 0, r.stderr
    loop = int(re.search(r"^loop = (\d+)", r.stdout, re.M).group(1))
    assert ("not converge" not in r.stdout) == meta["converged"]
    h = np.loadtxt(os.path.join(rd, "output", f"{meta['outer']}_his.txt"), ndmin=2)
    check_history(h[:, 0].astype(np.int64), h[:, 1], g["hist_iter"], g["hist_err"], g["envelope"], loop,
                  meta["loop"], meta["loop_range"])
    x = np.loadtxt(os.path.join(rd, "output", f"{meta['outer']}_xvec.txt"), ndmin=2)
    assert x.shape[0] == meta["n"]
    tr = float(re.search(r"\|b-ax\|2/\|b\|2 = (\S+)", r.stdout).group(1))
    if meta["converged"]:
        assert tr == pytest.approx(meta["true_res_log10"], abs=0.21)


def _mm_dir(tmp_path, name, prob, grid):
    """The Matrix Market layout the reference checks: <P>/<N>/<D>/<M>/<M>.mtx."""
    import scipy.io

    A, _, _ = config_problem(prob, grid)
    d = tmp_path / "Matrix" / "MM" / name
    d.mkdir(parents=True)
    scipy.io.mmwrite(str(d / f"{name}.mtx"), A.to_scipy(), precision=17)
    run_dir = tmp_path / "run"
    run_dir.mkdir(exist_ok=True)
    return A, str(run_dir)


def test_cli_matrix_market_input_checks(cli, tmp_path, ks):
    _, rd = _mm_dir(tmp_path, "mm", "poisson2d", 8)
    r = run(["-S", "cg", "-M", "nothere", "-P", str(tmp_path)], rd)
    assert r.returncode != 0 and "Error no MM files Dir" in r.stderr
    r = run(["-S", "cg", "-M", "mm", "-m", "mm", "-P", str(tmp_path)], rd)
    assert r.returncode != 0 and "Only can set one input source" in r.stderr
    bad = tmp_path / "Matrix" / "MM" / "bad"
    bad.mkdir()
    (bad / "bad.mtx").write_text("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n")
    r = run(["-S", "cg", "-M", "bad", "-P", str(tmp_path)], rd)
    assert r.returncode != 0 and "Error in mm file" in r.stderr
    if ks.lib().ks_device_count() == 0:  # the file is read; only the device is missing
        r = run(["-S", "cg", "-M", "mm", "-P", str(tmp_path)], rd)
        assert r.returncode == 1 and "no CUDA device" in r.stderr


@pytest.mark.gpu
def test_cli_matrix_market_solve(cli, tmp_path):
    A, rd = _mm_dir(tmp_path, "mm", "poisson2d", 40)
    r = run(["-S", "cg", "-M", "mm", "-P", str(tmp_path), "-E", "1e-12"], rd)
    assert r.returncode == 0, r.stderr
    assert "converge" in r.stdout and "not converge" not in r.stdout
    x = np.loadtxt(os.path.join(rd, "output", "CG_xvec.txt"), ndmin=2)[:, 1]
    assert x.shape[0] == A.n and np.max(np.abs(x - 1.0)) < 1e-9  # b = A * 1


def _data2csv_fields(log):
    """The fields data2csv.sh's Seek() extracts from a run log, restated:
    each is `grep PATTERN | head/tail -1 | cut -d ',' -f1 | sed 's/[^0-9.]//g'`
    (and `cut -c 2-` for H2D / D2H)."""
    lines = log.splitlines()

    def grep(p):
        return [ln for ln in lines if p in ln]

    def num(ln, comma=True):
        s = ln.split(",")[0] if comma else ln
        return re.sub(r"[^0-9.]", "", s)

    f = {"CUDA": grep("CUDA :")[0].split(":")[1].strip(), "MultiGPU": grep("MultiGPU :")[0].split(":")[1].strip()}
    f["Total"] = num(grep("time")[0], comma=False)
    f["Converge"] = grep("converge")
    f["Loop"] = re.sub(r"[^0-9]", "", grep("loop")[0]) if len(grep("loop")) == 1 else None
    f["CPU-Dot"], f["CPU-MV"] = num(grep("Dot")[0]), num(grep("MV")[0])
    f["GPU-Dot"], f["GPU-MV"] = num(grep("Dot")[-1]), num(grep("MV")[-1])
    f["GPU-H2D"], f["GPU-D2H"] = num(grep("H2D time")[0])[1:], num(grep("D2H time")[0])[1:]
    f["GPU-Memset"] = num(grep("Memset")[0])
    f["Other"] = num(grep("other")[0])
    return f


@pytest.mark.gpu
def test_cli_report_parses_like_data2csv(cli, tmp_path):
    """The log carries the reference's header and times report (times.cpp:44-76)
    line for line: every field data2csv.sh reads is there and numeric, the
    GPU Dot + MV + other add up to the solve time."""
    # GMRES(30): one kernel per step (CG, CR and BiCG run this system as one
    # on-chip launch, without separate dot kernels to time)
    A, b, rd = _problem_dir(tmp_path, "p3", "poisson3d", 40)
    r = run(["-S", "gmres", "-R", "30", "-E", "1e-10", "-m", "p3", "-p", str(tmp_path)], rd)
    assert r.returncode == 0, r.stderr
    f = _data2csv_fields(r.stdout)
    assert f["CUDA"] == "On" and f["MultiGPU"] == "Off"
    assert f["Converge"] == ["converge"] and int(f["Loop"]) > 10
    total = float(f["Total"])
    vals = {k: float(f[k]) for k in ("CPU-Dot", "CPU-MV", "GPU-Dot", "GPU-MV", "GPU-H2D", "GPU-D2H", "GPU-Memset",
                                       "Other")}
    assert total > 0 and vals["GPU-MV"] > 0 and vals["GPU-Dot"] > 0 and vals["GPU-H2D"] > 0
    assert vals["GPU-MV"] + vals["GPU-Dot"] + vals["Other"] == pytest.approx(total, rel=1e-3, abs=2e-6)
