"""Synthetic CSR test matrices and the reference's CRS text format.

The reference reads a square sparse matrix from three text files under
``<CRS_Path>/<L1_Dir_Name>/<CRS_Dir_Name>/<CRS_Matrix_Name>/``
(solver_collection.cpp:400-470, defaults ``../Matrix/CRS/<name>``):

* ``ColVal.txt``: header ``N M NNZ`` then one ``col val`` line per nonzero,
  0-based, rows in order (read with ``fscanf("%d %le")``,
  solver_collection.cpp:758-767);
* ``Ptr.txt``: header then ``N+1`` row offsets (solver_collection.cpp:786-794);
* ``bx.txt``: header then ``N`` lines ``b x`` (solver_collection.cpp:811-821).

The generators build the matrices named by the benchmark configurations:
5-/7-point Poisson, 7-point first-order upwind convection-diffusion, and
cell-wise log-normal variable-coefficient diffusion with harmonic-mean faces.
Rows use the natural ordering ``i = ix + nx*(iy + ny*iz)``; columns ascend
within each row. All randomness is seeded ``numpy.random.default_rng``.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

__all__ = [
    "CSR",
    "poisson2d",
    "poisson3d",
    "convdiff2d",
    "convdiff3d",
    "varcoef2d",
    "varcoef3d",
    "config_problem",
    "write_crs",
    "read_crs",
    "transpose",
]


@dataclasses.dataclass
class CSR:
    """Square CSR matrix: int32 ``ptr`` (n+1), int32 ``col`` and float64 ``val``."""

    ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray

    @property
    def n(self) -> int:
        return int(self.ptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x with row sums in index order (numpy, for host-side checks)."""
        rows = np.repeat(np.arange(self.n), np.diff(self.ptr))
        return np.bincount(rows, weights=self.val * x[self.col], minlength=self.n)

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.val, self.col, self.ptr), shape=(self.n, self.n))


def _assemble(offsets, coefs, masks, n) -> CSR:
    """Stencil assembly. ``offsets`` ascend, so row-major flattening of the
    (n, k) tables gives rows in order with ascending columns."""
    k = len(offsets)
    cols = np.empty((n, k), dtype=np.int64)
    vals = np.empty((n, k), dtype=np.float64)
    keep = np.empty((n, k), dtype=bool)
    base = np.arange(n, dtype=np.int64)
    for j, (off, c, m) in enumerate(zip(offsets, coefs, masks)):
        cols[:, j] = base + off
        vals[:, j] = c
        keep[:, j] = m
    counts = keep.sum(axis=1)
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    if ptr[-1] >= 2**31:
        raise ValueError("nnz exceeds the int32 index range of the CSR format")
    col = cols[keep].astype(np.int32)
    val = vals[keep]
    return CSR(ptr.astype(np.int32), col, val)


def _grid2(nx, ny):
    i = np.arange(nx * ny, dtype=np.int64)
    return i % nx, i // nx


def _grid3(nx, ny, nz):
    i = np.arange(nx * ny * nz, dtype=np.int64)
    return i % nx, (i // nx) % ny, i // (nx * ny)


def poisson2d(nx: int, ny: int | None = None) -> CSR:
    """5-point Laplacian, Dirichlet boundaries eliminated (4 / -1)."""
    ny = nx if ny is None else ny
    n = nx * ny
    ix, iy = _grid2(nx, ny)
    one = np.ones(n)
    return _assemble(
        [-nx, -1, 0, 1, nx],
        [-one, -one, 4 * one, -one, -one],
        [iy > 0, ix > 0, np.ones(n, bool), ix < nx - 1, iy < ny - 1],
        n,
    )


def poisson3d(nx: int, ny: int | None = None, nz: int | None = None) -> CSR:
    """7-point Laplacian, Dirichlet boundaries eliminated (6 / -1)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    n = nx * ny * nz
    ix, iy, iz = _grid3(nx, ny, nz)
    one = np.ones(n)
    pl = nx * ny
    return _assemble(
        [-pl, -nx, -1, 0, 1, nx, pl],
        [-one, -one, -one, 6 * one, -one, -one, -one],
        [iz > 0, iy > 0, ix > 0, np.ones(n, bool), ix < nx - 1, iy < ny - 1, iz < nz - 1],
        n,
    )


def _upwind_coefs(v, peclet, nu=1.0):
    """First-order upwind convection-diffusion coefficients per axis.

    The mesh width h is chosen so the cell Peclet number of the largest
    velocity component is ``peclet``: Pe = |v|max h / (2 nu). Row scaling is
    the plain finite-difference one: diffusion nu/h^2 (2d / -1 per axis),
    convection |v_d|/h on the upwind side.
    """
    vmax = max(abs(c) for c in v)
    h = 2.0 * nu * peclet / vmax
    d = nu / (h * h)
    lower, upper = [], []
    diag = 0.0
    for c in v:
        a = abs(c) / h
        diag += 2 * d + a
        if c >= 0:
            lower.append(-d - a)
            upper.append(-d)
        else:
            lower.append(-d)
            upper.append(-d - a)
    return diag, lower, upper


def convdiff3d(nx: int, v=(1.0, 0.5, 0.25), peclet: float = 0.5) -> CSR:
    """Nonsymmetric 7-point first-order upwind convection-diffusion."""
    n = nx**3
    ix, iy, iz = _grid3(nx, nx, nx)
    diag, lo, up = _upwind_coefs(v, peclet)
    one = np.ones(n)
    pl = nx * nx
    return _assemble(
        [-pl, -nx, -1, 0, 1, nx, pl],
        [lo[2] * one, lo[1] * one, lo[0] * one, diag * one, up[0] * one, up[1] * one, up[2] * one],
        [iz > 0, iy > 0, ix > 0, np.ones(n, bool), ix < nx - 1, iy < nx - 1, iz < nx - 1],
        n,
    )


def convdiff2d(nx: int, v=(1.0, 0.5), peclet: float = 0.5) -> CSR:
    """Nonsymmetric 5-point first-order upwind convection-diffusion."""
    n = nx * nx
    ix, iy = _grid2(nx, nx)
    diag, lo, up = _upwind_coefs(v, peclet)
    one = np.ones(n)
    return _assemble(
        [-nx, -1, 0, 1, nx],
        [lo[1] * one, lo[0] * one, diag * one, up[0] * one, up[1] * one],
        [iy > 0, ix > 0, np.ones(n, bool), ix < nx - 1, iy < nx - 1],
        n,
    )


def _harm(a, b):
    return 2.0 * a * b / (a + b)


def varcoef3d(nx: int, sigma: float = 1.5, seed: int = 3) -> CSR:
    """SPD 7-point diffusion with ln(kappa) ~ N(0, sigma^2) i.i.d. per cell.

    Interior face coefficients are harmonic means of the two cells; a boundary
    face (Dirichlet 0) takes the cell's own kappa. Row i: diagonal = sum of its
    six face coefficients, off-diagonals = -face coefficient.
    """
    n = nx**3
    rng = np.random.default_rng(seed)
    kap = np.exp(sigma * rng.standard_normal(n))
    ix, iy, iz = _grid3(nx, nx, nx)
    pl = nx * nx
    idx = np.arange(n, dtype=np.int64)
    faces = []
    masks = []
    for off, inside in (
        (-pl, iz > 0), (-nx, iy > 0), (-1, ix > 0),
        (1, ix < nx - 1), (nx, iy < nx - 1), (pl, iz < nx - 1),
    ):
        nb = np.clip(idx + off, 0, n - 1)
        f = np.where(inside, _harm(kap, kap[nb]), kap)
        faces.append(f)
        masks.append(inside)
    diag = np.sum(faces, axis=0)
    coefs = [-faces[0], -faces[1], -faces[2], diag, -faces[3], -faces[4], -faces[5]]
    msk = [masks[0], masks[1], masks[2], np.ones(n, bool), masks[3], masks[4], masks[5]]
    return _assemble([-pl, -nx, -1, 0, 1, nx, pl], coefs, msk, n)


def varcoef2d(nx: int, sigma: float = 1.0, seed: int = 5) -> CSR:
    """SPD 5-point diffusion, log-normal cell coefficients (see varcoef3d)."""
    n = nx * nx
    rng = np.random.default_rng(seed)
    kap = np.exp(sigma * rng.standard_normal(n))
    ix, iy = _grid2(nx, nx)
    idx = np.arange(n, dtype=np.int64)
    faces, masks = [], []
    for off, inside in ((-nx, iy > 0), (-1, ix > 0), (1, ix < nx - 1), (nx, iy < nx - 1)):
        nb = np.clip(idx + off, 0, n - 1)
        faces.append(np.where(inside, _harm(kap, kap[nb]), kap))
        masks.append(inside)
    diag = np.sum(faces, axis=0)
    coefs = [-faces[0], -faces[1], diag, -faces[2], -faces[3]]
    msk = [masks[0], masks[1], np.ones(n, bool), masks[2], masks[3]]
    return _assemble([-nx, -1, 0, 1, nx], coefs, msk, n)


def transpose(A: CSR) -> CSR:
    """CSR of A^T (rows of A^T ascend inside each row), by stable sort."""
    order = np.argsort(A.col, kind="stable")
    rows = np.repeat(np.arange(A.n, dtype=np.int32), np.diff(A.ptr))
    counts = np.bincount(A.col, minlength=A.n)
    ptr = np.zeros(A.n + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    return CSR(ptr.astype(np.int32), rows[order].astype(np.int32), A.val[order].copy())


def config_problem(name: str, size: int | None = None):
    """Matrix and right-hand side of a named benchmark configuration.

    ``size`` overrides the grid edge (for small parity cases). Returns
    ``(A, b, meta)``.

    * ``poisson2d``  (64^2): b = A*1 + U(-1e-3, 1e-3), seed 0
    * ``poisson3d``  (128^3): b ~ U(0, 1), seed 1
    * ``convdiff3d`` (128^3): v = (1, 0.5, 0.25), cell Peclet 0.5; b ~ U(0,1), seed 2
    * ``varcoef3d``  (160^3): ln kappa ~ N(0, 1.5^2) seed 3; b ~ N(0,1), seed 4
    * ``varcoef2d``  (512^2): ln kappa ~ N(0, 1) seed 5; b ~ U(0,1), seed 8
    * ``convdiff2d`` (512^2): v = (1, 0.5), Peclet 0.5; b ~ U(0,1), seed 9
    """
    if name == "poisson2d":
        nx = size or 64
        A = poisson2d(nx)
        rng = np.random.default_rng(0)
        b = A.matvec(np.ones(A.n)) + rng.uniform(-1e-3, 1e-3, A.n)
    elif name == "poisson3d":
        nx = size or 128
        A = poisson3d(nx)
        b = np.random.default_rng(1).uniform(0.0, 1.0, A.n)
    elif name == "convdiff3d":
        nx = size or 128
        A = convdiff3d(nx)
        b = np.random.default_rng(2).uniform(0.0, 1.0, A.n)
    elif name == "varcoef3d":
        nx = size or 160
        A = varcoef3d(nx)
        b = np.random.default_rng(4).standard_normal(A.n)
    elif name == "varcoef2d":
        nx = size or 512
        A = varcoef2d(nx)
        b = np.random.default_rng(8).uniform(0.0, 1.0, A.n)
    elif name == "convdiff2d":
        nx = size or 512
        A = convdiff2d(nx)
        b = np.random.default_rng(9).uniform(0.0, 1.0, A.n)
    else:
        raise ValueError(f"unknown configuration {name!r}")
    return A, np.ascontiguousarray(b, dtype=np.float64), {"name": name, "grid": nx}


_LINES_PER_CHUNK = 1 << 20


def _format_chunk(fmt, cols):
    """Text of the rows of one chunk (module level: runs in worker processes)."""
    block = np.column_stack(cols) if len(cols) > 1 else cols[0][:, None]
    return "".join(fmt % tuple(row) for row in block.tolist())


def _write_lines(path, header, columns, fmts, pool=None):
    """Write a header and whitespace-separated columns in bounded chunks;
    with a process pool the chunks are formatted in parallel and written in
    order."""
    fmt = " ".join(fmts) + "\n"
    n = columns[0].shape[0]
    spans = [(s, min(n, s + _LINES_PER_CHUNK)) for s in range(0, n, _LINES_PER_CHUNK)]
    with open(path, "w") as f:
        f.write(header)
        if pool is None:
            for s, e in spans:
                f.write(_format_chunk(fmt, [c[s:e] for c in columns]))
        else:
            futs = [pool.submit(_format_chunk, fmt, [c[s:e] for c in columns]) for s, e in spans]
            for fu in futs:
                f.write(fu.result())


def write_crs(directory: str, A: CSR, b: np.ndarray, x: np.ndarray | None = None, workers: int = 1) -> None:
    """Write ``ColVal.txt``, ``Ptr.txt`` and ``bx.txt`` in the reference format.

    Values are written with 17 significant digits so ``fscanf("%le")`` reads
    back the identical doubles. ``workers`` > 1 formats the text in that many
    processes (started with ``spawn``).
    """
    os.makedirs(directory, exist_ok=True)
    n, nnz = A.n, A.nnz
    header = f"{n} {n} {nnz}\n"
    x = np.zeros(n) if x is None else x
    pool = None
    if workers > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor

        pool = ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"))
    try:
        _write_lines(os.path.join(directory, "ColVal.txt"), header, [A.col, A.val], ["%d", "%.17e"], pool)
        _write_lines(os.path.join(directory, "Ptr.txt"), header, [A.ptr], ["%d"], pool)
        _write_lines(os.path.join(directory, "bx.txt"), header, [b, x], ["%.17e", "%.17e"], pool)
    finally:
        if pool is not None:
            pool.shutdown()


def read_crs(directory: str):
    """Read the three CRS files; returns ``(A, b, x)``. Checks the headers the
    way collection::checkCRSMatrix does (solver_collection.cpp:655-724)."""
    heads = []
    for name in ("ColVal.txt", "Ptr.txt", "bx.txt"):
        with open(os.path.join(directory, name)) as f:
            heads.append(tuple(int(t) for t in f.readline().split()[:3]))
    if len({h[0] for h in heads}) != 1 or len({h[1] for h in heads}) != 1 or len({h[2] for h in heads}) != 1:
        raise ValueError("CRS headers disagree on N, M or NNZ")
    n, m, nnz = heads[0]
    if n != m:
        raise ValueError("N != M")
    cv = np.loadtxt(os.path.join(directory, "ColVal.txt"), skiprows=1, ndmin=2)
    ptr = np.loadtxt(os.path.join(directory, "Ptr.txt"), skiprows=1, dtype=np.int64)
    bx = np.loadtxt(os.path.join(directory, "bx.txt"), skiprows=1, ndmin=2)
    A = CSR(ptr.astype(np.int32), cv[:nnz, 0].astype(np.int32), cv[:nnz, 1].copy())
    return A, bx[:n, 0].copy(), bx[:n, 1].copy()
