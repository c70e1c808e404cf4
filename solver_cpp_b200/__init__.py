"""B200-native (sm_100a) Krylov hot path of solver_cpp.

Python binding of the C ABI declared in ``include/krylov_sm100.h`` (the
library ``libkrylov_sm100.so`` is built in-tree by ``make -C
solver_cpp_b200/csrc``). The reference program drives its Krylov methods
through ``outerMethods::outerSelect`` (outerMethods.cpp:20-82) with the flags of
``collection::readCMD`` (solver_collection.cpp:278-307); :func:`solve` takes the
same method names and the same parameters (``L E R K F`` outer, ``l e r k f``
inner).

There is no CPU fallback: every compute call goes through the CUDA library and
raises if it is missing or no GPU is present.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import FP32, FP64, BF16, SOLVERS, LibraryMissing  # noqa: F401
from .matrices import CSR  # noqa: F401

__all__ = ["Context", "Matrix", "Vector", "KrylovError", "SolveResult", "solve", "lib", "SOLVERS"]


class KrylovError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"[ks status {status}] {message}")
        self.status = status


def lib():
    return _abi.load()


_CONVERGENCE_STATUSES = (_abi.KS_OK, _abi.KS_NOT_CONVERGED, _abi.KS_BREAKDOWN, _abi.KS_NAN_DETECTED)


def _check(status, ctx=None, what=""):
    if status == _abi.KS_OK:
        return
    L = lib()
    detail = L.ks_last_error(ctx).decode() if ctx else ""
    msg = L.ks_status_string(status).decode()
    raise KrylovError(status, f"{what}: {msg}" + (f" ({detail})" if detail else ""))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Context:
    """A device, a stream and reusable scratch (``ks_ctx``)."""

    def __init__(self, device: int = 0):
        L = lib()
        h = C.c_void_p()
        _check(L.ks_ctx_create(device, C.byref(h)), None, "ks_ctx_create")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().ks_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def synchronize(self):
        _check(lib().ks_ctx_synchronize(self.handle), self.handle, "synchronize")

    def set_stream(self, stream_ptr):
        _check(lib().ks_ctx_set_stream(self.handle, C.c_void_p(stream_ptr)), self.handle, "set_stream")

    def set_wait_limit(self, ns: int):
        """Limit of the kernels' bounded device waits in ns (<= 0: the 2 s default)."""
        _check(lib().ks_ctx_set_wait_limit(self.handle, int(ns)), self.handle, "set_wait_limit")

    def matrix(self, A: CSR, transpose=False, fp32=False, bf16=False, index32=False, diag=True) -> "Matrix":
        return Matrix(self, A, transpose=transpose, fp32=fp32, bf16=bf16, index32=index32, diag=diag)

    def vector(self, data=None, n=None, dtype=FP64) -> "Vector":
        return Vector(self, data=data, n=n, dtype=dtype)


class Matrix:
    """Device CSR matrix (``ks_mat``), optionally with its transpose and
    FP32 / BF16 value copies. ``index32`` keeps int32 column indices in the
    SpMV instead of the 16-bit row offsets used when they fit; ``diag=False``
    keeps CSR only (no diagonal copy of a stencil matrix)."""

    def __init__(self, ctx: Context, A: CSR, transpose=False, fp32=False, bf16=False, index32=False, diag=True):
        self.ctx = ctx
        self.n, self.nnz = A.n, A.nnz
        ptr = np.ascontiguousarray(A.ptr, dtype=np.int32)
        col = np.ascontiguousarray(A.col, dtype=np.int32)
        val = np.ascontiguousarray(A.val, dtype=np.float64)
        flags = (_abi.MAT_TRANSPOSE if transpose else 0) | (_abi.MAT_FP32 if fp32 else 0) | (
            _abi.MAT_BF16 if bf16 else 0) | (_abi.MAT_INDEX32 if index32 else 0) | (0 if diag else _abi.MAT_NO_DIAG)
        h = C.c_void_p()
        _check(lib().ks_csr_upload(ctx.handle, self.n, self.nnz, _ptr(ptr), _ptr(col), _ptr(val), flags,
                                   C.byref(h)), ctx.handle, "ks_csr_upload")
        self.handle = h
        self.flags = flags

    def close(self):
        # A matrix outliving its context (e.g. held by a traceback past the
        # context's close) has nothing left to free: the context released the
        # device with it, and the C call would read the freed context.
        if self.handle and self.ctx.handle:
            lib().ks_mat_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        n, nnz, rb = C.c_int64(), C.c_int64(), C.c_int64()
        _check(lib().ks_mat_info(self.handle, C.byref(n), C.byref(nnz), C.byref(rb)), self.ctx.handle, "info")
        a, t = C.c_int(), C.c_int()
        _check(lib().ks_mat_index_bytes(self.handle, C.byref(a), C.byref(t)), self.ctx.handle, "index_bytes")
        da, dt = C.c_int(), C.c_int()
        _check(lib().ks_mat_diagonals(self.handle, C.byref(da), C.byref(dt)), self.ctx.handle, "diagonals")
        sa, st = C.c_int32(), C.c_int32()
        _check(lib().ks_mat_dia_symmetric(self.handle, C.byref(sa), C.byref(st)), self.ctx.handle, "dia_symmetric")
        return {"n": n.value, "nnz": nnz.value, "row_blocks": rb.value, "index_bytes": a.value,
                "t_index_bytes": t.value, "diagonals": da.value, "t_diagonals": dt.value,
                "dia_symmetric": sa.value, "t_dia_symmetric": st.value}

    def transpose_arrays(self):
        tptr = np.zeros(self.n + 1, dtype=np.int32)
        trow = np.zeros(self.nnz, dtype=np.int32)
        tval = np.zeros(self.nnz)
        _check(lib().ks_mat_transpose_download(self.handle, _ptr(tptr), _ptr(trow), _ptr(tval)),
               self.ctx.handle, "transpose_download")
        return tptr, trow, tval


_NP = {FP64: np.float64, FP32: np.float32}


class Vector:
    """Device vector (``ks_vec``)."""

    def __init__(self, ctx: Context, data=None, n=None, dtype=FP64, wrap_ptr=None):
        self.ctx = ctx
        if data is not None:
            data = np.ascontiguousarray(data, dtype=_NP[dtype])
            n = data.shape[0]
        self.n = int(n)
        self.dtype = dtype
        h = C.c_void_p()
        if wrap_ptr is not None:
            _check(lib().ks_vec_wrap(ctx.handle, self.n, dtype, C.c_void_p(wrap_ptr), C.byref(h)), ctx.handle,
                   "ks_vec_wrap")
        else:
            _check(lib().ks_vec_create(ctx.handle, self.n, dtype, C.byref(h)), ctx.handle, "ks_vec_create")
        self.handle = h
        if data is not None:
            self.upload(data)

    def upload(self, data):
        data = np.ascontiguousarray(data, dtype=_NP[self.dtype])
        assert data.shape[0] == self.n
        _check(lib().ks_vec_upload(self.handle, _ptr(data)), self.ctx.handle, "upload")

    def numpy(self):
        out = np.empty(self.n, dtype=_NP[self.dtype])
        _check(lib().ks_vec_download(self.handle, _ptr(out)), self.ctx.handle, "download")
        return out

    def fill(self, v):
        _check(lib().ks_vec_fill(self.handle, float(v)), self.ctx.handle, "fill")

    @property
    def device_ptr(self):
        return lib().ks_vec_device_ptr(self.handle)

    def close(self):
        if self.handle and self.ctx.handle:  # as Matrix.close
            lib().ks_vec_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- primitives
def spmv(mat: Matrix, x: Vector, y: Vector, trans=False, values=None):
    L = lib()
    if values is None:
        _check(L.ks_spmv(mat.handle, int(trans), x.handle, y.handle), mat.ctx.handle, "spmv")
    else:
        _check(L.ks_spmv_values(mat.handle, int(trans), values, x.handle, y.handle), mat.ctx.handle, "spmv")


def dot(x: Vector, y: Vector) -> float:
    r = C.c_double()
    _check(lib().ks_dot(x.handle, y.handle, C.byref(r)), x.ctx.handle, "dot")
    return r.value


def nrm2(x: Vector) -> float:
    r = C.c_double()
    _check(lib().ks_nrm2(x.handle, C.byref(r)), x.ctx.handle, "nrm2")
    return r.value


def axpy(a: float, x: Vector, y: Vector):
    _check(lib().ks_axpy(float(a), x.handle, y.handle), x.ctx.handle, "axpy")


def axpy_dot(a: float, x: Vector, y: Vector, w: Vector | None = None) -> float:
    r = C.c_double()
    _check(lib().ks_axpy_dot(float(a), x.handle, y.handle, w.handle if w else None, C.byref(r)),
           x.ctx.handle, "axpy_dot")
    return r.value


def block_dot(V: Vector, ld: int, k: int, w: Vector, out_device_ptr: int = 0):
    """h = V^T w over k basis vectors. With out_device_ptr (device memory of
    the context's GPU, k doubles) the results go there in stream order and
    nothing is returned; else they come back as a numpy array."""
    if out_device_ptr:
        _check(lib().ks_block_dot(V.handle, ld, k, w.handle, C.c_void_p(out_device_ptr)), V.ctx.handle,
               "block_dot")
        return None
    h = np.zeros(max(k, 1))
    _check(lib().ks_block_dot(V.handle, ld, k, w.handle, _ptr(h)), V.ctx.handle, "block_dot")
    return h[:k]


def block_axpy(V: Vector, ld: int, k: int, h, w: Vector):
    """w -= V h. h: k coefficients as a host array, or an int device pointer
    (device memory of the context's GPU, read in stream order)."""
    if isinstance(h, int):
        _check(lib().ks_block_axpy(V.handle, ld, k, C.c_void_p(h), w.handle), V.ctx.handle, "block_axpy")
        return
    h = np.ascontiguousarray(h, dtype=np.float64)
    _check(lib().ks_block_axpy(V.handle, ld, k, _ptr(h), w.handle), V.ctx.handle, "block_axpy")


def matpow(mat: Matrix, r: Vector, p: Vector, k: int, Ar: Vector, Ap: Vector):
    _check(lib().ks_matpow(mat.handle, r.handle, p.handle, k, Ar.handle, Ap.handle), mat.ctx.handle, "matpow")


def gram_cg(Ar: Vector, Ap: Vector, r: Vector, p: Vector, k: int):
    d, e, z = np.zeros(max(2 * k, 1)), np.zeros(2 * k + 1), np.zeros(2 * k + 2)
    _check(lib().ks_gram_cg(Ar.handle, Ap.handle, r.handle, p.handle, k, _ptr(d), _ptr(e), _ptr(z)),
           r.ctx.handle, "gram_cg")
    return d[:2 * k], e, z


def gram_bicg(Ar: Vector, Ap: Vector, rs: Vector, ps: Vector, k: int):
    t, e, r_, f = np.zeros(max(2 * k, 1)), np.zeros(2 * k + 1), np.zeros(2 * k + 1), np.zeros(2 * k + 2)
    _check(lib().ks_gram_bicg(Ar.handle, Ap.handle, rs.handle, ps.handle, k, _ptr(t), _ptr(e), _ptr(r_), _ptr(f)),
           rs.ctx.handle, "gram_bicg")
    return t[:2 * k], e, r_, f


def pattern_grad(mat: Matrix, lam: Vector, x: Vector, g: Vector):
    _check(lib().ks_pattern_grad(mat.handle, lam.handle, x.handle, g.handle), mat.ctx.handle, "pattern_grad")


def check_error(mat: Matrix, b: Vector, x: Vector):
    lg, rel = C.c_double(), C.c_double()
    _check(lib().ks_check_error(mat.handle, b.handle, x.handle, C.byref(lg), C.byref(rel)), mat.ctx.handle,
           "check_error")
    return lg.value, rel.value


# ---------------------------------------------------------------- solve
_FLAG = {"L": "outer_maxloop", "E": "outer_eps", "R": "outer_restart", "K": "outer_kskip", "F": "outer_fix",
         "l": "inner_maxloop", "e": "inner_eps", "r": "inner_restart", "k": "inner_kskip", "f": "inner_fix"}


def make_params(**kw) -> _abi.Params:
    """ks_params from reference flag letters (L E R K F / l e r k f) or field
    names; ``inner_precision`` may be 'fp64' / 'fp32' / 'bf16'."""
    p = _abi.Params()
    lib().ks_params_default(C.byref(p))
    for k, v in kw.items():
        name = _FLAG.get(k, k)
        if name == "inner_precision" and isinstance(v, str):
            v = _abi.PRECISIONS[v]
        if name == "reference_defects" or name == "transpose":
            v = int(bool(v))
        setattr(p, name, v)
    return p


@dataclass
class SolveResult:
    status: int
    loop: int
    hist_iter: np.ndarray
    hist_err: np.ndarray
    x: np.ndarray | None
    true_res_log10: float
    true_rel_res: float
    solve_seconds: float
    inner_calls: int
    report: dict = field(default_factory=dict)

    @property
    def converged(self):
        return self.status == _abi.KS_OK


def _solver_code(name):
    return SOLVERS[name.upper()] if isinstance(name, str) else int(name)


def solve(ctx: Context, mat: Matrix, outer: str, b, inner: str = "NONE", x: Vector | None = None,
          hist_cap: int | None = None, **params) -> SolveResult:
    """Run one Krylov method. ``b`` is a numpy array (host path: uploaded,
    the solution downloaded) or a :class:`Vector` (device path, ``x`` then
    receives the solution on the device)."""
    L = lib()
    p = make_params(**params)
    cap = hist_cap if hist_cap is not None else int(min(p.outer_maxloop + 2, 1 << 22))
    hi = np.zeros(max(cap, 1), dtype=np.int64)
    he = np.zeros(max(cap, 1))
    rep = _abi.Report()
    oc, ic = _solver_code(outer), _solver_code(inner)
    xh = None
    if isinstance(b, Vector):
        if x is None:
            x = Vector(ctx, n=mat.n)
        st = L.ks_solve(ctx.handle, mat.handle, oc, ic, C.byref(p), b.handle, x.handle, _ptr(hi), _ptr(he), cap,
                        C.byref(rep))
    else:
        bh = np.ascontiguousarray(b, dtype=np.float64)
        xh = np.zeros(mat.n)
        st = L.ks_solve_host(ctx.handle, mat.handle, oc, ic, C.byref(p), _ptr(bh), _ptr(xh), _ptr(hi), _ptr(he),
                             cap, C.byref(rep))
    if st not in _CONVERGENCE_STATUSES:
        _check(st, ctx.handle, f"solve {outer}/{inner}")
    m = min(rep.hist_len, cap)
    report = {f: getattr(rep, f) for f, _ in _abi.Report._fields_}
    return SolveResult(status=st, loop=rep.loop, hist_iter=hi[:m].copy(), hist_err=he[:m].copy(), x=xh,
                       true_res_log10=rep.true_res_log10, true_rel_res=rep.true_rel_res,
                       solve_seconds=rep.solve_seconds, inner_calls=rep.inner_iterations, report=report)


def adjoint_grad(ctx: Context, mat: Matrix, solver: str, x: Vector, g: Vector, grad_b: Vector | None = None,
                 grad_val: Vector | None = None, inner: str = "NONE", **params):
    """grad_b = A^{-T} g and grad_val[j] = -grad_b[row(j)] * x[col(j)]."""
    p = make_params(**params)
    rep = _abi.Report()
    st = lib().ks_adjoint_grad(ctx.handle, mat.handle, _solver_code(solver), _solver_code(inner), C.byref(p),
                               x.handle, g.handle, grad_b.handle if grad_b else None,
                               grad_val.handle if grad_val else None, C.byref(rep))
    if st not in _CONVERGENCE_STATUSES:
        _check(st, ctx.handle, "adjoint_grad")
    return st, {f: getattr(rep, f) for f, _ in _abi.Report._fields_}


def crs_write(directory: str, A: CSR, b, x=None):
    """Write the reference's CRS text files with the library's writer."""
    import os

    os.makedirs(directory, exist_ok=True)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(A.n) if x is None else np.ascontiguousarray(x, dtype=np.float64)
    ptr = np.ascontiguousarray(A.ptr, dtype=np.int32)
    col = np.ascontiguousarray(A.col, dtype=np.int32)
    val = np.ascontiguousarray(A.val, dtype=np.float64)
    _check(lib().ks_crs_write(directory.encode(), A.n, A.nnz, _ptr(ptr), _ptr(col), _ptr(val), _ptr(b), _ptr(x)),
           None, "crs_write")


def crs_read(directory: str):
    n, nnz = C.c_int64(), C.c_int64()
    _check(lib().ks_crs_read_header(directory.encode(), C.byref(n), C.byref(nnz)), None, "crs_read_header")
    ptr = np.zeros(n.value + 1, dtype=np.int32)
    col = np.zeros(nnz.value, dtype=np.int32)
    val = np.zeros(nnz.value)
    b = np.zeros(n.value)
    x = np.zeros(n.value)
    _check(lib().ks_crs_read(directory.encode(), n.value, nnz.value, _ptr(ptr), _ptr(col), _ptr(val), _ptr(b),
                             _ptr(x)), None, "crs_read")
    return CSR(ptr, col, val), b, x


def mm_read(file: str) -> CSR:
    """Read a Matrix Market coordinate file (real / integer / pattern;
    general / symmetric / skew-symmetric) into CSR with the library's reader."""
    n, nnz = C.c_int64(), C.c_int64()
    _check(lib().ks_mm_read_header(file.encode(), C.byref(n), C.byref(nnz)), None, "mm_read_header")
    ptr = np.zeros(n.value + 1, dtype=np.int32)
    col = np.zeros(max(nnz.value, 1), dtype=np.int32)
    val = np.zeros(max(nnz.value, 1))
    _check(lib().ks_mm_read(file.encode(), n.value, nnz.value, _ptr(ptr), _ptr(col), _ptr(val)), None, "mm_read")
    return CSR(ptr, col[:nnz.value], val[:nnz.value])


# ----------------------------------------------------------------- multi-GPU plan
def partition_rows(n: int, nranks: int, align: int = 1) -> np.ndarray:
    """Row blocks of a solve split over nranks GPUs (ks_partition_rows)."""
    rs = np.zeros(nranks + 1, dtype=np.int64)
    _check(lib().ks_partition_rows(n, nranks, align, _ptr(rs)), None, "partition_rows")
    return rs


def halo_window(A: CSR, r0: int, r1: int):
    """Column window [lo, hi) that rows r0..r1-1 of A read (ks_halo_window)."""
    lo, hi = C.c_int64(), C.c_int64()
    ptr = np.ascontiguousarray(A.ptr[r0:r1 + 1], dtype=np.int32)
    col = np.ascontiguousarray(A.col[A.ptr[r0]:A.ptr[r1]], dtype=np.int32)
    _check(lib().ks_halo_window(r0, r1, _ptr(ptr), _ptr(col) if col.size else None, C.byref(lo), C.byref(hi)),
           None, "halo_window")
    return lo.value, hi.value


def halo_plan(row_start, win_lo, win_hi, rank: int):
    """Per-peer send and receive row ranges of `rank` (ks_halo_plan)."""
    P = len(row_start) - 1
    rs = np.ascontiguousarray(row_start, dtype=np.int64)
    lo = np.ascontiguousarray(win_lo, dtype=np.int64)
    hi = np.ascontiguousarray(win_hi, dtype=np.int64)
    out = [np.zeros(P, dtype=np.int64) for _ in range(4)]
    _check(lib().ks_halo_plan(P, rank, _ptr(rs), _ptr(lo), _ptr(hi), *[_ptr(o) for o in out]), None, "halo_plan")
    return {"send": list(zip(out[0], out[1])), "recv": list(zip(out[2], out[3]))}


# ----------------------------------------------------------------- row-split solves
class Comm:
    """Transport of a row-split solve (``ks_comm``)."""

    def __init__(self, handle, ctx: Context):
        self.handle = handle
        self.ctx = ctx
        n, r = C.c_int(), C.c_int()
        _check(lib().ks_comm_info(handle, C.byref(n), C.byref(r)), None, "comm_info")
        self.nranks, self.rank = n.value, r.value

    @staticmethod
    def unique_id() -> bytes:
        """NCCL id made on rank 0, to be handed to every rank."""
        buf = C.create_string_buffer(128)
        _check(lib().ks_comm_unique_id(buf), None, "comm_unique_id")
        return buf.raw

    @classmethod
    def nccl(cls, ctx: Context, nranks: int, rank: int, uid: bytes) -> "Comm":
        h = C.c_void_p()
        buf = C.create_string_buffer(uid, 128)
        _check(lib().ks_comm_create_nccl(ctx.handle, nranks, rank, buf, C.byref(h)), ctx.handle, "comm_create_nccl")
        return cls(h, ctx)

    @classmethod
    def local(cls, ctxs) -> list:
        """Ranks emulated in this process, one context each (each rank's calls
        must then run on its own thread)."""
        P = len(ctxs)
        arr = (C.c_void_p * P)(*[c.handle for c in ctxs])
        out = (C.c_void_p * P)()
        _check(lib().ks_comm_create_local(arr, P, out), None, "comm_create_local")
        return [cls(C.c_void_p(out[q]), ctxs[q]) for q in range(P)]

    def close(self):
        if self.handle and self.ctx.handle:  # as Matrix.close
            lib().ks_comm_destroy(self.handle)
        self.handle = None


class SplitMatrix(Matrix):
    """This rank's rows r0..r1-1 of a row-split matrix (``ks_dist_upload``);
    solves on it take and return vectors of the local length r1 - r0."""

    def __init__(self, ctx: Context, comm: Comm, A: CSR, r0: int, r1: int, transpose=False, fp32=False,
                 bf16=False, index32=False, AT: CSR | None = None, diag=True):
        self.ctx = ctx
        self.comm = comm
        self.r0, self.r1, self.n_global = int(r0), int(r1), A.n
        self.n = self.r1 - self.r0
        j0, j1 = A.ptr[r0], A.ptr[r1]
        ptr = np.ascontiguousarray(A.ptr[r0:r1 + 1], dtype=np.int32)
        col = np.ascontiguousarray(A.col[j0:j1], dtype=np.int32)
        val = np.ascontiguousarray(A.val[j0:j1], dtype=np.float64)
        self.nnz = int(j1 - j0)
        tp = tc = tv = None
        if transpose:
            from .matrices import transpose as _transpose

            T = AT if AT is not None else _transpose(A)
            k0, k1 = T.ptr[r0], T.ptr[r1]
            tp = np.ascontiguousarray(T.ptr[r0:r1 + 1], dtype=np.int32)
            tc = np.ascontiguousarray(T.col[k0:k1], dtype=np.int32)
            tv = np.ascontiguousarray(T.val[k0:k1], dtype=np.float64)
        flags = (_abi.MAT_TRANSPOSE if transpose else 0) | (_abi.MAT_FP32 if fp32 else 0) | (
            _abi.MAT_BF16 if bf16 else 0) | (_abi.MAT_INDEX32 if index32 else 0) | (0 if diag else _abi.MAT_NO_DIAG)
        h = C.c_void_p()
        _check(lib().ks_dist_upload(ctx.handle, comm.handle, A.n, self.r0, self.r1, _ptr(ptr),
                                    _ptr(col) if col.size else None, _ptr(val) if val.size else None,
                                    _ptr(tp) if tp is not None else None,
                                    _ptr(tc) if tc is not None and tc.size else None,
                                    _ptr(tv) if tv is not None and tv.size else None, flags, C.byref(h)),
               ctx.handle, "ks_dist_upload")
        self.handle = h
        self.flags = flags

    def window(self):
        vals = [C.c_int64() for _ in range(5)]
        _check(lib().ks_mat_dist_info(self.handle, *[C.byref(v) for v in vals]), self.ctx.handle, "dist_info")
        return {k: v.value for k, v in zip(("n_global", "r0", "r1", "ext_lo", "ext_hi"), vals)}
