"""Optional torch.autograd binding of a sparse solve x = A^{-1} b.

``sparse_solve(ctx, pattern, values, b, method="CG", **params)`` returns x as
a torch tensor and, under autograd, propagates a loss gradient g = dL/dx to
the right-hand side and to the CSR values through the library's adjoint
(``ks_adjoint_grad``: A^T lambda = g solved with the same method on the
transpose, grad_b = lambda, grad_val[j] = -lambda[row(j)] * x[col(j)]).
It exists to check those gradients against finite differences and dense
references (torch.autograd.gradcheck); every call uploads the matrix, so it
is not a fast path. The reference has no gradients at all.
"""
from __future__ import annotations

import numpy as np
import torch

from . import CSR, Context, Matrix, adjoint_grad, solve

__all__ = ["sparse_solve"]


class _SparseSolve(torch.autograd.Function):
    @staticmethod
    def forward(fctx, values, b, kctx, pattern, method, params):
        A = CSR(pattern.ptr, pattern.col, values.detach().cpu().numpy().astype(np.float64))
        M = Matrix(kctx, A, transpose=True)
        try:
            r = solve(kctx, M, method, b.detach().cpu().numpy().astype(np.float64), **params)
        finally:
            M.close()
        if r.status != 0:
            raise RuntimeError(f"{method} did not converge (status {r.status})")
        x = torch.from_numpy(r.x).to(dtype=values.dtype, device=values.device)
        fctx.save_for_backward(values, x)
        fctx.kctx, fctx.pattern, fctx.method, fctx.params = kctx, pattern, method, params
        return x

    @staticmethod
    def backward(fctx, grad_x):
        values, x = fctx.saved_tensors
        kctx, pattern = fctx.kctx, fctx.pattern
        if not bool(torch.any(grad_x != 0)):
            # A^T lambda = 0 has lambda = 0; the solvers' relative stopping
            # test |r| / |b| is undefined for a zero right-hand side
            return torch.zeros_like(values), torch.zeros_like(x), None, None, None, None
        A = CSR(pattern.ptr, pattern.col, values.detach().cpu().numpy().astype(np.float64))
        M = Matrix(kctx, A, transpose=True)
        try:
            X = kctx.vector(x.detach().cpu().numpy().astype(np.float64))
            G = kctx.vector(grad_x.detach().cpu().numpy().astype(np.float64))
            GB, GV = kctx.vector(n=A.n), kctx.vector(n=A.nnz)
            st, _ = adjoint_grad(kctx, M, fctx.method, X, G, GB, GV, **fctx.params)
            if st != 0:
                raise RuntimeError(f"adjoint {fctx.method} did not converge (status {st})")
            gb = torch.from_numpy(GB.numpy()).to(dtype=values.dtype, device=values.device)
            gv = torch.from_numpy(GV.numpy()).to(dtype=values.dtype, device=values.device)
            for v in (X, G, GB, GV):
                v.close()
        finally:
            M.close()
        return gv, gb, None, None, None, None


def sparse_solve(ctx: Context, pattern: CSR, values: torch.Tensor, b: torch.Tensor, method: str = "CG",
                 **params) -> torch.Tensor:
    """x = A^{-1} b with A = (pattern.ptr, pattern.col, values); differentiable
    in ``values`` and ``b``. ``params`` are ks_params fields or the reference's
    flag letters (E, L, R, ...)."""
    return _SparseSolve.apply(values, b, ctx, pattern, method, dict(params))
