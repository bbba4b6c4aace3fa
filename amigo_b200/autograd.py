"""Differentiating through the KKT solve.

``kkt_solve(ldl, vals, diag, b)`` factors K (the CSR ``vals`` of ``ldl``'s
pattern plus the diagonal ``diag``) and returns x = K^{-1} b as a
``torch.autograd.Function``. The backward pass reuses the stored factor: the
adjoint lam = K^{-1} (dloss/dx) is one more solve (K is symmetric), and

    dloss/db       = lam
    dloss/vals[e]  = -sum_r lam[i, r] x[j, r]   for each stored entry e = (i, j)
    dloss/diag[i]  = -sum_r lam[i, r] x[i, r]

computed by a CUDA kernel of the library. This is the post-optimality
derivative the reference computes on the host with a factor and an adjoint
solve (amigo/algorithm/ipm_driver.py:297-353). Values are treated entry by
entry; for a parameterization that keeps K symmetric (one parameter drives
K(i, j) and K(j, i)), the entry-wise derivatives sum to the exact total
derivative.
"""

from __future__ import annotations

import torch

from .sparse_ldl import SparseLDL, SparseLDLBatch, Vector

__all__ = ["kkt_solve"]


class _KKTSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, diag, b, ldl):
        if not (vals.is_cuda and b.is_cuda):
            raise TypeError("kkt_solve needs CUDA tensors")
        v = vals.detach().contiguous().to(torch.float64)
        d = None if diag is None else diag.detach().contiguous().to(torch.float64)
        dv = Vector(d) if d is not None else None
        if isinstance(ldl, SparseLDLBatch):
            ldl.factor(dv, values=v)
        else:
            ldl.mat.vals = v
            ldl.factor(dv)
        x = b.detach().to(torch.float64).clone()
        if x.dim() == 2:
            x = x.t().contiguous().t()
        ldl.solve(x)
        ctx.ldl = ldl
        ctx.has_diag = diag is not None
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, gx):
        (x,) = ctx.saved_tensors
        ldl: SparseLDL = ctx.ldl
        lam = gx.detach().to(torch.float64).clone()
        if lam.dim() == 2:
            lam = lam.t().contiguous().t()
        ldl.solve(lam)
        gvals, gdiag = ldl.value_gradient(lam, x)
        return gvals, (gdiag if ctx.has_diag else None), lam, None


def kkt_solve(ldl: SparseLDL, vals: torch.Tensor, diag: torch.Tensor | None,
              b: torch.Tensor) -> torch.Tensor:
    """x = K^{-1} b with K = CSR(vals) + diag(diag) on ``ldl``'s pattern;
    differentiable in vals, diag and b. ``ldl`` may be a SparseLDLBatch:
    vals, diag and b are then the systems' arrays concatenated, and K is
    block diagonal. The factor is stored in ``ldl`` and
    reused by the backward pass, so call backward before refactoring
    ``ldl``."""
    return _KKTSolve.apply(vals, diag, b, ldl)
