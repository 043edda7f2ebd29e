"""The H-matvec as a differentiable torch operation.

``HmatApply`` is a ``torch.autograd.Function``.
* Forward: y = H x.
* Backward: grad_x = Hᵀ grad_y, computed by the transposed kernel.
  That kernel applies Aᵀ block by block: FR blocks as Aᵀ, LR blocks as Bᵀ(Aᵀ g).
  Its output is owned by column panels, and no symmetry of H is assumed.
* Double backward: backward is the same Function with the transpose flag flipped.
  The operation is linear, so any order of differentiation works.

This lets a displacement-discontinuity field be fitted to target tractions
with torch optimisers, e.g. min ½‖H x − t*‖² by L-BFGS.  The reference has no
counterpart.  Its Python binding (interfaces/python/py_bigwham.cc:192-233,
bigwham4py/bigwham4py.py:143-181) only offers the forward product.

The operator object needs ``matvec(x, precision, transpose=…, permuted=…, out=…)``
on CUDA float64 vectors.  It also needs ``n_rows`` / ``n_cols``, and
``has_transpose`` for backward.  ``HmatGpu`` finalized with ``transpose=True``
provides all of these; it accepts CUDA tensors only and raises on anything else.
"""
from __future__ import annotations

import torch


def _apply_columns(op, x: torch.Tensor, precision: str, transpose: bool, permuted: bool) -> torch.Tensor:
    """op applied to x (n,) or to each column of x (n, k); float64 on x's device."""
    nout = op.n_cols if transpose else op.n_rows
    xd = x.detach()
    if xd.dtype != torch.float64:
        xd = xd.to(torch.float64)
    if xd.dim() == 1:
        y = torch.empty(nout, dtype=torch.float64, device=x.device)
        op.matvec(xd.contiguous(), precision, transpose=transpose, permuted=permuted, out=y)
        return y
    if hasattr(op, "matmat"):  # one call: the tensor-core path where the handle has it
        return op.matmat(xd, precision, permuted=permuted, transpose=transpose)
    xt = xd.t().contiguous()  # (k, n): each right-hand side contiguous
    yt = torch.empty(xt.shape[0], nout, dtype=torch.float64, device=x.device)
    for k in range(xt.shape[0]):
        op.matvec(xt[k], precision, transpose=transpose, permuted=permuted, out=yt[k])
    return yt.t()


class HmatApply(torch.autograd.Function):
    """y = H x (Hᵀ x with transpose=True); x of shape (n,) or (n, k).

    The kernels compute in the storage ``precision`` ("fp64", "fp32" or "bf16")
    and return float64; y has x's dtype.
    """

    @staticmethod
    def forward(ctx, x, op, precision="fp64", transpose=False, permuted=False):
        nin = op.n_rows if transpose else op.n_cols
        if x.dim() not in (1, 2) or x.shape[0] != nin:
            raise ValueError(f"x must have {nin} rows, got shape {tuple(x.shape)}")
        ctx.op, ctx.precision, ctx.transpose, ctx.permuted = op, precision, transpose, permuted
        ctx.in_dtype = x.dtype
        return _apply_columns(op, x, precision, transpose, permuted).to(x.dtype)

    @staticmethod
    def backward(ctx, g):
        gx = None
        if ctx.needs_input_grad[0]:
            if not ctx.transpose and not getattr(ctx.op, "has_transpose", False):
                raise RuntimeError("backward needs the transposed layout (finalize with transpose=True)")
            gx = HmatApply.apply(g.contiguous(), ctx.op, ctx.precision, not ctx.transpose, ctx.permuted)
            gx = gx.to(ctx.in_dtype)
        return gx, None, None, None, None


def hmatvec(x: torch.Tensor, op, precision: str = "fp64", transpose: bool = False,
            permuted: bool = False) -> torch.Tensor:
    """Differentiable y = H x (or Hᵀ x); see ``HmatApply``."""
    return HmatApply.apply(x, op, precision, transpose, permuted)


class TractionMisfit(torch.nn.Module):
    """½‖H x − t*‖² / ‖t*‖², the misfit for inverting a displacement-discontinuity
    field x from target tractions t* (both in original dof ordering)."""

    def __init__(self, op, target: torch.Tensor, precision: str = "fp64"):
        super().__init__()
        self.op, self.precision = op, precision
        self.register_buffer("target", target)
        self.scale = 1.0 / float(torch.dot(target, target))

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        r = hmatvec(x, self.op, self.precision) - self.target
        return 0.5 * self.scale * torch.dot(r, r)
