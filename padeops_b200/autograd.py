"""torch.autograd.Function over the forward and adjoint line kernels.

``CompactOp.apply(op, kind, axis, f, bc1, bcn)`` returns D f for a scheme
object ``op`` (cd06 / cd10 / cf90) along ``axis``; its backward applies D^T
with the hand-written adjoint kernel (B^T A^{-T}, transposed closures
included).  Nothing is saved for backward beyond the operator itself: D is
linear, so the adjoint needs only the incoming gradient.

Fields follow the library convention: a contiguous CUDA float64 tensor whose
memory is the column-major field f(n1,n2,n3), i.e. shape (n3, n2, n1).
"""
from __future__ import annotations

import torch

from . import _lib as L
from .operators import _Scheme

__all__ = ["CompactOp", "compact_op", "ddx", "ddy", "ddz"]


def _na_nb(shape: tuple[int, ...], axis: int) -> tuple[int, int]:
    n3, n2, n1 = shape
    return {1: (n2, n3), 2: (n1, n3), 3: (n1, n2)}[axis]


class CompactOp(torch.autograd.Function):
    @staticmethod
    def forward(ctx, op: _Scheme, kind: int, axis: int, f: torch.Tensor, bc1: int = 0, bcn: int = 0):
        if f.dim() != 3:
            raise ValueError("f must be a 3-d tensor of shape (n3, n2, n1)")
        f = f.contiguous()
        na, nb = _na_nb(tuple(f.shape), axis)
        out = torch.empty_like(f)
        op.apply(kind, axis, f, out, na, nb, bc1, bcn)
        ctx.op, ctx.kind, ctx.axis, ctx.bc1, ctx.bcn, ctx.shape = op, kind, axis, bc1, bcn, tuple(f.shape)
        return out

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        g = g.contiguous()
        na, nb = _na_nb(ctx.shape, ctx.axis)
        fbar = torch.empty_like(g)
        ctx.op.apply(ctx.kind, ctx.axis, g, fbar, na, nb, ctx.bc1, ctx.bcn, adjoint=True)
        return None, None, None, fbar, None, None


def compact_op(op: _Scheme, kind: int, axis: int, f: torch.Tensor, bc1: int = 0, bcn: int = 0) -> torch.Tensor:
    """Differentiable D f (see module docstring)."""
    return CompactOp.apply(op, kind, axis, f, bc1, bcn)


def ddx(op, f, bc1=0, bcn=0):
    return compact_op(op, L.D1, 1, f, bc1, bcn)


def ddy(op, f, bc1=0, bcn=0):
    return compact_op(op, L.D1, 2, f, bc1, bcn)


def ddz(op, f, bc1=0, bcn=0):
    return compact_op(op, L.D1, 3, f, bc1, bcn)
