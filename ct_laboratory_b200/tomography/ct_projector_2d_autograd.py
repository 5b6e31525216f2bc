"""Autograd Function of the 2-D projector (forward = A, backward = A^T).

Mirrors the reference's CTProjector2DFunction
(tomography/ct_projector_2d_autograd.py:16-72): arguments
``(image, tvals, M, b, src, dst, backend)``; ``tvals=None`` selects the
table-free kernel.  Optional trailing ``tiling``, ``M_inv`` and ``adjoint``
(a callable y -> A^T y used by the backward instead of the atomic adjoint,
e.g. the deterministic gather).
"""
from __future__ import annotations

import torch

from .ct_projector_2d_cuda import back_project_2d_cuda, forward_project_2d_cuda

__all__ = ["CTProjector2DFunction"]


class CTProjector2DFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image, tvals, M, b, src, dst, backend="cuda", tiling=None, M_inv=None, adjoint=None):
        if backend not in ("cuda", "torch"):
            raise ValueError(f"unknown backend {backend!r}")
        ctx.tvals = tvals
        ctx.geom = (M, b, src, dst)
        ctx.tiling = tiling
        ctx.M_inv = M_inv
        ctx.adjoint = adjoint
        ctx.image_shape = image.shape
        return forward_project_2d_cuda(image.contiguous(), tvals, M, b, src, dst, tiling=tiling, M_inv=M_inv)

    @staticmethod
    def backward(ctx, grad_output):
        M, b, src, dst = ctx.geom
        n_row, n_col = ctx.image_shape[-2:]
        if ctx.adjoint is not None:
            grad = ctx.adjoint(grad_output.contiguous())
        else:
            grad = back_project_2d_cuda(grad_output.contiguous(), ctx.tvals, M, b, src, dst, n_row, n_col,
                                        tiling=ctx.tiling, M_inv=ctx.M_inv)
        return grad.reshape(ctx.image_shape), None, None, None, None, None, None, None, None, None
