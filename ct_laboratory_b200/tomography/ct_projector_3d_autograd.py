"""Autograd Function of the 3-D projector: forward = A, backward = A^T.

Mirrors the reference's CTProjector3DFunction
(tomography/ct_projector_3d_autograd.py:16-170): same positional arguments
``(volume, t_main, t_start, t_scale, M, b, src, dst, backend)`` where
``t_main`` is None (on the fly), a float table, or the uint16 table when
``t_start``/``t_scale`` are given.  Gradients flow to the volume only.

Differences from the reference, none of which change the arithmetic:
 * the compressed path runs as one launch over all rays instead of a Python
   loop over 65536-ray chunks (reference :70, :141);
 * ``backend`` may be 'cuda' or 'torch'; both run the CUDA kernels (there is
   no CPU implementation);
 * four optional trailing arguments: ``tiling`` (launch options of the
   on-the-fly kernels), ``M_inv`` (a precomputed M^-1 so that modules can
   skip the per-call inversion), ``panels`` (a flat-panel table: the
   backward then gathers deterministically instead of scattering) and
   ``fixed_adjoint`` (the backward scatters in 64-bit fixed point:
   reproducible, same walk as the forward).
"""
from __future__ import annotations

import torch

from .ct_projector_3d_cuda import back_project_3d_cuda, forward_project_3d_cuda
from .fixed_adjoint import back_project_3d_fixed_cuda
from .gather import back_project_3d_gather_cuda

__all__ = ["CTProjector3DFunction"]


class CTProjector3DFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volume, t_main, t_start, t_scale, M, b, src, dst, backend="cuda", tiling=None, M_inv=None,
                panels=None, fixed_adjoint=False):
        if backend not in ("cuda", "torch"):
            raise ValueError(f"unknown backend {backend!r}")
        compressed = t_start is not None and t_scale is not None
        tv = (t_main, t_start, t_scale) if compressed else t_main
        ctx.tvals = tv
        ctx.geom = (M, b, src, dst)
        ctx.tiling = tiling
        ctx.M_inv = M_inv
        ctx.panels = panels
        ctx.fixed_adjoint = bool(fixed_adjoint)
        ctx.volume_shape = volume.shape
        ctx.compressed = compressed
        vol = volume.contiguous()
        sino = forward_project_3d_cuda(vol, tv, src, dst, M, b, tiling=tiling, M_inv=M_inv)
        if compressed and vol.dim() == 4 and vol.shape[0] == 1:
            # the reference's chunked compressed path returns [n_ray] for a
            # batch of one (ct_projector_3d_autograd.py:72-73)
            sino = sino.reshape(-1)
        return sino

    @staticmethod
    def backward(ctx, grad_output):
        M, b, src, dst = ctx.geom
        shape = ctx.volume_shape
        n_x, n_y, n_z = shape[-3:]
        g = grad_output.contiguous()
        if len(shape) == 4 and g.dim() == 1:
            g = g.unsqueeze(0)
        if ctx.panels is not None and ctx.tvals is None:
            grad = back_project_3d_gather_cuda(g, src, dst, M, b, n_x, n_y, n_z, ctx.panels, M_inv=ctx.M_inv)
        elif ctx.fixed_adjoint and ctx.tvals is None:
            grad = back_project_3d_fixed_cuda(g, src, dst, M, b, n_x, n_y, n_z, tiling=ctx.tiling, M_inv=ctx.M_inv)
        else:
            grad = back_project_3d_cuda(g, ctx.tvals, src, dst, M, b, n_x, n_y, n_z, tiling=ctx.tiling,
                                        M_inv=ctx.M_inv)
        return grad.reshape(shape), None, None, None, None, None, None, None, None, None, None, None, None
