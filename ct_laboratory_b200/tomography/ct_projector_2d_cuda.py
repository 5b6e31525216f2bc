"""2-D projector functions: the reference's function-level CUDA API.

Same names and argument orders as the reference's
tomography/ct_projector_2d_cuda.py (2-D takes ``(image, tvals, M, b, src,
dst)``).  ``tvals=None`` is an addition: it runs the table-free Siddon kernel
(same plane parameters evaluated on the fly).
"""
from __future__ import annotations

import torch

from .. import _C
from .. import _native as N
from ._common import inverse, require_cuda

__all__ = ["compute_intersections_2d_cuda", "forward_project_2d_cuda", "back_project_2d_cuda",
           "forward_project_2d_siddon", "back_project_2d_siddon"]


def compute_intersections_2d_cuda(n_row, n_col, M, b, src, dst, M_inv=None):
    """[n_ray, (n_row+1)+(n_col+1)] sorted plane parameters
    (reference ct_projector_2d_cuda.py:11-18)."""
    require_cuda(src, dst, M, b)
    return _C.compute_intersections_2d(n_row, n_col, src, dst, inverse(M) if M_inv is None else M_inv, b)


def forward_project_2d_cuda(image, tvals, M, b, src, dst, tiling=None, M_inv=None):
    """[B, n_ray] or [n_ray] line integrals (reference ct_projector_2d_cuda.py:21-31)."""
    require_cuda(image, src, dst, M, b)
    Mi = inverse(M) if M_inv is None else M_inv
    if tvals is None:
        out = forward_project_2d_siddon(image, Mi, b, src, dst, tiling)
    else:
        out = _C.forward_project_2d_cuda(image, tvals, src, dst, Mi, b)
    if image.dim() == 2:
        out = out.squeeze(0)
    return out


def back_project_2d_cuda(sinogram, tvals, M, b, src, dst, n_row, n_col, tiling=None, M_inv=None):
    """[B, R, C] or [R, C] adjoint (reference ct_projector_2d_cuda.py:34-46)."""
    require_cuda(sinogram, src, dst, M, b)
    Mi = inverse(M) if M_inv is None else M_inv
    if tvals is None:
        out = back_project_2d_siddon(sinogram, Mi, b, src, dst, n_row, n_col, tiling)
    else:
        out = _C.back_project_2d_cuda(sinogram.contiguous(), tvals, src, dst, Mi, b, n_row, n_col)
    if sinogram.dim() == 1:
        out = out.squeeze(0)
    return out


def _check(src, dst, M_inv, b, *data):
    for t in (src, dst, M_inv, b, *data):
        if t.dtype != torch.float32 or not t.is_contiguous() or not t.is_cuda:
            raise RuntimeError("2-D Siddon: tensors must be C-contiguous float32 CUDA tensors")
    if src.dim() != 2 or src.shape[1] != 2 or dst.shape != src.shape:
        raise RuntimeError(f"src/dst must be [n_ray, 2] (got {tuple(src.shape)}, {tuple(dst.shape)})")


def forward_project_2d_siddon(image, M_inv, b, src, dst, tiling=None):
    """Table-free 2-D Siddon forward, always batched [B, n_ray]."""
    img = image.contiguous()
    _check(src, dst, M_inv, b, img)
    batch, n_row, n_col = (1, *img.shape) if img.dim() == 2 else img.shape
    n_ray = src.shape[0]
    out = torch.empty((batch, n_ray), device=img.device, dtype=torch.float32)
    with torch.cuda.device(img.device):
        N.call("ctlab_forward_project_2d_siddon", N.ptr(img), batch, n_row, n_col, N.ptr(src), N.ptr(dst), n_ray,
               N.ptr(M_inv), N.ptr(b), N.ptr(out), N.tiling_ref(tiling), N.stream_of(img))
    return out


def back_project_2d_siddon(sinogram, M_inv, b, src, dst, n_row, n_col, tiling=None):
    """Exact adjoint of forward_project_2d_siddon, always batched [B, R, C].
    Rays running along the image's columns accumulate in a transposed
    scratch image (ctlab_back_project_2d_siddon_ws)."""
    sino = sinogram.contiguous()
    _check(src, dst, M_inv, b, sino)
    batch, n_ray = (1, sino.shape[0]) if sino.dim() == 1 else sino.shape
    out = torch.empty((batch, n_row, n_col), device=sino.device, dtype=torch.float32)
    scratch = torch.empty_like(out) if n_ray > 0 else None
    with torch.cuda.device(sino.device):
        N.call("ctlab_back_project_2d_siddon_ws", N.ptr(sino), batch, n_ray, N.ptr(src), N.ptr(dst), N.ptr(M_inv),
               N.ptr(b), n_row, n_col, N.ptr(out), 0, N.tiling_ref(tiling), N.ptr(scratch), N.stream_of(sino))
    return out
