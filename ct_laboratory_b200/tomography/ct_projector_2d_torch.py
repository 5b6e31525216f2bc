"""Names of the reference's pure-PyTorch 2-D backend
(tomography/ct_projector_2d_torch.py), served by the CUDA kernels: same
signatures (M, not M^-1), CUDA tensors only."""
from __future__ import annotations

from .. import _C
from ._common import inverse, require_cuda

__all__ = ["compute_intersections_2d_torch", "forward_project_2d_torch", "back_project_2d_torch"]


def compute_intersections_2d_torch(n_row, n_col, M, b, src, dst):
    require_cuda(src, dst, M, b)
    return _C.compute_intersections_2d(n_row, n_col, src, dst, inverse(M), b)


def forward_project_2d_torch(image, t_sorted, M, b, src, dst):
    require_cuda(image, t_sorted, src, dst, M, b)
    out = _C.forward_project_2d_cuda(image.contiguous(), t_sorted, src, dst, inverse(M), b)
    return out.squeeze(0) if image.dim() == 2 else out


def back_project_2d_torch(sinogram, t_sorted, M, b, src, dst, n_row, n_col):
    require_cuda(sinogram, t_sorted, src, dst, M, b)
    out = _C.back_project_2d_cuda(sinogram.contiguous(), t_sorted, src, dst, inverse(M), b, n_row, n_col)
    return out.squeeze(0) if sinogram.dim() == 1 else out
