"""3-D projector functions: the reference's function-level CUDA API.

Same names, argument orders and shape conventions as the reference's
tomography/ct_projector_3d_cuda.py (note its mixed orders:
``forward_project_3d_cuda(volume, tvals, src, dst, M, b)`` but
``forward_project_3d_on_the_fly_cuda(volume, M, b, src, dst)``).  ``tvals``
may be None or empty (on the fly), a float table, or a
``(t_uint16, t_start, t_scale)`` tuple (compressed).  Unbatched inputs give
unbatched outputs.

One deliberate difference: the reference's ``back_project_3d_cuda`` with no
tvals inverts M twice (ct_projector_3d_cuda.py:209-210 then :319), so its
on-the-fly adjoint uses M instead of M^-1 and is wrong whenever M != I.  Here
M is inverted once on every path, so the adjoint is the transpose of the
forward for any affine.
"""
from __future__ import annotations

import torch

from .. import _C
from ._common import inverse, require_cuda, single_affine, voxel_diag_len

__all__ = [
    "compute_intersections_3d_cuda",
    "compress_tvals_3d_cuda",
    "forward_project_3d_cuda",
    "forward_project_3d_compressed_cuda",
    "back_project_3d_cuda",
    "back_project_3d_compressed_cuda",
    "forward_project_3d_on_the_fly_cuda",
    "back_project_3d_on_the_fly_cuda",
]


def _empty_or_none(t) -> bool:
    if t is None:
        return True
    if isinstance(t, (tuple, list)):
        return len(t) == 0
    return t.numel() == 0


def _check_f32(**tensors):
    for name, t in tensors.items():
        assert t.is_contiguous(), f"{name} must be C-contiguous"
        assert t.dtype == torch.float32, f"{name} must be float32"


def compute_intersections_3d_cuda(n_x, n_y, n_z, M, b, src, dst, M_inv=None):
    """Sorted plane parameters of every ray, [n_ray, (n_x+1)+(n_y+1)+(n_z+1)]
    (reference ct_projector_3d_cuda.py:62-83)."""
    M, b = single_affine(M, b)
    require_cuda(src, dst, M, b)
    return _C.compute_intersections_3d(n_x, n_y, n_z, src, dst, inverse(M) if M_inv is None else M_inv, b)


def compress_tvals_3d_cuda(tvals, M, src, dst):
    """uint16 delta encoding with the reference CUDA encoder
    (ct_projector_3d_cuda.py:85-106)."""
    require_cuda(tvals, src, dst)
    return _C.compress_tvals_3d_cuda(tvals, src, dst, voxel_diag_len(M))


def forward_project_3d_cuda(volume, tvals, src, dst, M, b, tiling=None, M_inv=None):
    """Line integrals [B, n_ray] (or [n_ray] for a 3-D volume)
    (reference ct_projector_3d_cuda.py:112-161)."""
    M, b = single_affine(M, b)
    _check_f32(volume=volume, src=src, dst=dst, M=M, b=b)
    require_cuda(volume, src, dst, M, b)
    if _empty_or_none(tvals):
        return forward_project_3d_on_the_fly_cuda(volume, M, b, src, dst, tiling=tiling, M_inv=M_inv)
    Mi = inverse(M) if M_inv is None else M_inv
    if isinstance(tvals, (tuple, list)):
        t_uint16, t_start, t_scale = tvals
        out = _C.forward_project_3d_compressed_cuda(volume, t_uint16, t_start, t_scale, src, dst, Mi, b)
    else:
        assert tvals.dtype == torch.float32, "tvals must be float32"
        out = _C.forward_project_3d_cuda(volume, tvals, src, dst, Mi, b)
    if volume.dim() == 3:
        out = out.squeeze(0)
    return out


def forward_project_3d_compressed_cuda(volume, t_uint16, t_start, t_scale, M, b, src, dst, M_inv=None):
    """Forward projection from a compressed table
    (reference ct_projector_3d_cuda.py:163-180)."""
    M, b = single_affine(M, b)
    require_cuda(volume, src, dst, M, b)
    out = _C.forward_project_3d_compressed_cuda(volume, t_uint16, t_start, t_scale, src, dst,
                                                inverse(M) if M_inv is None else M_inv, b)
    if volume.dim() == 3:
        out = out.squeeze(0)
    return out


def back_project_3d_cuda(sinogram, tvals, src, dst, M, b, n_x, n_y, n_z, tiling=None, M_inv=None):
    """Adjoint [B, n_x, n_y, n_z] (or [n_x, n_y, n_z] for a 1-D sinogram)
    (reference ct_projector_3d_cuda.py:188-225)."""
    assert sinogram.is_contiguous(), "sinogram must be C-contiguous"
    assert sinogram.dtype == torch.float32, "sinogram must be float32"
    M, b = single_affine(M, b)
    require_cuda(sinogram, src, dst, M, b)
    if _empty_or_none(tvals):
        return back_project_3d_on_the_fly_cuda(sinogram, src, dst, M, b, n_x, n_y, n_z, tiling=tiling, M_inv=M_inv)
    Mi = inverse(M) if M_inv is None else M_inv
    if isinstance(tvals, (tuple, list)):
        t_uint16, t_start, t_scale = tvals
        out = _C.back_project_3d_compressed_cuda(sinogram, t_uint16, t_start, t_scale, src, dst, Mi, b, n_x, n_y,
                                                 n_z)
    else:
        assert tvals.dtype == torch.float32, "tvals must be float32"
        out = _C.back_project_3d_cuda(sinogram, tvals, src, dst, Mi, b, n_x, n_y, n_z)
    if sinogram.dim() == 1:
        out = out.squeeze(0)
    return out


def back_project_3d_compressed_cuda(sinogram, t_uint16, t_start, t_scale, M, b, src, dst, n_x, n_y, n_z,
                                    M_inv=None):
    """Adjoint from a compressed table (reference ct_projector_3d_cuda.py:228-248)."""
    M, b = single_affine(M, b)
    require_cuda(sinogram, src, dst, M, b)
    out = _C.back_project_3d_compressed_cuda(sinogram, t_uint16, t_start, t_scale, src, dst,
                                             inverse(M) if M_inv is None else M_inv, b, n_x, n_y, n_z)
    if sinogram.dim() == 1:
        out = out.squeeze(0)
    return out


def forward_project_3d_on_the_fly_cuda(volume, M, b, src, dst, tiling=None, M_inv=None):
    """Siddon forward projection without a table
    (reference ct_projector_3d_cuda.py:254-289)."""
    M, b = single_affine(M, b)
    M = M.contiguous().to(torch.float32)
    b = b.contiguous().to(torch.float32)
    _check_f32(volume=volume, src=src, dst=dst, M=M, b=b)
    require_cuda(volume, src, dst, M, b)
    out = _C.forward_project_3d_on_the_fly_cuda(volume, src, dst, inverse(M) if M_inv is None else M_inv, b,
                                                tiling=tiling)
    if volume.dim() == 3:
        out = out.squeeze(0)
    return out


def back_project_3d_on_the_fly_cuda(sinogram, src, dst, M, b, n_x, n_y, n_z, tiling=None, M_inv=None):
    """Exact adjoint of forward_project_3d_on_the_fly_cuda
    (reference ct_projector_3d_cuda.py:292-323, M inverted once)."""
    M, b = single_affine(M, b)
    _check_f32(sinogram=sinogram, src=src, dst=dst, M=M, b=b)
    require_cuda(sinogram, src, dst, M, b)
    out = _C.back_project_3d_on_the_fly_cuda(sinogram, src, dst, inverse(M) if M_inv is None else M_inv, b, n_x,
                                             n_y, n_z, tiling=tiling)
    if sinogram.dim() == 1:
        out = out.squeeze(0)
    return out
