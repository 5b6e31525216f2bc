"""Reproducible scatter adjoint of the 3-D on-the-fly projector.

``back_project_3d_fixed_cuda`` computes A^T y with the walk of
``back_project_3d_on_the_fly_cuda`` (the same rays, voxels and segment
lengths, under either voxel rule and for any ray layout) but adds every
contribution ``y * len`` as a 64-bit fixed-point integer
(ctlab_back_project_3d_fixed): integer addition is associative, so the volume
is bitwise the same on every run and whatever else shares the GPU.  The
fixed-point step 2^-e is chosen per sinogram on the device from
max|y| * (the grid's longest world diagonal) * n_ray <= 2^61, so no sum can
overflow; each contribution is rounded once, a relative error near 2^-61 * n_ray
of the largest possible sum, and the volume is then rounded once to float.
The reference has no counterpart: its adjoints scatter with float atomicAdd
(src/ct_projector_3d.cu:1005), whose last bits depend on the order in which
the additions land.
"""
from __future__ import annotations

import torch

from .. import _layout
from .. import _native as N
from ._common import inverse, require_cuda, single_affine

__all__ = ["back_project_3d_fixed_cuda", "fixed_workspace_bytes"]


def fixed_workspace_bytes(batch: int, n_x: int, n_y: int, n_z: int) -> int:
    """Bytes of device workspace one call needs (an int64 volume per sinogram
    plus a small header)."""
    n = int(N.lib.ctlab_back_project_3d_fixed_workspace_bytes(batch, n_x, n_y, n_z))
    if n < 0:
        raise ValueError(f"invalid batch or grid: {batch}, ({n_x}, {n_y}, {n_z})")
    return n


def back_project_3d_fixed_cuda(sinogram, src, dst, M, b, n_x, n_y, n_z, tiling=None, M_inv=None, out=None,
                               accumulate=False, workspace=None):
    """Reproducible A^T y: [B, n_x, n_y, n_z] (or [n_x, n_y, n_z] for a 1-D
    sinogram).  Arguments as back_project_3d_on_the_fly_cuda; ``out`` (a
    float32 volume to write, or with ``accumulate`` to add to) and
    ``workspace`` (a uint8 CUDA tensor of at least fixed_workspace_bytes
    bytes) let a caller keep the buffers between calls."""
    M, b = single_affine(M, b)
    if sinogram.dtype != torch.float32 or not sinogram.is_contiguous():
        raise RuntimeError("sinogram must be a C-contiguous float32 tensor")
    require_cuda(sinogram, src, dst, M, b)
    Mi = inverse(M) if M_inv is None else M_inv
    if tiling is None:
        tiling = _layout.detect_tiling(src, dst)
    squeeze = sinogram.dim() == 1
    sino = sinogram.unsqueeze(0) if squeeze else sinogram
    batch, n_ray = int(sino.shape[0]), int(sino.shape[1])
    if n_ray != src.shape[0]:
        raise RuntimeError(f"sinogram has {n_ray} rays, geometry {src.shape[0]}")
    need = fixed_workspace_bytes(batch, n_x, n_y, n_z)
    if workspace is None:
        workspace = torch.empty(need, dtype=torch.uint8, device=sino.device)
    elif workspace.numel() < need or workspace.dtype != torch.uint8 or workspace.device != sino.device:
        raise RuntimeError(f"workspace must be a uint8 tensor of >= {need} bytes on {sino.device}")
    if out is None:
        out = torch.empty((batch, n_x, n_y, n_z), device=sino.device, dtype=torch.float32)
        accumulate = False
    elif tuple(out.shape[-3:]) != (n_x, n_y, n_z) or out.numel() != batch * n_x * n_y * n_z or \
            out.dtype != torch.float32 or not out.is_contiguous():
        raise RuntimeError("out must be a contiguous float32 [B, n_x, n_y, n_z] volume")
    act = getattr(tiling, "active", None)  # a list of active tiles (_native.active_tiling): walk only those
    tiles, n_tiles = (N.ptr(act[0]), act[1]) if act is not None else (None, -1)
    with torch.cuda.device(sino.device):
        N.call("ctlab_back_project_3d_fixed", N.ptr(sino), batch, n_ray, N.ptr(src), N.ptr(dst), N.ptr(Mi),
               N.ptr(b), n_x, n_y, n_z, N.ptr(out), int(bool(accumulate)), N.tiling_ref(tiling), tiles, n_tiles,
               N.ptr(workspace), workspace.numel(), N.stream_of(sino))
    return out.reshape(n_x, n_y, n_z) if squeeze and out.dim() == 4 else out
