"""Names of the reference's pure-PyTorch 3-D backend, served by the CUDA kernels.

The reference's tomography/ct_projector_3d_torch.py implements the projector
with vectorised torch ops on any device.  This package has no CPU
implementation: these functions keep the same names and signatures (M, not
M^-1; unbatched volumes; ``t_sorted_arg`` a float table or a
``(t_uint16, t_start, t_scale)`` tuple) and run the CUDA kernels, raising for
CPU tensors.  The table codecs match the reference's torch functions:
``compress_tvals_to_uint16`` uses the torch encoder (inf -> 10.0, round half
to even, float running sum) and ``decompress_tvals_from_uint16`` the float
cumulative sum.
"""
from __future__ import annotations

import torch

from .. import _C
from ._common import inverse, require_cuda, single_affine

__all__ = [
    "compress_tvals_to_uint16",
    "decompress_tvals_from_uint16",
    "compute_intersections_3d_torch",
    "forward_project_3d_torch",
    "back_project_3d_torch",
]


def _diag_len_tensor(M):
    diags = torch.tensor([[1, 1, 1], [1, 1, -1], [1, -1, 1], [-1, 1, 1]], device=M.device, dtype=M.dtype).t()
    return torch.norm(M @ diags, dim=0).max()


def compress_tvals_to_uint16(tvals, M, src, dst):
    """(t_uint16 as int16 [N, K], starts [N], scales [N]) with the reference
    torch encoder (ct_projector_3d_torch.py:4-65).  The voxel diagonal is
    evaluated with the same torch ops on M's device."""
    if tvals.numel() == 0:
        return tvals.to(torch.int16), torch.empty(0, device=tvals.device), torch.empty(0, device=tvals.device)
    require_cuda(tvals, src, dst)
    M = M[0] if M.dim() > 2 else M
    vdl = _diag_len_tensor(M).item()
    return _C.compress_tvals_3d_mode(tvals.float().contiguous(), src.float().contiguous(), dst.float().contiguous(),
                                     vdl, mode=1)


def decompress_tvals_from_uint16(tvals_uint16, starts, scales):
    """Float table from the delta encoding: cumulative sum, times scale, plus
    start (ct_projector_3d_torch.py:68-75).  Works on any device."""
    t = tvals_uint16.view(torch.uint16).to(torch.float32) if tvals_uint16.dtype == torch.int16 else \
        tvals_uint16.to(torch.float32)
    t = t.cumsum_(dim=1)
    t.mul_(scales.unsqueeze(1))
    t.add_(starts.unsqueeze(1))
    return t


def compute_intersections_3d_torch(n_x, n_y, n_z, M, b, src, dst):
    M, b = single_affine(M, b)
    require_cuda(src, dst, M, b)
    return _C.compute_intersections_3d(n_x, n_y, n_z, src.float().contiguous(), dst.float().contiguous(),
                                       inverse(M), b.float().contiguous())


def forward_project_3d_torch(volume, t_sorted_arg, M, b, src, dst):
    M, b = single_affine(M, b)
    require_cuda(volume, src, dst, M, b)
    Mi = inverse(M)
    if isinstance(t_sorted_arg, (tuple, list)):
        t16, ts, tsc = t_sorted_arg
        out = _C.forward_project_3d_compressed_cuda(volume, t16, ts, tsc, src, dst, Mi, b)
    else:
        out = _C.forward_project_3d_cuda(volume, t_sorted_arg, src, dst, Mi, b)
    return out.squeeze(0) if volume.dim() == 3 else out


def back_project_3d_torch(sinogram, t_sorted_arg, M, b, src, dst, n_x, n_y, n_z):
    M, b = single_affine(M, b)
    require_cuda(sinogram, src, dst, M, b)
    Mi = inverse(M)
    sino = sinogram.contiguous()
    if isinstance(t_sorted_arg, (tuple, list)):
        t16, ts, tsc = t_sorted_arg
        out = _C.back_project_3d_compressed_cuda(sino, t16, ts, tsc, src, dst, Mi, b, n_x, n_y, n_z)
    else:
        out = _C.back_project_3d_cuda(sino, t_sorted_arg, src, dst, Mi, b, n_x, n_y, n_z)
    return out.squeeze(0) if sinogram.dim() == 1 else out
