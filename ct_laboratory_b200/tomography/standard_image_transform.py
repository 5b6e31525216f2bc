"""Voxel-index -> world affine of a centred grid.

Same contract as the reference's standard_image_transform_{2d,3d}
(tomography/standard_image_transform.py:3-50): M = diag(s) and
b = -(n-1)/2 * s, so voxel centre (n-1)/2 maps to the origin.
"""
from __future__ import annotations

import torch

__all__ = ["standard_image_transform_3d", "standard_image_transform_2d"]


def _centred(ns, ss, device=None):
    M = torch.diag(torch.tensor([float(s) for s in ss], dtype=torch.float32))
    b = torch.tensor([-((n - 1) / 2.0) * s for n, s in zip(ns, ss)], dtype=torch.float32)
    if device is not None:
        M, b = M.to(device), b.to(device)
    return M, b


def standard_image_transform_3d(n_x, n_y, n_z, s_x, s_y, s_z, device=None):
    return _centred((n_x, n_y, n_z), (s_x, s_y, s_z), device)


def standard_image_transform_2d(n_x, n_y, s_x, s_y):
    return _centred((n_x, n_y), (s_x, s_y))
