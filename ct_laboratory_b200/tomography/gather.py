"""Deterministic (voxel-driven gather) adjoint, 3-D and 2-D.

``back_project_3d_gather_cuda`` computes A^T y by gathering per voxel instead
of scattering with atomics (ctlab_back_project_3d_gather): the result is
bitwise reproducible and is the exact transpose of the forward walk with the
crossing voxel rule.  It needs the rays grouped into flat detector panels,
described by ``panels_from_grid``.

``back_project_2d_gather_cuda`` is the 2-D one: the image is the
one-voxel-thick volume [n_row, n_col, 1] and the rays lie in its z = 0
plane, where the 3-D arithmetic reduces to the 2-D walk's (every term of the
third axis is an exact zero: the z difference, its products in the affine
and in |v|^2, and the z plane parameters, which are absent), so the gathered
lengths are bitwise the 2-D crossing-rule segments.  Each detector line (a
fan-beam view, a StaticCT module lit by one source) is a one-row panel
(``panels_from_lines_2d``).
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _native as N
from ._common import inverse, require_cuda

__all__ = ["PANEL_DTYPE", "panels_from_grid", "back_project_3d_gather_cuda", "embed_2d_geometry",
           "panels_from_lines_2d", "back_project_2d_gather_cuda"]

# numpy mirror of ctlab_panel (include/ctlab_b200.h), 96 bytes
PANEL_DTYPE = np.dtype([("src", "<f4", 3), ("origin", "<f4", 3), ("eu", "<f4", 3), ("ev", "<f4", 3),
                        ("n", "<f4", 3), ("pad", "<i4"), ("first_ray", "<i8"), ("u_stride", "<i8"),
                        ("v_stride", "<i8"), ("n_u", "<i4"), ("n_v", "<i4")])
assert PANEL_DTYPE.itemsize == 96


def panels_from_grid(src, dst, first_rays, n_u, n_v, u_stride, v_stride, device=None, check=True):
    """Panel table for groups of rays laid out as cell grids.

    first_rays : ray index of cell (0, 0) of every panel
    n_u, n_v   : cells per row / rows per panel
    u_stride, v_stride : ray-index steps between columns / rows
    Every ray of a panel must share the panel's source, and the cell centres
    must form an affine grid (checked, to 1e-3 cell)."""
    src64 = src.detach().double().cpu()
    dst64 = dst.detach().double().cpu()
    first = torch.as_tensor(np.asarray(first_rays, dtype=np.int64))
    S = src64[first]
    O = dst64[first]
    last_u = first + (n_u - 1) * u_stride
    last_v = first + (n_v - 1) * v_stride
    du = (dst64[last_u] - O) / max(n_u - 1, 1)
    dv = (dst64[last_v] - O) / max(n_v - 1, 1)
    if n_u == 1 or n_v == 1:
        # a single row/column: complete the plane with the direction normal to
        # the row and to the central ray
        axis = du if n_u > 1 else dv
        other = torch.linalg.cross(axis, O - S)
        other = other / other.norm(dim=1, keepdim=True).clamp_min(1e-30) * axis.norm(dim=1, keepdim=True)
        if n_u == 1:
            du = other
        else:
            dv = other
    nrm = torch.linalg.cross(du, dv)
    nrm = nrm / nrm.norm(dim=1, keepdim=True)
    g00, g01, g11 = (du * du).sum(1), (du * dv).sum(1), (dv * dv).sum(1)
    det = g00 * g11 - g01 * g01
    eu = (g11[:, None] * du - g01[:, None] * dv) / det[:, None]
    ev = (g00[:, None] * dv - g01[:, None] * du) / det[:, None]
    if check:
        ju = torch.arange(n_u, dtype=torch.int64)
        jv = torch.arange(n_v, dtype=torch.int64)
        ray = first[:, None, None] + jv[None, :, None] * v_stride + ju[None, None, :] * u_stride
        model = O[:, None, None, :] + ju[None, None, :, None] * du[:, None, None, :] + \
            jv[None, :, None, None] * dv[:, None, None, :]
        P = dst64[ray.reshape(-1)].view_as(model)
        a = ((P - O[:, None, None, :]) * eu[:, None, None, :]).sum(-1) - ju[None, None, :]
        c = ((P - O[:, None, None, :]) * ev[:, None, None, :]).sum(-1) - jv[None, :, None]
        if float(a.abs().max()) > 1e-3 or float(c.abs().max()) > 1e-3 or \
                float((P - model).abs().max()) > 1e-3 * float(du.norm(dim=1).min()):
            raise ValueError("rays do not form flat-panel cell grids")
        if not torch.equal(src64[ray.reshape(-1)].view_as(model), S[:, None, None, :].expand_as(model)):
            raise ValueError("every ray of a panel must share the panel's source")
    arr = np.zeros(len(first), dtype=PANEL_DTYPE)
    arr["src"], arr["origin"] = S.numpy(), O.numpy()
    arr["eu"], arr["ev"], arr["n"] = eu.numpy(), ev.numpy(), nrm.numpy()
    arr["first_ray"] = first.numpy()
    arr["u_stride"], arr["v_stride"] = u_stride, v_stride
    arr["n_u"], arr["n_v"] = n_u, n_v
    t = torch.from_numpy(arr.view(np.uint8).copy())
    return t.to(device) if device is not None else t


def back_project_3d_gather_cuda(sinogram, src, dst, M, b, n_x, n_y, n_z, panels, M_inv=None):
    """Deterministic A^T y, [B, n_x, n_y, n_z] (or [n_x, n_y, n_z] for 1-D y)."""
    require_cuda(sinogram, src, dst, M, b, panels)
    M = M.to(torch.float32).contiguous()
    Mi = inverse(M) if M_inv is None else M_inv
    sino = sinogram.contiguous()
    batch, n_ray = (1, sino.shape[0]) if sino.dim() == 1 else sino.shape
    if panels.dtype != torch.uint8 or panels.numel() % PANEL_DTYPE.itemsize:
        raise RuntimeError("panels must be the uint8 table from panels_from_grid")
    out = torch.empty((batch, n_x, n_y, n_z), device=sino.device, dtype=torch.float32)
    # the ray table: each ray's set-up once, 32 bytes per ray
    table = torch.empty((max(int(n_ray), 1), 8), device=sino.device, dtype=torch.float32)
    with torch.cuda.device(sino.device):
        N.call("ctlab_back_project_3d_gather_ws", N.ptr(sino), batch, n_ray, N.ptr(src), N.ptr(dst), N.ptr(M),
               N.ptr(Mi), N.ptr(b), n_x, n_y, n_z, N.ptr(panels), panels.numel() // PANEL_DTYPE.itemsize, N.ptr(out),
               N.ptr(table), N.stream_of(sino))
    return out.squeeze(0) if sinogram.dim() == 1 else out


def embed_2d_geometry(src, dst, M, b):
    """The 2-D geometry as the z = 0 plane of a one-voxel-thick volume:
    src3, dst3 [n_ray, 3], M3 [3, 3] (z scale 1), b3 [3]."""
    z = torch.zeros((src.shape[0], 1), dtype=torch.float32, device=src.device)
    src3 = torch.cat([src.to(torch.float32), z], 1).contiguous()
    dst3 = torch.cat([dst.to(torch.float32), z], 1).contiguous()
    M3 = torch.eye(3, dtype=torch.float32, device=M.device)
    M3[:2, :2] = M.to(torch.float32)
    b3 = torch.cat([b.to(torch.float32).reshape(2), torch.zeros(1, dtype=torch.float32, device=b.device)])
    return src3, dst3, M3.contiguous(), b3.contiguous()


def panels_from_lines_2d(src, dst, first_rays, n_cells, cell_stride=1, device=None, check=True):
    """Panel table for 2-D rays laid out as detector lines: ``first_rays`` the
    ray of each line's first cell, ``n_cells`` cells per line, ``cell_stride``
    the ray-index step between cells (a fan-beam view, a StaticCT module lit
    by one source).  Every ray of a line must share its source."""
    z = torch.zeros((src.shape[0], 1), dtype=torch.float64, device=src.device)
    src3 = torch.cat([src.to(torch.float64), z], 1)
    dst3 = torch.cat([dst.to(torch.float64), z], 1)
    return panels_from_grid(src3, dst3, first_rays, n_cells, 1, cell_stride, 0, device=device, check=check)


def back_project_2d_gather_cuda(sinogram, geometry3, n_row, n_col, panels):
    """Deterministic 2-D A^T y, [B, n_row, n_col] (or [n_row, n_col] for 1-D
    y); ``geometry3`` from embed_2d_geometry."""
    src3, dst3, M3, b3 = geometry3
    out = back_project_3d_gather_cuda(sinogram, src3, dst3, M3, b3, n_row, n_col, 1, panels)
    return out.reshape(*out.shape[:-1])
