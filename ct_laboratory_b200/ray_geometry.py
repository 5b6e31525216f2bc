"""Ray geometry of the fan-beam and cone-beam scans, in plain torch / numpy.

Self-contained on purpose (no import of the package or its native library):
the projector classes use these builders, and the reference CPU arm of the
benchmark loads this file by path to build the same rays without mapping
libctlab_b200.so.

``build_conebeam_3d_geometry`` returns the same rays as the reference's
(tomography/conebeam_projector_3d.py:6-96), evaluated with the same float32
torch operations: circular source orbit of radius sid in the z = cz plane,
flat detector at sdd - sid beyond the isocentre with u along the in-plane
perpendicular and v along +z, rays ordered [view][det_v][det_u].

``build_fanbeam_2d_geometry`` returns the same rays as the reference's
(tomography/fanbeam_projector_2d.py:6-82): view angles
linspace(0, 2*pi - 2*pi/n_view, n_view) (float32) + offset, source at radius
sid, flat detector centred at distance sdd - sid beyond the isocentre,
cells (i - (n_det-1)/2) * spacing along the detector, rays ordered
[view][cell].  Per-view quantities are evaluated in double precision and
rounded to float32 once, as the reference's Python loop does; the cells of a
view are evaluated as one numpy float64 vector instead of a Python loop.
"""
from __future__ import annotations

import math

import numpy as np
import torch

__all__ = ["build_conebeam_3d_geometry", "build_fanbeam_2d_geometry"]


def build_conebeam_3d_geometry(n_view, det_nx, det_ny, sid, sdd, det_spacing=1.0, angle_offset=0.0,
                               volume_center_xyz=(0.0, 0.0, 0.0), device=None):
    """Rays of a circular cone-beam scan, [n_view * det_ny * det_nx, 3] each.
    `device` (an addition; default the host, as the reference) builds them
    directly on a GPU, where large scans take milliseconds instead of seconds
    (the same formulas; the device's cos / sin may round differently)."""
    cx, cy, cz = volume_center_xyz
    ang = torch.linspace(0, 2 * math.pi - 2 * math.pi / n_view, n_view, dtype=torch.float32,
                         device=device) + angle_offset
    cos_t, sin_t = torch.cos(ang), torch.sin(ang)
    view = lambda t: t.view(n_view, 1, 1)  # noqa: E731
    sx, sy = view(cx + sid * cos_t), view(cy + sid * sin_t)
    sz = torch.full_like(sx, cz)
    dcx, dcy = view(cx - (sdd - sid) * cos_t), view(cy - (sdd - sid) * sin_t)
    dcz = torch.full_like(dcx, cz)
    # in-plane unit vector perpendicular to the central ray
    px, py = -(dcy - sy), (dcx - sx)
    norm = torch.sqrt(px * px + py * py)
    px, py = px / norm, py / norm
    pz = torch.zeros_like(px)
    U = ((torch.arange(det_nx, dtype=torch.float32, device=device) - (det_nx - 1) / 2.0) * det_spacing) \
        .unsqueeze(0).expand(det_ny, det_nx)
    V = ((torch.arange(det_ny, dtype=torch.float32, device=device) - (det_ny - 1) / 2.0) * det_spacing) \
        .unsqueeze(1).expand(det_ny, det_nx)
    cell_x = dcx + px * U + 0.0 * V
    cell_y = dcy + py * U + 0.0 * V
    cell_z = dcz + pz * U + 1.0 * V
    shape = (n_view, det_ny, det_nx)
    src = torch.stack([sx.expand(shape), sy.expand(shape), sz.expand(shape)], dim=-1).reshape(-1, 3)
    dst = torch.stack([cell_x, cell_y, cell_z], dim=-1).reshape(-1, 3)
    return src, dst


def build_fanbeam_2d_geometry(n_view, n_det, sid, sdd, det_spacing=1.0, angle_offset=0.0,
                              image_center_xy=(0.0, 0.0)):
    cx, cy = image_center_xy
    angles = torch.linspace(0, 2 * math.pi - 2 * math.pi / n_view, n_view) + angle_offset
    cell = (np.arange(n_det, dtype=np.float64) - (n_det - 1) / 2.0) * det_spacing
    srcs, dsts = [], []
    for theta in angles.tolist():
        c, s = math.cos(theta), math.sin(theta)
        sx, sy = cx + sid * c, cy + sid * s
        dcx, dcy = cx - (sdd - sid) * c, cy - (sdd - sid) * s
        px, py = -(dcy - sy), (dcx - sx)
        norm = math.sqrt(px ** 2 + py ** 2)
        if norm < 1e-12:
            continue  # degenerate view
        px, py = px / norm, py / norm
        d = np.empty((n_det, 2), dtype=np.float64)
        d[:, 0] = dcx + cell * px
        d[:, 1] = dcy + cell * py
        srcs.append(np.broadcast_to(np.array([sx, sy]), (n_det, 2)))
        dsts.append(d)
    if not srcs:
        return torch.empty((0, 2), dtype=torch.float32), torch.empty((0, 2), dtype=torch.float32)
    src = torch.from_numpy(np.ascontiguousarray(np.concatenate(srcs), dtype=np.float32))
    dst = torch.from_numpy(np.ascontiguousarray(np.concatenate(dsts), dtype=np.float32))
    return src, dst
