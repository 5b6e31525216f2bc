"""2-D fan-beam geometry and projector class.

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

from .ct_projector_2d_module import CTProjector2DModule
from .gather import panels_from_lines_2d
from .standard_image_transform import standard_image_transform_2d

__all__ = ["build_fanbeam_2d_geometry", "FanBeam2DProjector"]


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


class FanBeam2DProjector(CTProjector2DModule):
    """Fan-beam projector (reference fanbeam_projector_2d.py:85-173)."""

    def __init__(self, n_row, n_col, n_view, n_det, sid, sdd, det_spacing=1.0, pixel_size=1.0, angle_offset=0.0,
                 backend="cuda", device=None, precomputed_intersections=False, deterministic_adjoint=False):
        src, dst = build_fanbeam_2d_geometry(n_view=n_view, n_det=n_det, sid=sid, sdd=sdd, det_spacing=det_spacing,
                                             angle_offset=angle_offset, image_center_xy=(0.0, 0.0))
        M, b = standard_image_transform_2d(n_x=n_row, n_y=n_col, s_x=pixel_size, s_y=pixel_size)
        if device is None:
            device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
        panels = None
        if deterministic_adjoint:  # one detector line per view
            panels = panels_from_lines_2d(src, dst, [v * n_det for v in range(n_view)], n_det, 1, device=device)
        super().__init__(n_row=n_row, n_col=n_col, M=M.to(device), b=b.to(device), src=src.to(device),
                         dst=dst.to(device), backend=backend, precomputed_intersections=precomputed_intersections,
                         panels=panels, deterministic_adjoint=deterministic_adjoint)
        self.n_view, self.n_det = n_view, n_det
        self.sid, self.sdd = sid, sdd
        self.det_spacing, self.pixel_size, self.angle_offset = det_spacing, pixel_size, angle_offset
        self.device = device
