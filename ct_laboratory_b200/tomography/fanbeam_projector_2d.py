"""2-D fan-beam geometry and projector class.

``build_fanbeam_2d_geometry`` (ct_laboratory_b200/ray_geometry.py) returns
the same rays as the reference's (tomography/fanbeam_projector_2d.py:6-82),
ordered [view][cell].
"""
from __future__ import annotations

import torch

from ..ray_geometry import build_fanbeam_2d_geometry
from .ct_projector_2d_module import CTProjector2DModule
from .gather import panels_from_lines_2d
from .standard_image_transform import standard_image_transform_2d

__all__ = ["build_fanbeam_2d_geometry", "FanBeam2DProjector"]


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
